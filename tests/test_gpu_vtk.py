"""Job(path=...) writes the reference's VTK files from the device state (Velocity Verlet and
Newton-Krylov jobs)."""
import os

import numpy as np
import pytest

import pdcuda as pd
from helpers import plate_body
from test_nk_host import small_beam
from vtk_read import find_vtk_files, read_vtk

pytestmark = pytest.mark.gpu


def test_velocity_verlet_job_exports(tmp_path):
    body = plate_body(pd.BBMaterial())
    job = pd.Job(body, pd.VelocityVerlet(steps=12), path=str(tmp_path), freq=5,
                 fields=("displacement", "velocity", "damage"))
    dev = pd.submit(job)
    files = find_vtk_files(str(tmp_path / "vtk"))
    assert [os.path.basename(f) for f in files] == ["timestep_0.pvtu", "timestep_5.pvtu",
                                                    "timestep_10.pvtu"]
    d0 = read_vtk(files[0])
    assert np.array_equal(d0["position"], body._pos.T) and np.all(d0["displacement"] == 0)


def test_newton_krylov_job_exports_last_increment(tmp_path):
    body = small_beam()
    nk = pd.NewtonKrylov(steps=2, tol=1e-8, tol_mode="relative", frechet="forward",
                         gmres_restart=50, gmres_maxiter=5000, maxiter=20,
                         preconditioner="block_jacobi")
    dev = pd.submit(pd.Job(body, nk, path=str(tmp_path), freq=1))
    files = find_vtk_files(str(tmp_path / "vtk"))
    assert len(files) == 3
    d = read_vtk(files[-1])
    assert np.array_equal(d["displacement"], dev.field("displacement"))
    assert np.array_equal(d["position"], dev.field("position"))
