"""VTK export in the reference's layout, read back the way the reference's reader reads it."""
import os

import numpy as np

from pdcuda.vtk import VtkExport, write_pvtu
from vtk_read import find_vtk_files, read_vtk


class FakeDev:
    def __init__(self, n, seed=0):
        rng = np.random.default_rng(seed)
        self.f = {"position": rng.standard_normal((3, n)), "displacement": rng.standard_normal((3, n)),
                  "damage": rng.uniform(0, 1, n), "n_active_bonds": rng.integers(0, 100, n)}

    def field(self, name):
        return self.f[name]


def test_pvtu_round_trip(tmp_path):
    n = 257
    dev = FakeDev(n)
    fb = str(tmp_path / "timestep_7")
    f = write_pvtu(fb, dev.field("position"), {"displacement": dev.field("displacement"),
                                               "damage": dev.field("damage"),
                                               "n_active_bonds": dev.field("n_active_bonds")}, 1.5e-3)
    assert os.path.isfile(f) and os.path.isfile(os.path.join(fb, "timestep_7_1.vtu"))
    d = read_vtk(f)
    assert np.array_equal(d["position"], dev.field("position"))
    assert np.array_equal(d["displacement"], dev.field("displacement"))
    assert np.array_equal(d["damage"], dev.field("damage"))
    assert np.array_equal(d["n_active_bonds"], dev.field("n_active_bonds"))
    assert d["n_active_bonds"].dtype == np.int64
    assert d["time"][0] == 1.5e-3


def test_export_cadence_and_names(tmp_path):
    dev = FakeDev(10)
    ex = VtkExport(str(tmp_path), freq=5)
    for step in range(0, 13):
        ex(step, step * 0.1, dev)
    files = find_vtk_files(str(tmp_path / "vtk"))
    assert [os.path.basename(f) for f in files] == ["timestep_0.pvtu", "timestep_5.pvtu",
                                                    "timestep_10.pvtu"]
    d = read_vtk(files[-1])
    assert set(d) == {"position", "displacement", "damage", "time"}
