"""EnergySurfaceCorrection on the device (csrc/pd_esc.cu and the ESC variants of the BB / OSB
force kernels) against the CPU restatement (oracle/pd_oracle.c: or_esc_*) and the reference's
known answers (test_bond_based.jl:184-211, test_bond_system_corrections.jl,
test_analytic_solutions.jl:96-107). The multiplication factors are computed in the
reference's order and equal the restatement bit for bit; the bond factors go through atan /
acos / cos / sin, whose last bits may differ between CUDA and the C library."""
import math

import numpy as np
import pytest

import pdcuda as pd
from pdcuda.halo import Partition, PartitionedBody
from dr import OracleDR
from helpers import oracle_bcs, oracle_body, plate_body
from test_dr_host import elongation_error
from test_esc_host import ESC, databc_bar, two_points, unit_box

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


def test_two_point_golden_on_device():
    dev = pd.DeviceBody(two_points(), precision="fp64")
    mf, sc = dev.surface_correction()
    assert sc == pytest.approx([3.1808625617603665] * 2, rel=1e-14)
    x = dev.body._pos.copy()
    x[1, 0] = 1.0015
    dev.set_state(position=x)
    dev.force(0.0, 0.0)
    b12 = 3.1808625617603665 * 18 * 210e9 / (3 * (1 - 2 * 0.25)) / (math.pi * 1.5 ** 4) * 0.0015
    b = dev.field("b_int")
    assert b[0] == pytest.approx([b12, -b12], rel=1e-12)
    assert not b[1:].any()


@pytest.mark.parametrize("name", ["BB", "OSB"])
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_factors_match_oracle(name, prec):
    mat = pd.BBMaterial(correction=ESC) if name == "BB" else pd.OSBMaterial(correction=ESC)
    body = unit_box(mat)
    ob = oracle_body(body)
    dev = pd.DeviceBody(body, precision=prec)
    mf, sc = dev.surface_correction()
    assert np.array_equal(mf, ob.mfactor)
    ref = ob.scfactor[:ob.n_bonds]
    if prec == "fp64":
        assert rel(sc, ref) <= 4e-16
    else:
        assert np.array_equal(sc, ref.astype(np.float32).astype(np.float64)) or \
            rel(sc, ref) <= 1.2e-7


def test_averaged_lame_factors_match_oracle():
    pos = np.zeros((3, 10))
    pos[0] = np.arange(10.0)
    body = pd.Body(pd.BBMaterial(correction=ESC), pos, np.linspace(1.1, 2.0, 10))
    pd.point_set(body, "left", where=lambda p: p[0] < 4.5)
    pd.point_set(body, "right", where=lambda p: p[0] > 4.5)
    pd.material(body, "left", horizon=1.01, rho=8000, E=105e9, nu=0.25)
    pd.material(body, "right", horizon=1.01, rho=8000, E=2 * 105e9, nu=0.25)
    mf, _ = pd.DeviceBody(body, precision="fp64").surface_correction()
    assert np.array_equal(mf, oracle_body(body).mfactor)


def oracle_with_device_factors(body, dev):
    """The restatement with the device's bond factors (the factors are compared on their own
    in test_factors_match_oracle): the rest of the path can then match bit for bit."""
    ob = oracle_body(body)
    ob.scfactor[:ob.n_bonds] = dev.surface_correction()[1]
    return ob


@pytest.mark.parametrize("name", ["BB", "OSB"])
def test_trajectories_match_oracle(name):
    mat = pd.BBMaterial(correction=ESC) if name == "BB" else pd.OSBMaterial(correction=ESC)
    body = plate_body(mat, nx=24, ny=12, nz=3, nu=None if name == "BB" else 0.25)
    ob = oracle_with_device_factors(body, pd.DeviceBody(body, precision="fp64"))
    dt = ob.stable_timestep(0.7)
    ob.force_density(0.0, dt)
    assert ob.run_vv(1, 100, dt, oracle_bcs(body, 1, 100, dt)) == 0
    for prec, mapping, tol in (("fp64", (0,), 0.0), ("fp64", (4,), 1e-10), ("fp32", (8,), 1e-5),
                               ("fp32", (1,), 1e-5)):
        dev = pd.DeviceBody(body, precision=prec)
        dev.set_mapping(*mapping)          # after the correction: its factors follow the layout
        assert dev.stable_timestep(0.7) == dt
        dev.force(0.0, dt)
        dev.run(1, 100, dt)
        assert rel(dev.field("displacement").T, ob.u) <= tol, (prec, mapping)
        if prec == "fp64":
            assert np.array_equal(dev.field("bond_active"), ob.bond_active[:ob.n_bonds])
        dev.close()
    assert np.count_nonzero(ob.bond_active[:ob.n_bonds] == 0) > 0


def test_data_condition_bar_band_by_relaxation():
    body = databc_bar(1 / 30)
    dev = pd.submit(pd.Job(body, pd.DynamicRelaxation(steps=1000), mapping=(0,)))
    err = elongation_error(dev.field("displacement").T, body)
    assert err < 0.2      # the reference's band (it measures 13 % at this spacing)
    ob = oracle_with_device_factors(body, dev)
    dr = OracleDR(ob, 1.0)
    bcs = oracle_bcs(body, 1, 1000, 1.0)
    ob.force_density(0.0, 1.0)
    for k in range(1, 1001):
        dr.step(k, bcs)
    # the serial damping sums and the correction in the reference's order: the same bits
    assert np.array_equal(dev.field("displacement").T, ob.u)


@pytest.mark.parametrize("prec,mapping", [("fp64", (0,)), ("fp32", (8,))])
def test_partitions_with_correction(prec, mapping):
    body = plate_body(pd.OSBMaterial(correction=ESC), nx=24, ny=12, nz=3, nu=0.25)
    dev = pd.DeviceBody(body, precision=prec)
    dev.set_mapping(*mapping)
    dt = dev.stable_timestep(0.7)
    dev.force(0.0, dt)
    dev.run(1, 80, dt)
    parts = [Partition(body, 3, p, prec, decomposition="slabs") for p in range(3)]
    for p in parts:
        p.dev.set_mapping(*mapping)
    pb = PartitionedBody(parts)
    assert pb.stable_timestep(0.7) == dt
    pb.force(0.0, dt)
    pb.run(1, 80, dt)
    for f in ("displacement", "velocity", "damage"):
        assert np.array_equal(pb.field(f), dev.field(f)), f
    assert np.array_equal(pb.field("bond_active"), dev.field("bond_active"))
    pb.close()
    dev.close()


@pytest.mark.parametrize("name", ["BB", "OSB"])
def test_two_row_kernels_equal_one_row_with_correction(name):
    """pipe 4 (two rows of gathers in flight) and pipe 0 add the same terms in the same order."""
    mat = pd.BBMaterial(correction=ESC) if name == "BB" else pd.OSBMaterial(correction=ESC)
    body = plate_body(mat, nx=24, ny=12, nz=3, nu=None if name == "BB" else 0.25)
    res = []
    for pipe in (0, 4):
        dev = pd.DeviceBody(body, precision="fp32")
        dev.set_mapping(1)
        dev.set_pipeline(pipe)
        dt = dev.stable_timestep(0.7)
        dev.force(0.0, dt)
        dev.run(1, 60, dt)
        res.append((dev.field("displacement"), dev.field("bond_active")))
        dev.close()
    assert np.array_equal(res[0][0], res[1][0]) and np.array_equal(res[0][1], res[1][1])
