"""The reference's known-answer tests through the C ABI on the GPU."""
import math

import numpy as np
import pytest

import pdcuda as pd

pytestmark = pytest.mark.gpu
PRECS = ["fp64", "fp32"]
TOL = {"fp64": 1e-12, "fp32": 2e-6}


def two_point_body(mat, vol=(1.0, 1.0), **kw):
    pos = np.array([[0.0, 1.0], [0.0, 0.0], [0.0, 0.0]])
    return pd.Body(mat, pos, np.array(vol))


@pytest.mark.parametrize("prec", PRECS)
def test_bb_two_point(prec):
    body = two_point_body(pd.BBMaterial())
    pd.material(body, horizon=1.5, rho=1, E=210e9)
    pd.no_failure(body)
    dev = pd.DeviceBody(body, precision=prec)
    x = body._pos.copy()
    x[1, 0] = 1.0015
    dev.set_state(position=x)
    dev.force(0.0, 0.0)
    E, d = 210e9, 1.5
    b12 = 18 * E / (3 * (1 - 2 * 0.25)) / (math.pi * d ** 4) * 1.0015 * 0.0015 / 1.0015 * 1.0
    b = dev.field("b_int")
    assert b[0, 0] == pytest.approx(b12, rel=TOL[prec])
    assert b[0, 1] == pytest.approx(-b12, rel=TOL[prec])
    assert np.all(b[1:] == 0)


@pytest.mark.parametrize("prec", PRECS)
def test_osb_two_point(prec, golden):
    body = two_point_body(pd.OSBMaterial())
    pd.material(body, horizon=1.5, rho=1, E=210e9, nu=0.25, Gc=1.0)
    pd.no_failure(body)
    dev = pd.DeviceBody(body, precision=prec)
    x = body._pos.copy()
    x[1, 0] = 1.0015
    dev.set_state(position=x)
    dev.force()
    b = dev.field("b_int")
    assert b[0, 0] == pytest.approx(golden["osb_two_point_b12"], rel=TOL[prec])
    assert b[0, 1] == pytest.approx(-golden["osb_two_point_b12"], rel=TOL[prec])


@pytest.mark.parametrize("prec", PRECS)
def test_osb_interface(prec, golden):
    body = two_point_body(pd.OSBMaterial(), vol=(1.0, 2.0))
    pd.point_set(body, "a", [0])
    pd.point_set(body, "b", [1])
    pd.material(body, "a", horizon=1.5, rho=1, E=105e9, nu=0.25, Gc=1.0)
    pd.material(body, "b", horizon=1.5, rho=1, E=210e9, nu=0.25, Gc=1.0)
    pd.no_failure(body)
    dev = pd.DeviceBody(body, precision=prec)
    x = body._pos.copy()
    x[1, 0] = 1.0015
    dev.set_state(position=x)
    dev.force()
    b = dev.field("b_int")
    assert b[0, 0] == pytest.approx(golden["osb_interface_b1"], rel=TOL[prec])
    assert b[0, 1] == pytest.approx(-golden["osb_interface_b2"], rel=TOL[prec])


@pytest.mark.parametrize("prec", PRECS)
def test_correspondence_nhp(prec, golden):
    pos = np.array([[0.0, 1, 0, 0, 2], [0, 0, 1, 0, 2], [0, 0, 0, 1, 2]])
    body = pd.Body(pd.CMaterial(model=pd.NeoHookePenalty()), pos, np.ones(5))
    pd.material(body, horizon=1.5, rho=1, E=1, nu=0.25, Gc=1.0)
    pd.no_failure(body)
    dev = pd.DeviceBody(body, precision=prec)
    x = body._pos.copy()
    x[1, 0] += 0.0015
    dev.set_state(position=x)
    dev.force()
    b = dev.field("b_int")
    tol = 1.5e-8 if prec == "fp64" else 2e-5
    assert np.all(b[:, 4] == 0)
    assert b[:, 0] == pytest.approx(golden["c_nhp_b_int_1"], rel=tol)
    assert b[0, 1] == pytest.approx(golden["c_nhp_b_int_12"], rel=tol)
    assert b[1, 2] == pytest.approx(golden["c_nhp_b_int_23"], rel=tol)
    # isolated point: no bonds, killed (too_much_damage!) and no stress
    assert dev.field("n_active_bonds")[4] == 0


def test_timestep_two_point():
    body = two_point_body(pd.BBMaterial())
    pd.material(body, horizon=1.5, rho=1, E=1, Gc=1)
    dev = pd.DeviceBody(body)
    bc = 18 * 1 / (3 * (1 - 2 * 0.25)) / (math.pi * 1.5 ** 4)
    assert dev.stable_timestep(0.7) == pytest.approx(0.7 * math.sqrt(2 / bc), abs=2.3e-16)
    vv = pd.VelocityVerlet(steps=10)
    pd.submit(pd.Job(body, vv))
    assert vv.dt == pytest.approx(0.7 * math.sqrt(2 / bc), abs=2.3e-16)
    assert vv.end_time == pytest.approx(10 * vv.dt)


def tetra_body(mat=None):
    pos = np.array([[0.0, 1, 0, 0], [0, 0, 1, 0], [0, 0, 0, 1]])
    body = pd.Body(mat or pd.BBMaterial(), pos, np.array([1.1, 1.2, 1.3, 1.4]))
    pd.material(body, horizon=2, rho=1, E=1, Gc=1)
    return body


def test_bond_lists_tetra():
    import ctypes as C
    body = tetra_body()
    lib = pd.lib()
    n = 4
    delta = np.full(n, 2.0)
    nb = C.c_int64()
    assert lib.pd_find_bonds(n, body._pos.ctypes.data, delta.ctypes.data, None, 0, None, None, 0,
                             None, None, None, None, C.byref(nb), 0) == 0
    off = np.zeros(n + 1, np.int64)
    nbr = np.zeros(nb.value, np.int32)
    L = np.zeros(nb.value)
    fp = np.zeros(nb.value, np.uint8)
    assert lib.pd_find_bonds(n, body._pos.ctypes.data, delta.ctypes.data, None, 0, None, None,
                             nb.value, off.ctypes.data, nbr.ctypes.data, L.ctypes.data,
                             fp.ctypes.data, C.byref(nb), 0) == 0
    r2 = math.sqrt(2)
    assert off.tolist() == [0, 3, 6, 9, 12]
    assert nbr.tolist() == [1, 2, 3, 0, 2, 3, 0, 1, 3, 0, 1, 2]
    assert L.tolist() == [1, 1, 1, 1, r2, r2, 1, r2, r2, 1, r2, r2]
    assert fp.all()


@pytest.mark.parametrize("prec", PRECS)
def test_precrack_damage(prec):
    body = tetra_body()
    pd.point_set(body, "a", [0, 1])
    pd.point_set(body, "b", [2, 3])
    pd.precrack(body, "a", "b")
    dev = pd.DeviceBody(body, precision=prec)
    assert dev.field("bond_active")[:6].tolist() == [1, 0, 0, 1, 0, 0]
    assert dev.field("damage") == pytest.approx([2 / 3] * 4)
    assert dev.field("n_active_bonds").tolist() == [1, 1, 1, 1]
    body = tetra_body()
    pd.point_set(body, "a", [0, 1])
    pd.point_set(body, "b", [2, 3])
    pd.precrack(body, "a", "b", update_dmg=False)
    dev = pd.DeviceBody(body, precision=prec)
    assert dev.n_bonds == 4
    assert dev.field("damage").tolist() == [0, 0, 0, 0]


def test_storage_init(golden):
    pos, vol = pd.uniform_box(1, 1, 1, 0.25)
    body = pd.Body(pd.BBMaterial(), pos, vol)
    pd.material(body, horizon=2, rho=1, E=1, Gc=1)
    dev = pd.DeviceBody(body)
    assert dev.n_bonds == golden["bb_storage_bond_count"]
    assert np.all(dev.field("n_active_bonds") == 63)
    assert np.all(dev.field("bond_active") == 1)
    assert np.all(dev.field("damage") == 0)
    for f in ("displacement", "velocity", "velocity_half", "acceleration", "b_int", "b_ext"):
        assert np.all(dev.field(f) == 0)
    assert np.array_equal(dev.field("position"), body.position)
