"""Edge cases of the reference's bond system on the device: coinciding points are rejected
(check_point_duplicates, bond_system.jl:125-132: "point duplicate found"), and a point without
bonds runs like the reference's one: no force, its step is not the minimum, its damage is
1 - 0/0 (bond_system.jl:338-343), against the FP64 oracle. A ragged body (a lattice, an
isolated point and a pair of points with one bond each that breaks under a pull) matches the
oracle over a loaded run for BB, OSB and CMat with both stabilisations: OSB returns early for
a zero weighted volume (ordinary_state_based.jl:128-149), CMat kills points whose shape tensor
is singular (correspondence.jl:288-298)."""
import numpy as np
import pytest

import pdcuda as pd
from helpers import oracle_bcs, oracle_body

pytestmark = pytest.mark.gpu

MATS = {"BB": (pd.BBMaterial, None), "OSB": (pd.OSBMaterial, 0.25), "C": (pd.CMaterial, 0.25)}


def test_point_duplicates_are_rejected():
    pos = np.array([[0.0, 1.0, 1.0], [0.0, 0.0, 0.0], [0.0, 0.0, 0.0]])
    body = pd.Body(pd.BBMaterial(), pos, np.ones(3))
    pd.material(body, horizon=1.5, rho=1.0, E=1.0)
    with pytest.raises(Exception, match="point duplicate"):
        pd.DeviceBody(body)


@pytest.mark.parametrize("name", ["BB", "OSB", "C"])
def test_point_without_bonds(name):
    mat, nu = MATS[name]
    pos, vol = pd.uniform_box(4e-3, 4e-3, 4e-3, 1e-3)
    far = np.array([[1.0], [1.0], [1.0]])           # out of every horizon
    pos = np.concatenate([pos, far], axis=1)
    vol = np.concatenate([vol, [1e-9]])
    body = pd.Body(mat(), pos, vol)
    kw = dict(horizon=3.015e-3, rho=2700.0, E=70e9, Gc=100.0)
    if nu is not None:
        kw["nu"] = nu
    pd.material(body, **kw)
    pd.point_set(body, "far", [body.n_points - 1])
    pd.point_set(body, "corner", [0])
    pd.velocity_ic(body, "far", "x", 3.0)
    pd.velocity_ic(body, "corner", "y", 0.5)
    ob = oracle_body(body)
    dt = ob.stable_timestep(0.7)
    ob.force_density(0.0, dt)
    assert ob.run_vv(1, 20, dt, []) == 0
    dev = pd.DeviceBody(body, precision="fp64")
    dev.set_mapping(0)
    assert dev.stable_timestep(0.7) == dt and np.isfinite(dt)
    dev.force(0.0, dt)
    dev.run(1, 20, dt)
    u = dev.field("displacement").T
    if name == "C":
        assert np.max(np.abs(u - ob.u)) <= 1e-10 * np.max(np.abs(ob.u))
    else:
        assert np.array_equal(u, ob.u)
    assert u[-1, 0] == pytest.approx(3.0 * 20 * dt, rel=1e-12)   # the free point drifts
    assert not dev.field("b_int")[:, -1].any()
    d_dev, d_ob = dev.field("damage"), ob.damage
    assert np.isnan(d_dev[-1]) and np.isnan(d_ob[-1])
    assert np.array_equal(d_dev[:-1], d_ob[:-1])
    dev.close()
    # the FP32 form as well
    dev = pd.DeviceBody(body, precision="fp32")
    dev.force(0.0, dt)
    dev.run(1, 20, dt)
    u32 = dev.field("displacement").T
    assert np.max(np.abs(u32 - ob.u)) <= 1e-5 * np.max(np.abs(ob.u))
    assert not dev.field("b_int")[:, -1].any()
    dev.close()


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_near_critical_bonds_are_counted(prec):
    body = pd.Body(pd.BBMaterial(), np.array([[0.0, 1.0], [0.0, 0.0], [0.0, 0.0]]), np.ones(2))
    pd.material(body, horizon=1.5, rho=1.0, E=1.0, Gc=1.0)
    epsc = body.point_params[0].epsilon_c
    dev = pd.DeviceBody(body, precision=prec)
    for x, expected in ((1.0 + epsc, 2), (1.0 + 2 * epsc, 0), (1.0, 0)):
        pos = body._pos.copy()
        pos[1, 0] = x
        if prec == "fp64":
            dev.set_state(position=pos)
        else:
            dev.set_state(displacement=pos - body._pos)
        assert dev.near_critical(1e-12) == expected, x
    assert dev.near_critical(2 * epsc) == 2
    dev.close()


RAGGED_MATERIALS = {
    "BB": lambda: pd.BBMaterial(),
    "OSB": lambda: pd.OSBMaterial(),
    "C": lambda: pd.CMaterial(),
    "C-Wan": lambda: pd.CMaterial(zem=pd.ZEMWan()),
}


def ragged_body(mat):
    """A 6x6x6 lattice, a point far from everything, and a pair of points one spacing apart
    far from both; the lattice's right face is pulled gently along x (no bond of the lattice
    breaks), one point of the pair fast (their bond breaks)."""
    dx = 0.1
    pos, vol = pd.uniform_box(0.6, 0.6, 0.6, dx)
    extra = np.array([[5.0, 5.0, 5.0], [-5.0, -5.0, -5.0], [-5.0 + dx, -5.0, -5.0]]).T
    pos = np.concatenate([pos, extra], axis=1)
    vol = np.concatenate([vol, np.full(3, dx ** 3)])
    body = pd.Body(mat, pos, vol)
    kw = dict(horizon=3.015 * dx, rho=7850.0, E=210e9, Gc=1e6)
    if not isinstance(mat, pd.BBMaterial):
        kw["nu"] = 0.25
    pd.material(body, **kw)
    pd.point_set(body, "right", where=lambda p: (p[0] > 0.2) & (p[0] < 1.0))
    pd.point_set(body, "pair", [body.n_points - 1])
    pd.velocity_bc(lambda t: 0.25, body, "right", "x")
    pd.velocity_bc(lambda t: 30.0, body, "pair", "x")
    return body


@pytest.mark.parametrize("name", list(RAGGED_MATERIALS))
def test_isolated_point_and_breaking_pair(name):
    body = ragged_body(RAGGED_MATERIALS[name]())
    n = body.n_points
    ob = oracle_body(body)
    assert ob.off[n - 2] - ob.off[n - 3] == 0            # the isolated point has no bond
    assert ob.off[n] - ob.off[n - 2] == 2                # the pair: one bond each way
    dt = ob.stable_timestep(0.7)
    steps = 120
    ob.force_density(0.0, dt)
    assert ob.run_vv(1, steps, dt, oracle_bcs(body, 1, steps, dt)) == 0
    dmg = ob.damage.copy()
    assert np.isnan(dmg[n - 3])
    # the pair's bond broke under the pull (CMat: both points are killed at once, their shape
    # tensors being singular), its points are fully damaged
    assert dmg[n - 2] == 1.0 and dmg[n - 1] == 1.0
    assert np.count_nonzero(ob.bond_active[:ob.n_bonds] == 0) == 2
    lattice, pair = np.arange(n - 3), np.array([n - 2, n - 1])
    for prec in ("fp64", "fp32"):
        dev = pd.DeviceBody(body, precision=prec)
        if prec == "fp64":
            dev.set_mapping(0)
        assert dev.stable_timestep(0.7) == dt
        dev.force(0.0, dt)
        dev.run(1, steps, dt)
        u = dev.field("displacement").T
        assert np.array_equal(dev.field("damage"), dmg, equal_nan=True), prec
        assert np.array_equal(dev.field("bond_active"), ob.bond_active[:ob.n_bonds]), prec
        exact = prec == "fp64" and name in ("BB", "OSB")
        tol = 1e-10 if prec == "fp64" else 1e-5
        for part in (lattice, pair):
            if exact:
                assert np.array_equal(u[part], ob.u[part]), prec
            else:
                assert np.abs(u[part] - ob.u[part]).max() <= tol * np.abs(ob.u[part]).max(), prec
        # no force on the isolated point; it never moves
        assert np.all(dev.field("b_int")[:, n - 3] == 0)
        assert np.all(u[n - 3] == 0)
        dev.close()
