"""Edge cases of the bond system through the C ABI, against the oracle: points without bonds
(an isolated point: its damage is 1 - 0/0, NaN, as in calc_damage!, bond_system.jl:338-343;
OSB returns early with a zero weighted volume, ordinary_state_based.jl:128-149; CMat kills it,
its shape tensor being singular, correspondence.jl:288-298), a pair of points with one bond
each, and a point whose only bond breaks. FP64 in the serial order bit for bit, FP32 within
its tolerance, over a loaded run with fracture.
"""
import numpy as np
import pytest

import pdcuda as pd
from helpers import oracle_bcs, oracle_body

pytestmark = pytest.mark.gpu

MATERIALS = {
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


@pytest.mark.parametrize("name", list(MATERIALS))
def test_ragged_bodies_match_the_oracle(name):
    body = ragged_body(MATERIALS[name]())
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
