"""Edge cases of the reference's bond system on the device: coinciding points are rejected
(check_point_duplicates, bond_system.jl:125-132: "point duplicate found"), and a point without
bonds runs like the reference's one: no force, its step is not the minimum, its damage is
1 - 0/0 (bond_system.jl:338-343), against the FP64 oracle."""
import numpy as np
import pytest

import pdcuda as pd
from helpers import oracle_body

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
