"""The oracle's serial-order gather (or_set_serial_order) on several threads reproduces the
serial loop of bond_system.jl:285-297 bit for bit: force density, bond states, active-bond
counts, damage and (CMat) deformation gradient and Cauchy stress, through fracture, several
parameter sets, the surface correction and CMat kills. The threads backend's chunked scatter
differs from it only in summation order."""
import numpy as np
import pytest

import oracle as O
import pdcuda as pd
from helpers import cube_body, deform, oracle_bcs, oracle_body, plate_body

FIELDS = ("b_int", "bond_active", "n_active", "damage", "u", "v")


def snapshot(ob):
    out = {f: np.array(getattr(ob, f)) for f in FIELDS}
    if ob.defgrad is not None:
        out["defgrad"] = np.array(ob.defgrad)
        out["cauchy"] = np.array(ob.cauchy)
    return out


def run(body, threads, serial_order, steps):
    O.set_threads(threads)
    O.set_serial_order(serial_order)
    try:
        ob = oracle_body(body)
        dt = ob.stable_timestep(0.7)
        ob.force_density(0.0, dt)
        assert ob.run_vv(1, steps, dt, oracle_bcs(body, 1, steps, dt)) == 0
        return snapshot(ob)
    finally:
        O.set_threads(1)
        O.set_serial_order(False)


def bodies():
    yield "osb-plate", plate_body(pd.OSBMaterial(), nx=24, ny=12, nz=3, nu=0.25)
    yield "osb-esc", plate_body(pd.OSBMaterial(correction=pd.EnergySurfaceCorrection), nx=20,
                                ny=10, nz=3, nu=0.25)
    yield "cmat-svk", plate_body(pd.CMaterial(), nx=20, ny=10, nz=3, nu=0.25)
    yield "cmat-nh", plate_body(pd.CMaterial(model=pd.NeoHooke()), nx=20, ny=10, nz=3, nu=0.25)
    pos, vol = pd.uniform_box(1.0, 0.5, 0.25, 0.0625)
    body = pd.Body(pd.OSBMaterial(), pos, vol)
    pd.point_set(body, "a", where=lambda p: p[0] < 0)
    pd.point_set(body, "b", where=lambda p: p[0] >= 0)
    pd.material(body, "a", horizon=3.015 * 0.0625, rho=8000.0, E=210e9, Gc=1e3, nu=0.25)
    pd.material(body, "b", horizon=3.015 * 0.0625, rho=2700.0, E=70e9, Gc=1e3, nu=0.25)
    pd.velocity_ic(body, "a", "x", -20.0)
    yield "osb-two-sets", body


@pytest.mark.parametrize("name,body", list(bodies()), ids=lambda v: v if isinstance(v, str) else "")
def test_serial_order_gather_equals_serial_loop(name, body):
    ref = run(body, 1, False, 80)
    got = run(body, 8, True, 80)
    for f in ref:
        assert np.array_equal(got[f], ref[f], equal_nan=True), f
    broken = int(np.count_nonzero(ref["bond_active"] == 0))
    print(f"{name}: {broken} bonds broken, serial-order gather on 8 threads bit-identical")


def test_chunked_scatter_differs_only_in_order():
    body = cube_body(pd.OSBMaterial(), n=9)
    u = deform(body._pos)
    res = []
    for th, so in ((1, False), (8, False), (8, True)):
        O.set_threads(th)
        O.set_serial_order(so)
        try:
            ob = oracle_body(body)
            ob.pos[:] = body._pos + u
            ob.force_density()
            res.append(np.array(ob.b_int))
        finally:
            O.set_threads(1)
            O.set_serial_order(False)
    assert np.array_equal(res[2], res[0])
    scale = np.abs(res[0]).max()
    assert np.abs(res[1] - res[0]).max() <= 1e-12 * scale
