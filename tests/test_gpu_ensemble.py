"""Ensembles of specimens on one device against the oracle run on every specimen alone,
each with its own CFL step (the reference runs such studies one job after the other)."""
import numpy as np
import pytest

import oracle as O
import pdcuda as pd
from helpers import oracle_bcs, oracle_body

pytestmark = pytest.mark.gpu


def specimen(mat_factory, nx, ny, nz, E, rho, crack_frac, seed, dx=1e-3, filt=False):
    lx, ly, lz = nx * dx, ny * dx, nz * dx
    pos, vol = pd.uniform_box(lx, ly, lz, dx, center=(lx / 2, ly / 2, lz / 2))
    mat = mat_factory()
    body = pd.Body(mat, pos, vol)
    kw = dict(horizon=3.015 * dx, rho=rho, E=E, Gc=100.0)
    if not isinstance(mat, pd.BBMaterial):
        kw["nu"] = 0.3 if isinstance(mat, pd.CMaterial) else 0.25
    pd.material(body, **kw)
    a = crack_frac * lx
    pd.point_set(body, "ca", where=lambda p: (p[1] <= ly / 2) & (p[0] < a))
    pd.point_set(body, "cb", where=lambda p: (p[1] > ly / 2) & (p[0] < a))
    pd.precrack(body, "ca", "cb", update_dmg=not filt)
    pd.point_set(body, "left", where=lambda p: p[0] < 1.5 * dx)
    pd.point_set(body, "right", where=lambda p: p[0] > lx - 1.5 * dx)
    pd.velocity_bc(lambda t: -0.6, body, "left", "x")
    pd.velocity_bc(lambda p, t: 0.6 + 10.0 * p[1] * t, body, "right", "x")
    pd.velocity_ic(lambda p: 0.01 * p[2], body, "all_points", "z")
    return body


def build(mat_factory, filt=False):
    rng = np.random.default_rng(7)
    bodies = []
    for k in range(3):
        nx, ny, nz = int(rng.integers(10, 16)), int(rng.integers(6, 10)), 3
        bodies.append(specimen(mat_factory, nx, ny, nz, E=float(rng.uniform(50e9, 200e9)),
                               rho=float(rng.uniform(2000, 8000)),
                               crack_frac=float(rng.uniform(0.1, 0.4)), seed=k, filt=filt))
    return bodies


@pytest.mark.parametrize("name,factory", [("BB", pd.BBMaterial), ("OSB", pd.OSBMaterial),
                                          ("C", lambda: pd.CMaterial(model=pd.NeoHooke()))])
def test_ensemble_matches_specimens_run_alone(name, factory):
    bodies = build(factory)
    n_steps = 60
    for prec, mapping in (("fp64", 0), ("fp32", 1)):
        ens = pd.Ensemble(bodies, precision=prec, graph_steps=16 if prec == "fp32" else 0)
        ens.dev.set_mapping(mapping)
        ens.run(n_steps)
        for k, b in enumerate(bodies):
            ob = oracle_body(b)
            dt = ob.stable_timestep(0.7)
            assert ens.dt[k] == dt
            ob.force_density(0.0, dt)
            assert ob.run_vv(1, n_steps, dt, oracle_bcs(b, 1, n_steps, dt)) == 0
            u = ens.field("displacement", k).T
            if prec == "fp64":
                if name == "C":
                    assert np.abs(u - ob.u).max() <= 1e-10 * np.abs(ob.u).max()
                else:
                    assert np.array_equal(u, ob.u), (name, k)
                assert np.array_equal(ens.field("bond_active", k), ob.bond_active[:ob.n_bonds])
            else:
                assert np.abs(u - ob.u).max() <= 1e-5 * np.abs(ob.u).max(), (name, k)
        ens.close()


def test_ensemble_rejects_mixed_materials():
    a = specimen(pd.BBMaterial, 8, 6, 3, 70e9, 2700, 0.2, 0)
    b = specimen(pd.OSBMaterial, 8, 6, 3, 70e9, 2700, 0.2, 0)
    with pytest.raises(ValueError):
        pd.Ensemble([a, b])


def test_ensemble_with_filter_cracks_matches_specimens_run_alone():
    """precrack!(...; update_dmg=false) of every specimen: the ensemble merges the k-th crack of
    all specimens into one filter (no bond joins two specimens); bonds and trajectories equal
    those of each specimen alone, bit for bit in serial FP64 order."""
    bodies = build(pd.BBMaterial, filt=True)
    ens = pd.Ensemble(bodies, precision="fp64")
    ens.dev.set_mapping(0)
    ens.run(40)
    for k, b in enumerate(bodies):
        ob = oracle_body(b)
        dt = ob.stable_timestep(0.7)
        ob.force_density(0.0, dt)
        assert ob.run_vv(1, 40, dt, oracle_bcs(b, 1, 40, dt)) == 0
        assert np.array_equal(ens.field("n_neighbors", k), ob.n_neighbors)
        assert np.array_equal(ens.field("displacement", k).T, ob.u)
    ens.close()


@pytest.mark.parametrize("name,factory", [("OSB", pd.OSBMaterial),
                                          ("C", lambda: pd.CMaterial(model=pd.NeoHooke()))])
def test_size_classes_in_one_graph_match_specimens_run_alone(name, factory):
    """Specimens cut into size classes (each class one device body with its own mapping),
    advanced by one CUDA graph per block of steps: every specimen's trajectory is the one it
    has alone — bit for bit in serial FP64 order (CMat within 1e-10: CUDA's and the C library's
    log may differ in the last bit), within the FP32 tolerance with different lane mappings per
    class."""
    rng = np.random.default_rng(11)
    bodies = []
    for k in range(5):
        nx, ny = int(rng.integers(8, 20)), int(rng.integers(5, 10))
        bodies.append(specimen(factory, nx, ny, 3, E=float(rng.uniform(50e9, 200e9)),
                               rho=float(rng.uniform(2000, 8000)),
                               crack_frac=float(rng.uniform(0.1, 0.4)), seed=k))
    n_steps = 48
    refs = []
    for b in bodies:
        ob = oracle_body(b)
        dt = ob.stable_timestep(0.7)
        ob.force_density(0.0, dt)
        assert ob.run_vv(1, n_steps, dt, oracle_bcs(b, 1, n_steps, dt)) == 0
        refs.append((ob, dt))
    for prec in ("fp64", "fp32"):
        ens = pd.Ensemble(bodies, precision=prec, graph_steps=16, classes=3)
        assert len(ens.devs) == 3 and sorted(sum(ens.members, [])) == list(range(5))
        sizes = [max(bodies[k].n_points for k in m) for m in ens.members]
        assert sizes == sorted(sizes)
        if prec == "fp64":
            ens.set_mapping(0)
        else:
            for d, g in zip(ens.devs, (1, 4, 32)):
                d.set_mapping(g)
        launches0 = ens.launch_count()
        ens.run(n_steps)
        assert ens.launch_count() > launches0
        for k, (ob, dt) in enumerate(refs):
            assert ens.dt[k] == dt
            u = ens.field("displacement", k).T
            if prec == "fp64":
                if name == "C":
                    assert np.abs(u - ob.u).max() <= 1e-10 * np.abs(ob.u).max()
                else:
                    assert np.array_equal(u, ob.u), (name, k)
                assert np.array_equal(ens.field("bond_active", k), ob.bond_active[:ob.n_bonds])
            else:
                assert np.abs(u - ob.u).max() <= 1e-5 * np.abs(ob.u).max(), (name, k)
        ens.close()
