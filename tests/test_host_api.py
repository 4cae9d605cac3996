"""Host logic of the pdcuda package and the C ABI surface (CPU only)."""
import ctypes
import math
import os
import re

import numpy as np
import pytest

import pdcuda as pd

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_material_parameters(golden):
    # test/unit/physics/test_bond_based.jl:25-60
    pos, vol = pd.uniform_box(1, 1, 1, 0.5)
    body = pd.Body(pd.BBMaterial(), pos, vol)
    pd.material(body, horizon=2, rho=1, E=1, nu=0.25, Gc=1)
    p = body.point_params[0]
    assert (p.delta, p.rho, p.E, p.nu) == pytest.approx((2.0, 1.0, 1.0, 0.25))
    assert (p.G, p.K, p.lambda_, p.mu, p.Gc) == pytest.approx((0.4, 0.6666666666666666, 0.4, 0.4, 1.0))
    assert p.epsilon_c == pytest.approx(golden["bb_epsilon_c"], rel=1e-15)
    with pytest.raises(ValueError):
        pd.material(body, horizon=2, rho=1, E=1, nu=0.26, Gc=1)
    pd.material(body, horizon=2, rho=1, E=1, Gc=1)
    assert body.point_params[0].nu == 0.25 and len(body.point_params) == 1
    with pytest.raises(ValueError):
        pd.material(body, horizon=2, rho=1, nu=0.25, Gc=1)
    with pytest.raises(ValueError):
        pd.material(body, horizon=2, rho=1, E=1, G=1, Gc=1)
    with pytest.raises(ValueError):
        pd.material(body, horizon=2, rho=1, E=1, Gc=1, epsilon_c=0.1)
    # fracture parameters switch failure on; none switch it off (fracture.jl:147-175)
    assert body.fail_permit.all()
    pd.material(body, horizon=2, rho=1, E=1)
    assert not body.fail_permit.any()


def test_elastic_conversions():
    body = pd.Body(pd.OSBMaterial(), *pd.uniform_box(1, 1, 1, 0.5))
    for kw in ({"E": 70e9, "nu": 0.25}, {"E": 70e9, "G": 28e9}, {"K": 46.666666666666664e9, "G": 28e9},
               {"lambda": 28e9, "mu": 28e9}, {"nu": 0.25, "K": 46.666666666666664e9}):
        pd.material(body, horizon=0.1, rho=2700, **kw)
        p = body.point_params[0]
        assert p.E == pytest.approx(70e9, rel=1e-12) and p.nu == pytest.approx(0.25, rel=1e-12)
        assert p.bc == pytest.approx(18 * p.K / (math.pi * 0.1 ** 4), rel=1e-14)


def test_uniform_box_ordering():
    # point_generators.jl:45-60: x fastest, then y, then z, centred
    pos, vol = pd.uniform_box(1.0, 0.5, 0.25, 0.25)
    assert pos.shape == (3, 4 * 2 * 1)
    assert pos[:, 0] == pytest.approx([-0.375, -0.125, 0.0])
    assert pos[:, 1] == pytest.approx([-0.125, -0.125, 0.0])
    assert pos[:, 4] == pytest.approx([-0.375, 0.125, 0.0])
    assert np.all(vol == 0.25 ** 3)
    pos, _ = pd.uniform_box(1.0, 1.0, 1.0, 0.5, center=(1.0, 2.0, 3.0))
    assert pos.mean(axis=1) == pytest.approx([1.0, 2.0, 3.0])


def test_conditions_and_errors():
    pos, vol = pd.uniform_box(1, 1, 1, 0.25)
    body = pd.Body(pd.BBMaterial(), pos, vol)
    pd.material(body, horizon=0.8, rho=1, E=1, Gc=1)
    pd.point_set(body, "a", [0, 1, 2])
    pd.point_set(body, "top", where=lambda p: p[2] > 0.3)
    with pytest.raises(ValueError):
        pd.point_set(body, "a", [3])
    pd.velocity_bc(lambda t: 1.0, body, "a", 1)
    pd.velocity_bc(lambda p, t: p[0] * t, body, "a", "y")
    with pytest.raises(ValueError):  # same field, dim and points
        pd.velocity_bc(lambda t: 2.0, body, "a", "x")
    with pytest.raises(ValueError):  # argument names decide the kind
        pd.velocity_bc(lambda s: 2.0, body, "a", "z")
    with pytest.raises(ValueError):
        pd.velocity_bc(lambda t: 2.0, body, "a", 4)
    with pytest.raises(ValueError):
        pd.velocity_bc(lambda t: 2.0, body, "nope", 1)
    pd.forcedensity_bc(lambda t: 5.0, body, "top", "z")
    with pytest.raises(ValueError):
        pd.displacement_bc(lambda t: 1.0, body, "top", 1)
    pd.velocity_ic(body, "top", "x", 3.0)
    pd.velocity_ic(lambda p: p[0], body, "top", "y")
    pd.point_set(body, "b", [5, 6])
    pd.precrack(body, "a", "b")
    pd.point_set(body, "c", [1, 7])
    with pytest.raises(ValueError):
        pd.precrack(body, "a", "c")
    assert len(body.single_dim_bcs) == 2 and len(body.posdep_single_dim_bcs) == 1
    with pytest.raises(ValueError):
        pd.VelocityVerlet()
    with pytest.raises(ValueError):
        pd.VelocityVerlet(time=1.0, steps=10)
    with pytest.raises(ValueError):
        pd.VelocityVerlet(time=1.0, safety_factor=1)
    vv = pd.VelocityVerlet(time=11)
    vv.init(1.0)
    assert vv.n_steps == 12 and vv.end_time == 11


def header_symbols():
    src = open(os.path.join(ROOT, "include", "pdcuda.h")).read()
    return sorted(set(re.findall(r"^(?:pd_status|const char \*)\s*(pd_\w+)\(", src, re.M)))


def test_library_exports_every_declared_symbol():
    """libpdcuda.so loads without a GPU and exports every entry point of include/pdcuda.h."""
    lib = pd.lib()
    syms = header_symbols()
    assert len(syms) >= 20
    assert sorted(pd.EXPORTS) == syms
    for s in syms:
        assert hasattr(lib, s), s
    assert lib.pd_version() == b"0.1.0"


def test_library_errors_without_device_are_reported():
    """Without a device the C ABI returns an error status, never a silent fallback."""
    lib = pd.lib()
    h = ctypes.c_void_p()
    desc = pd._lib.BodyDesc()
    desc.n_points = -1
    assert lib.pd_create(ctypes.byref(desc), ctypes.byref(h)) == pd._lib.PD_ERR_ARG
    assert b"n_points" in lib.pd_last_error()
