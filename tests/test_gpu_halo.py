"""Partitioned bodies on the device (pdcuda/halo.py, csrc/pd_halo.cu): the partitions of a body,
held by one process on one GPU and exchanging their halo rows by device copies, step exactly
like the undivided body. Owned points keep the body's bond lists and summation order, so the
trajectories are bit-identical in every mapping, for both bond-state modes and with CMaterial
kills. The transfer between processes (torch.distributed point-to-point) is covered on CPU by
tests/test_halo_gloo.py."""
import numpy as np
import pytest

import pdcuda as pd
from pdcuda.halo import Partition, PartitionedBody
from helpers import plate_body

pytestmark = pytest.mark.gpu

MATS = {
    "BB": (pd.BBMaterial, None),
    "OSB": (pd.OSBMaterial, 0.25),
    "C": (lambda: pd.CMaterial(maxdmg=0.3), 0.25),
    "C-Wan": (lambda: pd.CMaterial(zem=pd.ZEMWan(), maxdmg=0.3), 0.25),
}


def make_plate(name, two_sets=False):
    mat, nu = MATS[name]
    body = plate_body(mat(), nx=24, ny=12, nz=3, nu=nu)
    if two_sets:
        # a second parameter set with another Gc on the right half: interface bonds get the
        # critical stretch of their owner, so the bond states are directed
        pd.point_set(body, "right_half", where=lambda p: p[0] > 0.03)
        kw = dict(horizon=3.015 * 2.5e-3, rho=2700.0, E=70e9, Gc=300.0)
        if nu is not None:
            kw["nu"] = nu
        pd.material(body, "right_half", **kw)
    return body


def run_body(body, prec, mapping, n):
    dev = pd.DeviceBody(body, precision=prec)
    dev.set_mapping(*mapping)
    dt = dev.stable_timestep(0.7)
    dev.force(0.0, dt)
    dev.run(1, n, dt)
    return dev, dt


def run_parts(body, n_parts, prec, mapping, n, how="index"):
    parts = [Partition(body, n_parts, p, prec, decomposition=how) for p in range(n_parts)]
    for p in parts:
        p.dev.set_mapping(*mapping)
    pb = PartitionedBody(parts)
    dt = pb.stable_timestep(0.7)
    pb.force(0.0, dt)
    pb.run(1, n // 2, dt)
    pb.run(n // 2 + 1, n - n // 2, dt)   # two runs: the closing kick and the next opening one
    return pb, dt


def assert_same(dev, pb):
    for f in ("displacement", "velocity", "velocity_half", "acceleration", "position", "damage"):
        assert np.array_equal(pb.field(f), dev.field(f)), f
    assert np.array_equal(pb.field("bond_active"), dev.field("bond_active"))


@pytest.mark.parametrize("name", ["BB", "OSB", "C", "C-Wan"])
@pytest.mark.parametrize("prec,mapping,how", [("fp64", (0,), "index"), ("fp32", (8,), "index"),
                                              ("fp64", (4,), "slabs"), ("fp32", (1,), "slabs")])
def test_partitions_step_like_the_body(name, prec, mapping, how):
    body = make_plate(name)
    dev, dt = run_body(body, prec, mapping, 100)
    pb, dt2 = run_parts(body, 3, prec, mapping, 100, how)
    assert dt2 == dt
    assert_same(dev, pb)
    assert np.count_nonzero(dev.field("bond_active") == 0) > 0
    for p in pb.parts:
        # halo rows are exactly the points bonded to an owned point
        nn = p.dev.field("n_neighbors")
        assert (nn[p.owned == 0] > 0).all()
        assert p.dev.info()[2] == dev.info()[2]   # the same bond-state mode
    pb.close()
    dev.close()


@pytest.mark.parametrize("name", ["OSB", "C", "C-Wan"])
def test_directed_bond_states(name):
    body = make_plate(name, two_sets=True)
    dev, dt = run_body(body, "fp64", (0,), 100)
    assert dev.info()[2] == 0      # directed states: reverse-bond lookups
    pb, _ = run_parts(body, 2, "fp64", (0,), 100)
    assert_same(dev, pb)
    if name.startswith("C"):
        # points were killed (damage above maxdmg), on both sides of the cut
        assert (dev.field("damage") == 1.0).any()
    pb.close()
    dev.close()


def test_random_pairs_and_single_partition():
    body = make_plate("OSB")
    dev = pd.DeviceBody(body, precision="fp32")
    dev.break_random_pairs(0.05, 1234)
    parts = [Partition(body, 4, p, "fp32", decomposition="slabs") for p in range(4)]
    for p in parts:
        p.break_random_pairs(0.05, 1234)
    pb = PartitionedBody(parts)
    assert np.array_equal(pb.field("bond_active"), dev.field("bond_active"))
    pb.close()
    dev.close()
    one, dt = run_parts(body, 1, "fp32", (1,), 20)
    ref, dt1 = run_body(body, "fp32", (1,), 20)
    assert dt == dt1
    assert_same(ref, one)
    one.close()
    ref.close()
