"""Parity with the FP64 CPU oracle on the benchmark workloads at their stated sizes.

- Mode-I tensile plate, BBMaterial, 40 x 20 x 4 points (3,200) at dx = 2.5e-3 m, horizon
  3.015 dx, rho = 2700, E = 70 GPa, Gc = 100 (critical stretch from Gc), bonds crossing
  x = 0.05 m for y < 0.01 m filtered, the top and bottom two rows pulled at +-0.6 m/s, 500
  Velocity Verlet steps at the CFL step with safety factor 0.7. FP64 in the reference's
  serial order must equal the oracle bit for bit (displacement, velocity, bond states,
  damage); the FP32-compensated form is held to 1e-5 in displacement, with the broken-bond
  counts of both reported.
- Jittered OSBMaterial block of 200 x 100 x 50 points (1.0M, 106.4M bonds) at dx = 1 mm with a
  5 m/s Gaussian velocity pulse on the x-min face and a 0.3 L through slit (the workload of
  bench.py --config pulse1m), 200 steps, against the oracle on all host cores in the serial
  loop's summation order (its serial-order gather, bit for bit the one-thread loop): the
  plain FP64 path in the serial-order mapping must equal it bit for bit (displacement,
  velocity, bond states); in lane groups (another summation order) it must stay within
  1e-8 relative in displacement, with the same broken-bond set except for bonds within
  1e-12 of the critical stretch, which are counted and reported. Two valid summation orders
  drift apart on this workload: the oracle's threads backend (chunked scatter) against its
  serial order differs by 5.5e-10 after 200 steps on a 125k-point block of the same kind,
  and lane group 1 against the chunked oracle by 2.1e-9 on this block, so 1e-10 holds only
  in one order.

Reference: velocity_verlet.jl:165-295 (step order), bond_system.jl:309-343 (failure, damage),
bond_based.jl:146-161, ordinary_state_based.jl:107-204.
"""
import os

import numpy as np
import pytest

import oracle as O
import pdcuda as pd
from helpers import oracle_bcs, oracle_body, plate_body

pytestmark = pytest.mark.gpu

PLATE_STEPS = 500
PULSE_STEPS = 200


def rel_err(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.fixture(scope="module")
def plate():
    """The plate, its oracle run (500 steps, serial order) and its CFL step."""
    body = plate_body(pd.BBMaterial())
    assert body.n_points == 3200
    ob = oracle_body(body)
    # 254,120 directed bonds in the lattice, 1,208 of them across the pre-crack filtered
    assert ob.n_bonds == 252_912
    dt = ob.stable_timestep(0.7)
    ob.force_density(0.0, dt)
    assert ob.run_vv(1, PLATE_STEPS, dt, oracle_bcs(body, 1, PLATE_STEPS, dt)) == 0
    return body, ob, dt


def run_device(body, prec, dt, steps, mapping=None):
    dev = pd.DeviceBody(body, precision=prec)
    if mapping is not None:
        dev.set_mapping(mapping)
    assert dev.stable_timestep(0.7) == dt
    dev.force(0.0, dt)
    dev.run(1, steps, dt)
    return dev


def test_plate_fp64_serial_order_bit_exact(plate):
    body, ob, dt = plate
    dev = run_device(body, "fp64", dt, PLATE_STEPS, mapping=0)
    for f, ref in (("displacement", ob.u), ("velocity", ob.v), ("position", ob.pos)):
        got = dev.field(f).T
        assert np.array_equal(got, ref), (f, rel_err(got, ref))
    assert np.array_equal(dev.field("bond_active"), ob.bond_active[:ob.n_bonds])
    assert np.array_equal(dev.field("damage"), ob.damage)
    broken = int(np.count_nonzero(ob.bond_active[:ob.n_bonds] == 0))
    print(f"plate FP64: {broken} broken bonds (filtered crack bonds are not in the list)")
    assert broken > 0   # the crack grows in this run
    dev.close()


def test_plate_fp32_compensated(plate):
    body, ob, dt = plate
    dev = run_device(body, "fp32", dt, PLATE_STEPS)
    err_u = rel_err(dev.field("displacement").T, ob.u)
    err_v = rel_err(dev.field("velocity").T, ob.v)
    ref_states = ob.bond_active[:ob.n_bonds]
    states = dev.field("bond_active")
    broken_ref = int(np.count_nonzero(ref_states == 0))
    broken = int(np.count_nonzero(states == 0))
    differ = int(np.count_nonzero(states != ref_states))
    print(f"plate FP32: displacement {err_u:.3e}, velocity {err_v:.3e}, broken bonds "
          f"{broken} (oracle {broken_ref}), states differing {differ}")
    assert err_u <= 1e-5
    assert abs(broken - broken_ref) <= max(2, broken_ref // 100)
    dev.close()


@pytest.fixture(scope="module")
def pulse():
    from bench import make_pulse_block
    body = make_pulse_block()
    assert body.n_points == 1_000_000
    O.set_threads(os.cpu_count() or 1)
    O.set_serial_order(True)
    try:
        ob = oracle_body(body)
        dt = ob.stable_timestep(0.7)
        ob.force_density(0.0, dt)
        assert ob.run_vv(1, PULSE_STEPS, dt, oracle_bcs(body, 1, PULSE_STEPS, dt)) == 0
    finally:
        O.set_threads(1)
        O.set_serial_order(False)
    return body, ob, dt


def run_pulse(pulse, mapping):
    body, ob, dt = pulse
    dev = pd.DeviceBody(body, precision="fp64")
    dev.set_mapping(mapping)
    assert dev.n_bonds == ob.n_bonds == 106_394_104
    assert np.array_equal(dev.field("n_neighbors"), np.diff(ob.off))
    # the CFL step is a minimum over points of per-point sums in the reference's order
    assert dev.stable_timestep(0.7) == dt
    dev.force(0.0, dt)
    dev.run(1, PULSE_STEPS, dt)
    return dev


def test_pulse_block_fp64_serial_order_bit_exact(pulse):
    body, ob, dt = pulse
    dev = run_pulse(pulse, 0)
    for f, ref in (("displacement", ob.u), ("velocity", ob.v)):
        got = dev.field(f).T
        assert np.array_equal(got, ref), (f, rel_err(got, ref))
    assert np.array_equal(dev.field("bond_active"), ob.bond_active[:ob.n_bonds])
    assert np.array_equal(dev.field("damage"), ob.damage)
    dev.close()


@pytest.mark.parametrize("group", [1, 4])
def test_pulse_block_fp64_lane_groups(pulse, group):
    body, ob, dt = pulse
    dev = run_pulse(pulse, group)
    err_u = rel_err(dev.field("displacement").T, ob.u)
    err_v = rel_err(dev.field("velocity").T, ob.v)
    states = dev.field("bond_active")
    ref_states = ob.bond_active[:ob.n_bonds]
    differ = int(np.count_nonzero(states != ref_states))
    near = dev.near_critical(1e-12)
    broken = int(np.count_nonzero(ref_states == 0))
    print(f"pulse FP64 group {group}: displacement {err_u:.3e}, velocity {err_v:.3e}, broken "
          f"{broken}, states differing {differ}, within 1e-12 of the critical stretch {near}")
    assert err_u <= 1e-8
    assert differ <= near
    dev.close()


@pytest.mark.skipif(os.environ.get("PD_FULL_RUNS") != "1",
                    reason="the whole 2000-step run (about 5 minutes of oracle time on 16 host "
                           "cores); set PD_FULL_RUNS=1")
def test_pulse_block_full_run_against_oracle():
    """All 2000 steps of the pulse block against the serial-order oracle: the FP64 path in the
    serial-order mapping (bit for bit) and in its tuned lane groups, and the FP32-compensated
    form."""
    from bench import make_pulse_block
    steps = 2000
    body = make_pulse_block()
    O.set_threads(os.cpu_count() or 1)
    O.set_serial_order(True)
    try:
        ob = oracle_body(body)
        dt = ob.stable_timestep(0.7)
        ob.force_density(0.0, dt)
        assert ob.run_vv(1, steps, dt, []) == 0
    finally:
        O.set_threads(1)
        O.set_serial_order(False)
    ref_states = ob.bond_active[:ob.n_bonds]
    res = {}
    for prec in ("fp64-serial", "fp64", "fp32"):
        dev = pd.DeviceBody(body, precision=prec[:4])
        if prec == "fp64-serial":
            dev.set_mapping(0)
        else:
            dev.autotune()
        assert dev.stable_timestep(0.7) == dt
        dev.force(0.0, dt)
        dev.run(1, steps, dt)
        states = dev.field("bond_active")
        res[prec] = dict(u=rel_err(dev.field("displacement").T, ob.u),
                         v=rel_err(dev.field("velocity").T, ob.v),
                         differ=int(np.count_nonzero(states != ref_states)),
                         near=dev.near_critical(1e-12), mapping=dev.mapping(),
                         damage=rel_err(dev.field("damage"), ob.damage))
        dev.close()
    broken = int(np.count_nonzero(ref_states == 0))
    print(f"pulse block, {steps} steps, oracle broken bonds {broken}: {res}")
    assert res["fp64-serial"]["u"] == 0 and res["fp64-serial"]["differ"] == 0
    assert res["fp64"]["u"] <= 1e-8
    assert res["fp64"]["differ"] <= res["fp64"]["near"]
    assert res["fp32"]["u"] <= 1e-5
