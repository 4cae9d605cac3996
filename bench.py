"""Benchmark of the explicit-dynamics hot path: bond-updates/s per Velocity Verlet step.

Workload (default): OSBMaterial dynamic fracture block of 400 x 200 x 100 points (8.0M
points, ~0.96B directed bonds) at dx = 5e-4 m, horizon 3.015 dx, E = 70 GPa, nu = 0.25,
rho = 2700 kg/m^3, Gc = 100 J/m^2, 5 % of the bond pairs broken at random (seeded),
+-1 m/s velocity conditions on the outermost point layer of both y faces, FP32-compensated
bond arithmetic with FP64 integration. One step = one Velocity Verlet step of the whole body.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
Under torchrun every rank runs its own body (replicas: specimens do not interact); the
time is the maximum over ranks.
"""
import argparse
import ctypes as C
import json
import math
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
for p in (os.path.join(ROOT, "peridynamics.jl_b200"),):
    if p not in sys.path:
        sys.path.insert(0, p)

METRIC = "bond-updates/s per VV step"
UNIT = "bond-updates/s"

CONFIGS = {
    # name: (nx, ny, nz, dx, material, random broken fraction, bc velocity)
    "osb8m": (400, 200, 100, 5e-4, "OSB", 0.05, 1.0),
    # mode-I tensile plate, BBMaterial, 40 x 20 x 4 points (see make_plate)
    "plate3200": (40, 20, 4, 2.5e-3, "BB", 0.0, 0.6),
    # quasi-static Newton-Krylov: bond-based three-point bending beam (x span, y height)
    "jfnk500k": (250, 50, 40, 1e-3, "BB", 0.0, 0.0),
    "osb1m": (200, 100, 50, 1e-3, "OSB", 0.0, 0.6),
    "bb1m": (200, 100, 50, 1e-3, "BB", 0.0, 0.6),
    "c1m": (200, 100, 50, 1e-3, "C", 0.0, 0.6),
    # the same block with ZEMWan's stabilisation (CW: NeoHooke, C : K^-1 per point)
    "cwan1m": (200, 100, 50, 1e-3, "CW", 0.0, 0.6),
    # jittered OSB block with a velocity pulse and a slit: the FP32 / FP64 precision study
    "pulse1m": (200, 100, 50, 1e-3, "OSB", 0.0, 0.0),
    # 64 CMat NeoHooke specimens of 20k-200k points in one device body (see make_ensemble)
    "ens64": (0, 0, 0, 1e-3, "C", 0.0, 0.6),
    # dynamic relaxation of an OSB block in uniform tension (see make_dr_block)
    "dr1m": (200, 100, 50, 1e-3, "OSB", 0.0, 0.0),
}
# configs of one body (the multi-GPU run partitions them; --replicas runs copies instead)
SINGLE_BODY = ("osb8m", "plate3200", "osb1m", "bb1m", "c1m", "cwan1m")
DR_STRAIN = 5e-5
# algorithmic bytes per point of the damping and velocity-update kernels of one relaxation step
# (damping: u, v_half, b_int, b_int_old, v_half_old, Lambda; update: Lambda, b_int, b_ext,
# v_half_old read, v_half, v, v_half_old, b_int_old written)
# (FP64: 128 + 176 B; FP32: b_int is 12 B, 116 + 164 B)
B_DR_POINT = {"fp64": 304.0, "fp32": 280.0}
# algorithmic bytes (FP32-compensated form): per directed bond nbr 4 + xi 12 + L 4 + 1/8 bit;
# per point 140 (u, v FP64 read+write, own u, b_ext/BC, parameter id, damage) + 8 for OSB
# (m, theta) + 72 for CMat (F, P K^-1) + 24 with ZEMWan (the symmetric stiffness C : K^-1)
B_BOND = {"fp32": 20.125, "fp64": 36.125}
B_POINT = {"fp32": 140.0, "fp64": 184.0}
B_POINT_EXTRA = {"BB": 0.0, "OSB": 8.0, "C": 72.0, "CW": 96.0}
# steps of the legs beside the timed run (per-kernel events, end to end): at most this many
EAGER_STEPS = 500


def pinned(*shape):
    """A zeroed float64 host array in page-locked memory (torch owns the allocation; the
    returned tensor keeps it alive)."""
    import torch
    t = torch.zeros(shape, dtype=torch.float64, pin_memory=True)
    return t, t.numpy()


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def make_body(cfg, jitter_seed=None, correction=None):
    import pdcuda as pd
    nx, ny, nz, dx, mat, frac, vbc = CONFIGS[cfg]
    if cfg == "plate3200":
        if correction == "energy":
            raise ValueError("the plate runs without the surface correction")
        return make_plate(pd.BBMaterial(), nx, ny, nz, dx, v=vbc), frac
    lx, ly, lz = nx * dx, ny * dx, nz * dx
    pos, vol = pd.uniform_box(lx, ly, lz, dx)
    corr = pd.EnergySurfaceCorrection if correction == "energy" else None
    if corr is not None and mat in ("C", "CW"):
        raise ValueError("the surface correction is available for BB and OSB")
    material = {"OSB": lambda: pd.OSBMaterial(correction=corr),
                "BB": lambda: pd.BBMaterial(correction=corr),
                "C": lambda: pd.CMaterial(model=pd.NeoHooke()),
                "CW": lambda: pd.CMaterial(model=pd.NeoHooke(), zem=pd.ZEMWan())}[mat]()
    body = pd.Body(material, pos, vol)
    kw = dict(horizon=3.015 * dx, rho=2700.0, E=70e9, Gc=100.0)
    if mat != "BB":
        kw["nu"] = 0.25
    pd.material(body, **kw)
    y = body._pos[:, 1]
    pd.point_set(body, "ymin", np.nonzero(y < y.min() + 0.5 * dx)[0])
    pd.point_set(body, "ymax", np.nonzero(y > y.max() - 0.5 * dx)[0])
    pd.velocity_bc(lambda t: -vbc, body, "ymin", "y")
    pd.velocity_bc(lambda t: vbc, body, "ymax", "y")
    return body, frac


def make_plate(mat, nx=40, ny=20, nz=4, dx=2.5e-3, E=70e9, rho=2700.0, Gc=100.0, v=0.6, nu=None):
    """Mode-I tensile plate (the defaults: 40 x 20 x 4 points, 3,200, at dx = 2.5 mm, a plate of
    0.1 x 0.05 x 0.01 m with its corner at the origin), horizon 3.015 dx: bonds crossing
    x = 0.5 lx for y < 0.2 ly are filtered (precrack! without damage update), the top and
    bottom two rows are pulled at +-v in y."""
    import pdcuda as pd
    lx, ly, lz = nx * dx, ny * dx, nz * dx
    pos, vol = pd.uniform_box(lx, ly, lz, dx, center=(lx / 2, ly / 2, lz / 2))
    body = pd.Body(mat, pos, vol)
    args = dict(horizon=3.015 * dx, rho=rho, E=E, Gc=Gc)
    if nu is not None:
        args["nu"] = nu
    pd.material(body, **args)
    pd.point_set(body, "crack_a", where=lambda p: (p[0] <= lx / 2) & (p[1] < 0.2 * ly))
    pd.point_set(body, "crack_b", where=lambda p: (p[0] > lx / 2) & (p[1] < 0.2 * ly))
    pd.precrack(body, "crack_a", "crack_b", update_dmg=False)
    pd.point_set(body, "top", where=lambda p: p[1] > ly - 2 * dx)
    pd.point_set(body, "bottom", where=lambda p: p[1] < 2 * dx)
    pd.velocity_bc(lambda t: v, body, "top", "y")
    pd.velocity_bc(lambda t: -v, body, "bottom", "y")
    return body


def make_dr_block(nx, ny, nz, dx, mat="OSB"):
    """A block in uniform tension for dynamic relaxation (the reference's relaxation bar at
    scale): the two x = min layers held by zero velocity conditions, a force density on the
    x = max layer that gives the strain DR_STRAIN, no pre-damage."""
    import pdcuda as pd
    pos, vol = pd.uniform_box(nx * dx, ny * dx, nz * dx, dx)
    material = {"OSB": pd.OSBMaterial, "BB": pd.BBMaterial,
                "C": lambda: pd.CMaterial(model=pd.NeoHooke()),
                "CW": lambda: pd.CMaterial(model=pd.NeoHooke(), zem=pd.ZEMWan())}[mat]()
    body = pd.Body(material, pos, vol)
    kw = dict(horizon=3.015 * dx, rho=2700.0, E=70e9, Gc=100.0)
    if mat != "BB":
        kw["nu"] = 0.25
    pd.material(body, **kw)
    x = body._pos[:, 0]
    pd.point_set(body, "left", np.nonzero(x < x.min() + 1.5 * dx)[0])
    right = np.nonzero(x > x.max() - 0.5 * dx)[0]
    pd.point_set(body, "right", right)
    b_right = DR_STRAIN * 70e9 * (ny * dx) * (nz * dx) / vol[right].sum()
    for d in ("x", "y", "z"):
        pd.velocity_bc(lambda t: 0.0, body, "left", d)
    pd.forcedensity_bc(lambda t: b_right, body, "right", "x")
    return body


def make_ensemble(n=64, seed=0xE45, dx=1e-3, vbc=0.6):
    """Specimens of the ensemble workload: cuboids of aspect 4:2:1 with a seeded point count
    in [20k, 200k] at dx = 1 mm, horizon 3.015 dx, CMaterial (NeoHooke, ZEM Cs = 0.5),
    E ~ U[50, 200] GPa, nu = 0.3, rho ~ U[2000, 8000] kg/m^3, Gc = 100 J/m^2, an edge crack on
    the plane y = 0 from the x-min face of length ~ U[0.1, 0.4] of the specimen length
    (precrack! filter), +-vbc m/s on the outermost y layers."""
    import pdcuda as pd
    rng = np.random.default_rng(seed)
    bodies = []
    for _ in range(n):
        m = max(3, int(round((rng.uniform(20e3, 200e3) / 8.0) ** (1.0 / 3.0))))
        E, rho, a = rng.uniform(50e9, 200e9), rng.uniform(2000.0, 8000.0), rng.uniform(0.1, 0.4)
        pos, vol = pd.uniform_box(4 * m * dx, 2 * m * dx, m * dx, dx)
        body = pd.Body(pd.CMaterial(model=pd.NeoHooke()), pos, vol)
        pd.material(body, horizon=3.015 * dx, rho=rho, E=E, nu=0.3, Gc=100.0)
        x, y = pos[0], pos[1]
        tip = x.min() + a * (x.max() - x.min())
        pd.point_set(body, "crack_a", np.nonzero((y < 0) & (x <= tip))[0])
        pd.point_set(body, "crack_b", np.nonzero((y >= 0) & (x <= tip))[0])
        pd.precrack(body, "crack_a", "crack_b", update_dmg=False)
        pd.point_set(body, "ymin", np.nonzero(y < y.min() + 0.5 * dx)[0])
        pd.point_set(body, "ymax", np.nonzero(y > y.max() - 0.5 * dx)[0])
        pd.velocity_bc(lambda t: -vbc, body, "ymin", "y")
        pd.velocity_bc(lambda t: vbc, body, "ymax", "y")
        bodies.append(body)
    return bodies


def make_pulse_block(seed=0x1A5, dx=1e-3):
    """OSB block of 200 x 100 x 50 points at dx = 1 mm with seeded uniform jitter of +-0.05 dx
    per coordinate, horizon 3.015 dx, E = 70 GPa, nu = 0.25, rho = 2700, Gc = 100; a Gaussian
    velocity pulse v_x = 5 exp(-((y - y_c)^2 + (z - z_c)^2) / (2 (5 dx)^2)) m/s on the x-min
    layer; a through slit (bonds across the mid-height plane removed) of length 0.3 L centred
    in x."""
    import pdcuda as pd
    nx, ny, nz = 200, 100, 50
    pos, vol = pd.uniform_box(nx * dx, ny * dx, nz * dx, dx)
    rng = np.random.default_rng(seed)
    pos = pos + rng.uniform(-0.05 * dx, 0.05 * dx, pos.shape)
    body = pd.Body(pd.OSBMaterial(), pos, vol)
    pd.material(body, horizon=3.015 * dx, rho=2700.0, E=70e9, nu=0.25, Gc=100.0)
    ix = np.arange(body.n_points) % nx
    iy = (np.arange(body.n_points) // nx) % ny
    L = nx * dx
    x, y, z = pos
    slit = np.abs(x) <= 0.15 * L
    pd.point_set(body, "slit_a", np.nonzero(slit & (iy < ny // 2))[0])
    pd.point_set(body, "slit_b", np.nonzero(slit & (iy >= ny // 2))[0])
    pd.precrack(body, "slit_a", "slit_b", update_dmg=False)
    pd.point_set(body, "face", np.nonzero(ix == 0)[0])
    yc, zc, s = y.mean(), z.mean(), 5 * dx
    pd.velocity_ic(lambda p: 5.0 * math.exp(-((p[1] - yc) ** 2 + (p[2] - zc) ** 2) / (2 * s * s)),
                   body, "face", "x")
    return body


def run_precision_study(args, local):
    """--config pulse1m: the same run in the plain FP64 form and the FP32-compensated form;
    errors of the FP32 run against the FP64 one (displacement, velocity, damage, bond states)."""
    import pdcuda as pd
    body = make_pulse_block()
    out = {}
    steps = args.steps
    for prec in ("fp64", "fp32"):
        dev = pd.DeviceBody(body, precision=prec, device=local)
        dt = dev.stable_timestep(0.7)
        dev.autotune()
        dev.force(0.0, dt)
        t0 = time.perf_counter()
        dev.run(1, steps, dt)
        out[prec] = {"s": time.perf_counter() - t0, "dt": dt, "near": dev.near_critical(1e-12),
                     "u": dev.field("displacement"), "v": dev.field("velocity"),
                     "damage": dev.field("damage"), "bonds": dev.field("bond_active"),
                     "mapping": dev.mapping()}
        dev.close()
    a, b = out["fp64"], out["fp32"]
    rel = lambda x, y: float(np.abs(x - y).max() / np.abs(x).max())
    rms = lambda x, y: float(np.sqrt(((x - y) ** 2).mean()) / np.sqrt((x ** 2).mean()))
    line = {"study": "FP32-compensated vs plain FP64 (GPU; the FP64 path equals the oracle in "
                     "serial order, to 1e-12 in lane groups)",
            "workload": "pulse1m: OSB 200x100x50 points (1.0M), jitter +-0.05 dx, 5 m/s Gaussian "
                        "pulse on the x-min face, 0.3 L through slit at mid-height",
            "points": body.n_points, "bonds": int(a["bonds"].size), "steps": steps,
            "dt": a["dt"], "dt_equal": a["dt"] == b["dt"],
            "displacement": {"max_rel": rel(a["u"], b["u"]), "rms_rel": rms(a["u"], b["u"])},
            "velocity": {"max_rel": rel(a["v"], b["v"]), "rms_rel": rms(a["v"], b["v"])},
            "damage": {"max_abs": float(np.abs(a["damage"] - b["damage"]).max()),
                       "points_differing": int((a["damage"] != b["damage"]).sum()),
                       "points_damaged_fp64": int((a["damage"] > 0).sum())},
            "broken_bonds": {"fp64": int((a["bonds"] == 0).sum()), "fp32": int((b["bonds"] == 0).sum()),
                             "state_differs": int((a["bonds"] != b["bonds"]).sum()),
                             "near_critical_1e-12": {"fp64": a["near"], "fp32": b["near"]}},
            "seconds": {"fp64": a["s"], "fp32": b["s"], "ratio": a["s"] / b["s"]},
            "mapping": {"fp64": a["mapping"], "fp32": b["mapping"]}}
    print(json.dumps(line), flush=True)


def run_spot_checks(args, local):
    """--check-every K: the FP32-compensated run of --steps steps (CUDA graphs, timed on the
    device) with the plain FP64 path of the same body advanced beside it; every K steps the two
    are compared: displacement and velocity (largest and RMS difference relative to the FP64
    field), bond states that differ, bonds broken in each, and the bonds within 1e-8 and 1e-12
    of the critical stretch (FP64 positions)."""
    import pdcuda as pd
    body, frac = make_body(args.config)
    devs = {}
    for prec in ("fp64", "fp32"):
        d = pd.DeviceBody(body, precision=prec, device=local)
        if frac > 0:
            d.break_random_pairs(frac, 0x5EED)
        d.autotune()
        devs[prec] = d
    d64, d32 = devs["fp64"], devs["fp32"]
    dt = d32.stable_timestep(0.7)
    dt64 = d64.stable_timestep(0.7)
    every = args.check_every
    d32.set_graph(min(args.graph, every) if args.graph > 0 else 0)
    for d in (d32, d64):
        d.force(0.0, dt)
    n_bonds = d32.info()[1]
    active0 = int(np.count_nonzero(d64.field("bond_active")))
    rel = lambda a, b: float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
    rms = lambda a, b: float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))
    checks, ms32, ms64, done = [], 0.0, 0.0, 0
    with ClockSampler(local) as clk:
        while done < args.steps:
            k = min(every, args.steps - done)
            ms32 += d32.run_timed(done + 1, k, dt, phases=False)
            ms64 += d64.run_timed(done + 1, k, dt, phases=False)
            done += k
            u32, u64 = d32.field("displacement"), d64.field("displacement")
            v32, v64 = d32.field("velocity"), d64.field("velocity")
            s32, s64 = d32.field("bond_active"), d64.field("bond_active")
            checks.append({"step": done,
                           "displacement": {"max_rel": rel(u32, u64), "rms_rel": rms(u32, u64)},
                           "velocity": {"max_rel": rel(v32, v64), "rms_rel": rms(v32, v64)},
                           "broken_in_run": {"fp64": active0 - int(np.count_nonzero(s64)),
                                             "fp32": active0 - int(np.count_nonzero(s32))},
                           "states_differ": int(np.count_nonzero(s32 != s64)),
                           "near_critical_fp64": {"1e-8": d64.near_critical(1e-8),
                                                  "1e-12": d64.near_critical(1e-12)}})
            print(json.dumps({"spot_check": checks[-1]}), flush=True)
    nx, ny, nz, dx, mat, _, vbc = CONFIGS[args.config]
    line = {"study": "FP32-compensated run with FP64 spot checks (both on the GPU; the FP64 path "
                     "equals the oracle bit for bit in serial order, to 1e-10 in lane groups)",
            "workload": f"{args.config}: {mat} {nx}x{ny}x{nz} points, dx={dx}, {frac:.0%} pairs "
                        f"broken, +-{vbc} m/s on the y faces",
            "bonds": n_bonds, "steps": args.steps, "check_every": every, "dt": dt,
            "dt_equal": dt == dt64,
            "graph_steps": min(args.graph, every) if args.graph > 0 else 0,
            "fp32": {"ms_per_step": ms32 / args.steps, "bond_updates_per_s": n_bonds * args.steps / (ms32 / 1e3),
                     "mapping": d32.mapping()},
            "fp64": {"ms_per_step": ms64 / args.steps, "bond_updates_per_s": n_bonds * args.steps / (ms64 / 1e3),
                     "mapping": d64.mapping()},
            "checks": checks, "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    d32.close()
    d64.close()


def run_ensemble(args, rank, world, local, dist):
    """--config ens64: all specimens advanced together, every one with its own CFL step; one
    step = one Velocity Verlet step of every specimen. The specimens are cut into --ens-classes
    size classes, each one device body with its own autotuned mapping, all advanced by one CUDA
    graph. Ranks own disjoint specimen sets (replicas: no exchange)."""
    import pdcuda as pd
    from pdcuda.replicas import partition_specimens, reduce_max, reduce_sum
    bodies = make_ensemble()
    mine = partition_specimens([b.n_points for b in bodies], world)[rank]
    gsteps = min(args.graph if args.graph else 50, args.steps)
    t0 = time.perf_counter()
    ens = pd.Ensemble([bodies[k] for k in mine], precision=args.precision, device=local,
                      graph_steps=gsteps, classes=args.ens_classes)
    setup_s = time.perf_counter() - t0
    ens.autotune()
    ens.run(args.warmup)
    step = args.warmup + 1
    ens.run(gsteps, first_step=step)   # untimed: captures the graph of the timed blocks
    step += gsteps
    n_pts, n_bonds = ens.info()
    launches0 = ens.launch_count()
    if dist:
        dist.barrier()
    with ClockSampler(local) as clk:
        ms = ens.run_timed(step, args.steps, phases=False)
        step += args.steps
        launches = ens.launch_count() - launches0
        # per-kernel durations: every class alone for the same number of steps, eagerly
        per_class = ens.class_phase_times(step, args.steps)
        step += args.steps
    ms_max = reduce_max(ms, dist, f"cuda:{local}")
    bonds_all = reduce_sum(n_bonds, dist, f"cuda:{local}")
    value = bonds_all * args.steps / (ms_max / 1e3)
    classes = ens.class_info()
    for c, t in zip(classes, per_class):
        c["ms_per_step_alone"] = {"total": t[0] / args.steps, "phase_a": t[1] / args.steps,
                                  "phase_b": t[2] / args.steps, "integrate": t[3] / args.steps}
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": "f32" if args.precision == "fp32" else "f64", "data": "synthetic",
                "config": {"workload": "ens64: 64 CMat NeoHooke specimens of 20k-200k points (seeded), "
                                       "edge cracks, +-0.6 m/s, own CFL step each, size classes in "
                                       "one CUDA graph",
                           "specimens": len(mine), "points": n_pts, "bonds": n_bonds,
                           "classes": classes, "graph_steps": gsteps,
                           "setup_s": setup_s, "parallelism": f"replicas x{world}"},
                "ms": {"phase_a": sum(t[1] for t in per_class) / args.steps,
                       "phase_b": sum(t[2] for t in per_class) / args.steps,
                       "integrate": sum(t[3] for t in per_class) / args.steps,
                       "note": "per-kernel sums of the classes run alone, eagerly"},
                "gpu_launches": launches, "clocks": clk.summary()}
        print(json.dumps(line), flush=True)
    ens.close()


class ClockSampler:
    """SM clock and clock-event reasons sampled during the timed region.

    NVML is polled every 10 ms from a thread, so that a timed region of a fraction of a second
    still gets a dozen samples; nvidia-smi at its 200 ms period is the fallback. The raw
    samples go to PD_BENCH_CLOCKS_DIR if set, else the temporary directory (the JSON line
    carries their summary)."""

    REASONS = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, index, period_s=0.01):
        import tempfile
        self.index = index
        self.period = period_s
        self.proc = None
        self.thread = None
        self.rows = []        # (sm_mhz, max_mhz, power_w, reasons tuple)
        self.source = None
        base = os.environ.get("PD_BENCH_CLOCKS_DIR") or tempfile.gettempdir()
        self.path = os.path.join(base, f"clocks_{index}.csv")

    def _nvml_handle(self):
        import pynvml as N
        N.nvmlInit()
        try:   # the NVML device of this CUDA device (CUDA_VISIBLE_DEVICES may renumber)
            import torch
            uuid = str(torch.cuda.get_device_properties(self.index).uuid)
            return N, N.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            return N, N.nvmlDeviceGetHandleByIndex(self.index)

    def _poll(self, N, h):
        import threading
        bits = (N.nvmlClocksEventReasonHwSlowdown, N.nvmlClocksEventReasonHwThermalSlowdown,
                N.nvmlClocksEventReasonSwThermalSlowdown, N.nvmlClocksEventReasonSwPowerCap)
        mx = float(N.nvmlDeviceGetMaxClockInfo(h, N.NVML_CLOCK_SM))
        while not self.stop.is_set():
            try:
                sm = float(N.nvmlDeviceGetClockInfo(h, N.NVML_CLOCK_SM))
                r = N.nvmlDeviceGetCurrentClocksEventReasons(h)
                pw = N.nvmlDeviceGetPowerUsage(h) / 1000.0
                self.rows.append((sm, mx, pw, tuple(nm for b, nm in zip(bits, self.REASONS) if r & b)))
            except Exception:
                pass
            self.stop.wait(self.period)
        assert isinstance(self.stop, threading.Event)

    def __enter__(self):
        import threading
        try:
            N, h = self._nvml_handle()
            self.stop = threading.Event()
            self.thread = threading.Thread(target=self._poll, args=(N, h), daemon=True)
            self.thread.start()
            self.source = "nvml 10 ms"
            return self
        except Exception:
            self.thread = None
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                stderr=subprocess.DEVNULL)
            self.source = "nvidia-smi 200 ms"
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.thread is not None:
            self.stop.set()
            self.thread.join(timeout=5)
            try:
                os.makedirs(os.path.dirname(self.path), exist_ok=True)
                with open(self.path, "w") as f:
                    for sm, mx, pw, rs in self.rows:
                        f.write(f"{sm},{mx},{pw},{'|'.join(rs)}\n")
            except Exception:
                pass
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()
            try:
                for r in open(self.path).read().strip().splitlines():
                    r = r.split(",")
                    self.rows.append((float(r[1]), float(r[2]), float(r[3]),
                                      tuple(nm for k, nm in enumerate(self.REASONS)
                                            if r[5 + k].strip() == "Active")))
            except Exception:
                pass

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0,
                    "source": self.source}
        sm = [r[0] for r in self.rows]
        reasons = sorted({nm for r in self.rows for nm in r[3]})
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": self.rows[0][1], "reasons": reasons,
                "samples": len(sm), "sm_mhz_min": min(sm), "power_w_max": max(r[2] for r in self.rows),
                "source": self.source}


def cpu_model():
    """The host CPU's model name (/proc/cpuinfo)."""
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except Exception:
        pass
    import platform
    return platform.processor() or "unknown"


def oracle_sample(cfg, threads):
    """The FP64 oracle (CPU restatement of the reference, OpenMP) on a 64x64x40 sub-block of the
    same lattice, spacing and parameters, initialised and ready to step."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    nx, ny, nz, dx, mat, frac, vbc = CONFIGS[cfg]
    sx, sy, sz = min(nx, 64), min(ny, 64), min(nz, 40)
    g = lambda n: (np.arange(n) - (n - 1) / 2) * dx
    X = np.array(np.meshgrid(g(sx), g(sy), g(sz), indexing="ij")).reshape(3, -1).T
    X = np.ascontiguousarray(X[np.lexsort((X[:, 0], X[:, 1], X[:, 2]))])
    V = np.full(len(X), dx ** 3)
    om = {"OSB": O.OSB, "BB": O.BB, "C": O.CMAT, "CW": O.CMAT}[mat]
    kw = {} if mat == "BB" else {"nu": 0.25}
    p = O.point_params(om, 3.015 * dx, 2700.0, E=70e9, Gc=100.0, **kw)
    O.set_threads(threads)
    b = O.OracleBody(om, X, V, [p], cmodel=O.NEOHOOKE,
                     zem=O.ZEM_WAN if mat == "CW" else O.ZEM_SILLING)
    dt = b.stable_timestep(0.7)
    b.v[:, 1] = np.where(X[:, 1] > 0, vbc, -vbc)
    b.force_density(0.0, dt)
    return b, dt, (sx, sy, sz)


def plate_oracle(threads):
    """The oracle twin of the mode-I plate (all of it), its CFL step and its conditions."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from twin import oracle_bcs, oracle_body
    body, _ = make_body("plate3200")
    O.set_threads(threads)
    ob = oracle_body(body)
    dt = ob.stable_timestep(0.7)
    ob.force_density(0.0, dt)
    return ob, dt, lambda first, n: oracle_bcs(body, first, n, dt)


def cpu_baseline(cfg, threads, budget_s=15.0, correction="none", steps=500):
    """bond-updates/s of the oracle sample over whole Velocity Verlet steps (a run of about
    budget_s seconds); the plate runs whole (all its points, `steps` steps)."""
    if cfg == "plate3200":
        ob, dt, bcs = plate_oracle(threads)
        table = bcs(1, steps)
        t0 = time.perf_counter()
        ob.run_vv(1, steps, dt, table)
        el = time.perf_counter() - t0
        return {"value": ob.n_bonds * steps / el, "unit": UNIT, "cores": threads,
                "cpu_model": cpu_model(), "kind": "port",
                "sample": f"the whole job: {ob.n} points, {ob.n_bonds} bonds, {steps} FP64 VV "
                          f"steps in {el:.2f} s"}
    b, dt, (sx, sy, sz) = oracle_sample(cfg, threads)
    if correction == "energy":
        b.init_surface_correction()
    steps, t0 = 0, time.perf_counter()
    while True:
        b.run_vv(steps + 1, 1, dt)
        steps += 1
        el = time.perf_counter() - t0
        if el > budget_s or steps >= 5000:
            break
    return {"value": b.n_bonds * steps / el, "unit": UNIT, "cores": threads, "cpu_model": cpu_model(), "kind": "port",
            "sample": f"{sx}x{sy}x{sz} sub-block ({b.n} points, {b.n_bonds} bonds) of the same "
                      f"lattice and parameters, {steps} FP64 VV steps in {el:.1f} s"}


def dr_oracle_sample(cfg, threads):
    """The FP64 oracle with its dynamic relaxation on a 64x64x40 sub-block of the dr1m block
    (same spacing, parameters and loading), initialised and ready to step."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from dr import OracleDR
    nx, ny, nz, dx, mat, frac, vbc = CONFIGS[cfg]
    sx, sy, sz = min(nx, 64), min(ny, 64), min(nz, 40)
    g = lambda n: (np.arange(n) - (n - 1) / 2) * dx
    X = np.array(np.meshgrid(g(sx), g(sy), g(sz), indexing="ij")).reshape(3, -1).T
    X = np.ascontiguousarray(X[np.lexsort((X[:, 0], X[:, 1], X[:, 2]))])
    V = np.full(len(X), dx ** 3)
    om = {"OSB": O.OSB, "BB": O.BB, "C": O.CMAT, "CW": O.CMAT}[mat]
    kw = {} if mat == "BB" else {"nu": 0.25}
    p = O.point_params(om, 3.015 * dx, 2700.0, E=70e9, Gc=100.0, **kw)
    O.set_threads(threads)
    b = O.OracleBody(om, X, V, [p], cmodel=O.NEOHOOKE)
    left = np.nonzero(X[:, 0] < X[:, 0].min() + 1.5 * dx)[0]
    right = np.nonzero(X[:, 0] > X[:, 0].max() - 0.5 * dx)[0]
    b_right = DR_STRAIN * 70e9 * (sy * dx) * (sz * dx) / V[right].sum()
    bcs = [dict(field=0, dim=d, kind=2, pts=left, values=np.zeros(len(left))) for d in range(3)]
    bcs.append(dict(field=1, dim=0, kind=2, pts=right, values=np.full(len(right), b_right)))
    dr = OracleDR(b, 1.0, fast=True)
    b.force_density(0.0, 1.0)
    return b, dr, bcs, (sx, sy, sz)


def dr_cpu_baseline(cfg, threads, budget_s=15.0):
    """bond-updates/s of the oracle sample over whole relaxation steps (about budget_s s)."""
    b, dr, bcs, (sx, sy, sz) = dr_oracle_sample(cfg, threads)
    steps, t0 = 0, time.perf_counter()
    while True:
        steps += 1
        dr.step(steps, bcs)
        el = time.perf_counter() - t0
        if el > budget_s or steps >= 5000:
            break
    return {"value": b.n_bonds * steps / el, "unit": UNIT, "cores": threads, "cpu_model": cpu_model(), "kind": "port",
            "sample": f"{sx}x{sy}x{sz} sub-block ({b.n} points, {b.n_bonds} bonds) of the same "
                      f"lattice, parameters and loading, {steps} FP64 relaxation steps in {el:.1f} s "
                      f"(force on all threads, damping sums in numpy)"}


def run_dr(args, rank, world, local, dist):
    """--config dr1m: dynamic relaxation of a 1M-point OSB block in uniform tension; one step =
    one relaxation step (conditions and drift, force density, damping, velocity update).
    Ranks run independent replicas."""
    import pdcuda as pd
    from pdcuda import dynamic_relaxation as drm
    from pdcuda.replicas import reduce_max
    nx, ny, nz, dx, mat, _, _ = CONFIGS[args.config]
    prec = args.precision
    body = make_dr_block(nx, ny, nz, dx, mat)
    dev = pd.DeviceBody(body, precision=prec, device=local)
    n_pts, n_bonds, _ = dev.info()
    dev.autotune()
    mapping = dev.mapping()
    dr = pd.DynamicRelaxation(steps=args.warmup + args.steps)
    drm.init(dev, dr)
    drm.run(dev, dr, 1, args.warmup)
    launches0 = dev.launch_count()

    def barrier():
        if dist:
            import torch
            dist.barrier()
            torch.cuda.synchronize()

    barrier()
    with ClockSampler(local) as clk:
        ms, ms_drift, ms_force, ms_relax = drm.run_timed(dev, dr, args.warmup + 1, args.steps)
    launches = dev.launch_count() - launches0
    barrier()
    ms_max = reduce_max(ms, dist, f"cuda:{local}")
    value = n_bonds * args.steps * world / (ms_max / 1e3)
    right = body.point_sets["right"]
    u = dev.field("displacement")
    exact = DR_STRAIN * (body._pos[right, 0].mean() - body._pos[body.point_sets["left"], 0].max())
    progress = float(u[0, right].mean() / exact)
    # roofline: the force kernels of a step (OSB: phases A and B each stream every bond once)
    n_phase = 1 if mat == "BB" else 2
    pt = {"fp32": 64 + 8 + 16 + 4 + 4, "fp64": 128 + 8 + 32 + 4 + 4}[prec]
    force_bytes = n_phase * (n_bonds * B_BOND[prec] + n_pts * pt)
    peak, peak_kind = load_peaks()
    force_ms = ms_force / args.steps
    achieved = force_bytes / (force_ms / 1e3) / 1e9
    relax_ms = ms_relax / args.steps
    relax_gbs = n_pts * B_DR_POINT[prec] / (relax_ms / 1e3) / 1e9

    # end to end through the public API with host buffers: upload the state, restart the
    # relaxation, run, read back
    # (page-locked host buffers)
    bufs = [pinned(n_pts, 3), pinned(n_pts, 3), pinned(n_pts, 3), pinned(n_pts)]
    h_u, h_v, out_u, out_d = (b[1] for b in bufs)
    # untimed warm-up through the same calls
    dev.set_state(displacement=h_u, velocity=h_v)
    drm.init(dev, dr)
    drm.run(dev, dr, 1, max(args.warmup, 3))
    dev.field("displacement", out=out_u)
    barrier()
    t0 = time.perf_counter()
    dev.set_state(displacement=h_u, velocity=h_v)
    drm.init(dev, dr)
    drm.run(dev, dr, 1, args.steps)
    dev.field("displacement", out=out_u)
    dev.field("damage", out=out_d)
    e2e_s = reduce_max(time.perf_counter() - t0, dist, f"cuda:{local}")
    e2e = n_bonds * args.steps * world / e2e_s
    dev.close()
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = dr_cpu_baseline(args.config, os.cpu_count() or 1)
    if rank == 0:
        line = {
            "metric": "bond-updates/s per relaxation step", "value": value, "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if prec == "fp32" else "f64", "data": "synthetic",
            "config": {"workload": f"dr1m: {mat} {nx}x{ny}x{nz} points, dx={dx}, horizon 3.015dx, "
                                   f"uniform tension (strain {DR_STRAIN}), dynamic relaxation step",
                       "points": n_pts, "bonds": n_bonds, "precision": prec,
                       "mapping": dict(zip(("group", "block", "pipe"), mapping)),
                       "l2": "inputs larger than L2 (bond arrays of ~2.5 GB)",
                       "parallelism": f"replicas x{world}"},
            "roofline": {"bound": "hbm", "kernel": f"{mat.lower()} force (all phases of a step)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None, "peak_kind": peak_kind,
                         "alg_bytes_per_step": force_bytes, "ms_per_step": force_ms},
            "relax_kernels": {"ms_per_step": relax_ms, "alg_bytes_per_step": n_pts * B_DR_POINT[prec],
                              "achieved_gbs": relax_gbs, "frac": relax_gbs / peak},
            "ms": {"drift": ms_drift / args.steps, "force": force_ms, "relax": relax_ms},
            "relaxation": {"steps": args.warmup + args.steps, "elongation_over_exact": progress},
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": (h_u.nbytes + h_v.nbytes) / args.steps,
                    "d2h_bytes_per_step": (out_u.nbytes + out_d.nbytes) / args.steps},
            "gpu_launches": launches, "clocks": clk.summary(), "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)


def run_halo(args, rank, world, local, dist):
    """--halo: one body cut into partitions with halo exchange (pdcuda.halo): one partition per
    rank over NCCL (strong scaling), or --halo-parts P partitions held by one process on one GPU
    (the exchange is then device copies: the cost of partitioning without the link)."""
    import pdcuda as pd
    from pdcuda.halo import Partition, PartitionedBody
    from pdcuda.replicas import reduce_max
    nx, ny, nz, dx, mat, frac, vbc = CONFIGS[args.config]
    body, frac = make_body(args.config)
    n_parts = world if world > 1 else max(args.halo_parts, 1)
    mine = [rank] if world > 1 else list(range(n_parts))
    t0 = time.perf_counter()
    from pdcuda.halo import decompose
    owner = decompose(body, n_parts, args.halo_decomposition)
    parts = [Partition(body, n_parts, p, args.precision, device=local, owner=owner) for p in mine]
    for p in parts:
        if frac > 0:
            p.break_random_pairs(frac, 0x5EED)
        p.dev.autotune()
    pb = PartitionedBody(parts, dist if world > 1 else None, device=local)
    setup_s = time.perf_counter() - t0
    dt = pb.stable_timestep(0.7)
    pb.force(0.0, dt)
    pb.run(1, args.warmup, dt)
    launches0 = sum(p.dev.launch_count() for p in parts)
    if dist:
        dist.barrier()
    with ClockSampler(local) as clk:
        ms = pb.run(args.warmup + 1, args.steps, dt, timed=True)
    launches = sum(p.dev.launch_count() for p in parts) - launches0
    ms_max = reduce_max(ms["total"], dist, f"cuda:{local}")
    owned_bonds = sum(len(p.owned_field("bond_active")) for p in parts)
    halo_rows = sum(int(np.count_nonzero(p.owned == 0)) for p in parts)
    rows = sum(len(p.rows) for p in parts)
    all_bonds = sum(p.dev.info()[1] for p in parts)
    from pdcuda.replicas import reduce_sum
    body_bonds = reduce_sum(owned_bonds, dist, f"cuda:{local}")
    value = body_bonds * args.steps / (ms_max / 1e3)
    mapping = [dict(zip(("group", "block", "pipe"), p.dev.mapping())) for p in parts]
    step = args.warmup + 1 + args.steps

    # roofline of the dominant kernel on this process's partitions: the second force kernel
    # (state-based) or the only one (BB), algorithmic bytes of the bonds and rows it sweeps
    prec = args.precision
    dom = "force_b" if "force_b" in ms else "force_a"
    pt_bytes = {"fp32": 32 + 8 + 16 + 12 + 4, "fp64": 64 + 8 + 32 + 24 + 4}[prec]
    alg = all_bonds * B_BOND[prec] + rows * pt_bytes
    dom_ms = ms[dom] / args.steps
    peak, peak_kind = load_peaks()
    achieved = alg / (dom_ms / 1e3) / 1e9

    # end to end through the public API with host buffers: every partition's state uploaded
    # from page-locked host memory, the steps, its owned displacement and damage read back
    bufs = [(pinned(len(p.rows), 3), pinned(len(p.rows), 3)) for p in parts]
    for p, (hu, hv) in zip(parts, bufs):
        p.dev.set_state(displacement=hu[1], velocity=hv[1])
    pb.run(step, max(args.warmup, 3), dt)
    step += max(args.warmup, 3)
    if dist:
        dist.barrier()
    e2e_steps = min(args.steps, EAGER_STEPS)
    t0 = time.perf_counter()
    for p, (hu, hv) in zip(parts, bufs):
        p.dev.set_state(displacement=hu[1], velocity=hv[1])
    pb.run(step, e2e_steps, dt)
    back = [(p.owned_field("displacement"), p.owned_field("damage")) for p in parts]
    e2e_s = reduce_max(time.perf_counter() - t0, dist, f"cuda:{local}")
    h2d = reduce_sum(sum(hu[1].nbytes + hv[1].nbytes for hu, hv in bufs), dist, f"cuda:{local}")
    d2h = reduce_sum(sum(u.nbytes + d.nbytes for u, d in back), dist, f"cuda:{local}")
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None,
            "dtype": "f32" if args.precision == "fp32" else "f64", "data": "synthetic",
            "config": {"workload": f"{args.config}: {mat} {nx}x{ny}x{nz} points, dx={dx}, "
                                   f"{frac:.0%} pairs broken, VV step, {n_parts} partitions",
                       "partitions": n_parts, "decomposition": args.halo_decomposition, "parallelism": f"halo x{world}" if world > 1 else
                       f"{n_parts} partitions in one process", "mapping": mapping,
                       "setup_s": setup_s},
            "halo": {"ms_per_step": {k: v / args.steps for k, v in ms.items()},
                     "rows_here": rows, "halo_rows_here": halo_rows,
                     "bonds_here": all_bonds, "owned_bonds_here": owned_bonds},
            "roofline": {"bound": "hbm", "kernel": f"{mat.lower()} {dom} (rank 0's partitions)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None, "peak_kind": peak_kind,
                         "alg_bytes_per_launch": alg, "ms_per_launch": dom_ms},
            "e2e": {"value": body_bonds * e2e_steps / e2e_s, "unit": UNIT,
                    "h2d_bytes_per_step": h2d / e2e_steps, "d2h_bytes_per_step": d2h / e2e_steps,
                    "steps": e2e_steps},
            "cpu_baseline": None,
            "gpu_launches": launches, "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    pb.close()


def run_reference(args, rank, world):
    """The reference arm: the CPU restatement of the reference (Julia is not installed) on all
    host threads; every step is one Velocity Verlet step of the bounded sample."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    if args.config == "dr1m":
        b, dr, bcs, (sx, sy, sz) = dr_oracle_sample(args.config, threads)
        step = lambda n: dr.step(n, bcs)
    elif args.config == "plate3200":
        b, dt, bcs = plate_oracle(threads)
        table = bcs(1, max(args.warmup, 0) + args.steps)
        step = lambda n: b.run_vv(n, 1, dt, table)   # the table starts at step 1
        sx, sy, sz = CONFIGS["plate3200"][:3]
    else:
        b, dt, (sx, sy, sz) = oracle_sample(args.config, threads)
        step = lambda n: b.run_vv(n, 1, dt)
    for k in range(max(args.warmup, 0)):
        step(k + 1)
    t0 = time.perf_counter()
    for k in range(args.steps):
        step(args.warmup + k + 1)
    el = time.perf_counter() - t0
    v = b.n_bonds * args.steps / el
    nx, ny, nz, dx, mat, frac, vbc = CONFIGS[args.config]
    kind = "relaxation" if args.config == "dr1m" else "VV"
    sample = (f"{sx}x{sy}x{sz} sub-block ({b.n} points, {b.n_bonds} bonds) of the {args.config} "
              f"lattice and parameters, {args.steps} FP64 {kind} steps in {el:.2f} s")
    metric = "bond-updates/s per relaxation step" if args.config == "dr1m" else METRIC
    line = {"metric": metric, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * el / max(args.steps, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": args.config, "points": nx * ny * nz, "material": mat},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "cpu_model": cpu_model(), "kind": "port",
                             "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "Julia is not installed: the reference arm is the CPU restatement of the "
                    "reference (oracle/, FP64, OpenMP on all host threads)"}
    print(json.dumps(line), flush=True)


JFNK_WEIGHTS = os.path.join(ROOT, "peridynamics.jl_b200", "pdcuda", "weights", "beam_block_pc.npz")
JFNK_ARMS = ("block_jacobi", "block_poly", "learned_poly")


def _jfnk_arm(pd, mpnn, nkm, body, device, pc, G, increments, n_steps, weights, gmres_maxiter,
              newton_maxiter, budget):
    net = None
    if pc.startswith("learned"):
        if not os.path.exists(weights):
            return None
        net = mpnn.BlockPreconditionerNet.load(weights, device=device)
    dev = pd.DeviceBody(body, precision="fp64", device=device)
    dev.set_mapping(G, 256)
    nk = pd.NewtonKrylov(steps=n_steps, tol=1e-8, tol_mode="relative", frechet="forward",
                         gmres_restart=50, gmres_maxiter=gmres_maxiter,
                         maxiter=newton_maxiter, preconditioner=pc, corrections=net)
    t0 = time.perf_counter()
    nkm.setup(dev, nk)
    done = 0
    try:
        for n in range(1, increments + 1):
            nkm.step(dev, nk, n)
            done = n
            if budget and time.perf_counter() - t0 > budget:
                break
    except pd.NotConvergedError:
        pass
    t = time.perf_counter() - t0
    st = nk.stats
    dev.close()
    if net is not None:
        net.close()
    if done < increments:
        return {"s": t, "converged": False, "increments_done": done,
                "gmres_iters": sum(x["gmres_iters"] for x in st), "group": G}
    return {"s": t, "increments": increments, "group": G,
            "newton_iters": sum(x["newton_iters"] for x in st),
            "gmres_iters": sum(x["gmres_iters"] for x in st),
            "force_evals": sum(x["force_evals"] for x in st),
            "max_rel_residual": max(x["residual"] / x["residual_first"] for x in st),
            "ms_per_krylov_step": 1e3 * t / max(1, sum(x["gmres_iters"] for x in st))}


def jfnk_compare(device, increments, n_steps=20, weights=JFNK_WEIGHTS, arms=JFNK_ARMS,
                 gmres_maxiter=8000, newton_maxiter=12, groups=(4,), repeats=1):
    """The 500k-point three-point-bending beam (250 x 50 x 40 points, dx = 1 mm, E = 70 GPa,
    no fracture, mid-span line pushed 0.5 mm down over n_steps load increments): wall time
    of the first `increments` increments to a 1e-8 relative nonlinear residual per increment,
    FGMRES(50) with the forward Frechet step sqrt(eps) |u| / |v|, for each preconditioner.
    The learned arm's time includes the network's inference on the beam. Each arm runs with
    every lane mapping in `groups` (lanes per point of the force kernels): the mapping sets the
    FP64 summation order, and the finite-difference products carry that rounding into the
    Krylov counts, so several mappings give the spread of a count; the first one is the
    reported run. With repeats > 1 every arm runs that many times (the solves are
    deterministic: the same Krylov counts) and reports its fastest time, so that a transient
    clock drop of a power-capped GPU does not decide the comparison; all times are listed."""
    import pdcuda as pd
    from pdcuda import mpnn
    from pdcuda import newton_krylov as nkm
    from pdcuda.train_preconditioner import bending_beam
    body = bending_beam(250, 50, 40)
    out = {}
    budget = None  # other arms stop (reported as not converged) past 3x the block-Jacobi time
    for pc in arms:
        runs = []
        for G in groups:
            rep = []
            for _ in range(max(repeats, 1)):
                rep.append(_jfnk_arm(pd, mpnn, nkm, body, device, pc, G, increments, n_steps,
                                     weights, gmres_maxiter, newton_maxiter, budget))
            done = [r for r in rep if r is not None]
            best = (min(done, key=lambda r: (not r.get("converged", True), r["s"]))
                    if done else None)
            if best is not None and len(rep) > 1:
                best["repeats_s"] = [None if r is None else r["s"] for r in rep]
            runs.append(best)
        r0 = runs[0]
        if r0 is not None and len(runs) > 1:
            r0["spread"] = {str(G): (None if r is None else {"s": r["s"], "gmres_iters": r["gmres_iters"]})
                            for G, r in zip(groups, runs)}
        out[pc] = r0
        if pc == "block_jacobi" and r0 is not None and r0.get("converged", True):
            budget = 3.0 * r0["s"]
    bj = out.get("block_jacobi")
    for pc in arms:
        if out.get(pc) and bj and out[pc].get("converged", True):
            out[pc]["speedup_vs_block_jacobi"] = bj["s"] / out[pc]["s"]
    return {"workload": f"bond-based beam 250x50x40 points (500k), first {increments} of "
                        f"{n_steps} load increments, 1e-8 relative residual, FGMRES(50)",
            "points": body.n_points, "arms": out}


def run_jfnk(args, rank, world):
    """--config jfnk500k: every load increment of the quasi-static solve, per preconditioner."""
    if rank != 0:
        return
    import torch  # noqa: F401  (device plumbing only)
    res = jfnk_compare(int(os.environ.get("LOCAL_RANK", "0")), args.jfnk_increments,
                       arms=tuple(args.jfnk_arms.split(",")),
                       gmres_maxiter=args.jfnk_gmres_maxiter,
                       newton_maxiter=args.jfnk_newton_maxiter,
                       groups=tuple(int(g) for g in args.jfnk_groups.split(",")),
                       repeats=max(args.jfnk_repeats, 1))
    arms = res["arms"]
    ok = lambda a: a is not None and a.get("converged", True)
    ran = [arms[k] for k in ("learned_poly", "block_poly", "block_jacobi") if arms.get(k)]
    best = next((a for a in ran if ok(a)), ran[0])
    cpu = None
    if not args.no_cpu:
        bj = arms.get("block_jacobi") or {}
        cpu = jfnk_cpu_baseline(bj.get("force_evals", 0))
    line = {"metric": "JFNK wall time to 1e-8 relative residual (learned preconditioner)",
            "value": best["s"], "unit": "s", "n_gpus": 1, "steps": args.jfnk_increments,
            "warmup": 0, "higher_is_better": False, "scaling": "none", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "config": {"workload": res["workload"],
                                                            "points": res["points"]},
            "arms": arms, "cpu_baseline": cpu}
    print(json.dumps(line), flush=True)


def jfnk_cpu_baseline(force_evals, budget_s=20.0):
    """The oracle's FP64 force evaluation (all host threads) on the same beam, timed on a few
    evaluations; the projection multiplies by the block-Jacobi arm's force-evaluation count."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from twin import oracle_body
    from pdcuda.train_preconditioner import bending_beam
    threads = os.cpu_count() or 1
    O.set_threads(threads)
    ob = oracle_body(bending_beam(250, 50, 40))
    k, t0 = 0, time.perf_counter()
    while k < 2 or (time.perf_counter() - t0 < budget_s and k < 20):
        ob.force_density()
        k += 1
    per = (time.perf_counter() - t0) / k
    return {"value": per, "unit": "s per force evaluation", "cores": threads, "cpu_model": cpu_model(), "kind": "port",
            "sample": f"{k} FP64 force evaluations of the 500k-point beam",
            "projected_block_jacobi_s": per * force_evals}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default: the workload's own run, 5000 for osb8m and 500 "
                         "for plate3200; 200 otherwise)")
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="osb8m", choices=list(CONFIGS))
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--fp64-steps", type=int, default=-1, help="steps of the FP64 comparison (0 = skip)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--graph", type=int, default=50,
                    help="steps per CUDA graph of the timed Velocity Verlet run (0: eager)")
    ap.add_argument("--replicas", action="store_true",
                    help="with --gpus N > 1 on a single-body config: N independent copies of the "
                         "body (weak scaling) instead of one body in N partitions")
    ap.add_argument("--mapping", default="",
                    help="lanes per point, block size, bond-stream variant (e.g. 1,128,5) instead "
                         "of the autotuner's choice")
    ap.add_argument("--ens-classes", type=int, default=3,
                    help="ens64: size classes of specimens, each with its own mapping")
    ap.add_argument("--check-every", type=int, default=0,
                    help="FP32 run of --steps steps compared with an FP64 run of the same body "
                         "every this many steps (spot checks; prints a precision line)")
    ap.add_argument("--correction", default="none", choices=["none", "energy"],
                    help="BB / OSB with EnergySurfaceCorrection")
    ap.add_argument("--halo", action="store_true",
                    help="one body in partitions with halo exchange (one per rank) instead of replicas")
    ap.add_argument("--halo-parts", type=int, default=1,
                    help="with --halo on one GPU: partitions held by the one process")
    ap.add_argument("--halo-decomposition", default="slabs", choices=["index", "slabs"],
                    help="index: the reference's contiguous point ranges; slabs: along the longest side")
    ap.add_argument("--jfnk-increments", type=int, default=-1,
                    help="load increments of the JFNK comparison (default: 20 with --config "
                         "jfnk500k, 2 in the default run, 0 = skip)")
    ap.add_argument("--jfnk-arms", default=",".join(JFNK_ARMS))
    ap.add_argument("--jfnk-repeats", type=int, default=-1,
                    help="runs per arm, fastest reported (default: 2 beside the VV line, 1 alone)")
    ap.add_argument("--jfnk-gmres-maxiter", type=int, default=8000)
    ap.add_argument("--jfnk-newton-maxiter", type=int, default=12)
    ap.add_argument("--jfnk-groups", default="4",
                    help="lane mappings per arm (the first is reported, the others give the spread)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup
    if args.steps is None:
        own = {"osb8m": 5000, "plate3200": 500}
        args.steps = own.get(args.config, 200) if args.impl == "ours" else 200

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(local)
        import datetime
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = tdist

    if args.config == "jfnk500k":
        if args.jfnk_increments < 0:
            args.jfnk_increments = 20
        if args.impl == "reference":
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable": "the reference arm times the "
                                  "explicit-dynamics path; the JFNK CPU baseline is in cpu_baseline"}))
        else:
            run_jfnk(args, rank, world)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return
    if args.jfnk_increments < 0:
        args.jfnk_increments = 2
    if args.config == "pulse1m":
        if rank == 0 and args.impl == "ours":
            run_precision_study(args, local)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return
    if (world > 1 and args.impl == "ours" and not args.replicas and not args.halo
            and args.config in SINGLE_BODY and args.check_every <= 0):
        args.halo = True     # one body on N GPUs: partitions with halo exchange
    if args.check_every > 0:
        if rank == 0 and args.impl == "ours":
            run_spot_checks(args, local)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return
    if args.halo and args.impl == "ours":
        run_halo(args, rank, world, local, dist)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return
    if args.config == "dr1m" and args.impl == "ours":
        run_dr(args, rank, world, local, dist)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return
    if args.config == "ens64" and args.impl == "ours":
        run_ensemble(args, rank, world, local, dist)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return

    if args.impl == "reference":
        run_reference(args, rank, world)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return

    import pdcuda as pd
    nx, ny, nz, dx, mat, frac, vbc = CONFIGS[args.config]

    def barrier():
        if dist:
            import torch
            dist.barrier()
            torch.cuda.synchronize()

    from pdcuda.replicas import reduce_max

    def max_over_ranks(x):
        return reduce_max(x, dist, device=f"cuda:{local}")

    def build(prec):
        body, frac_ = make_body(args.config, correction=args.correction)
        dev = pd.DeviceBody(body, precision=prec, device=local)
        if frac_ > 0:
            dev.break_random_pairs(frac_, 0x5EED + rank)
            if args.correction == "energy":  # the correction sees the initial damage
                pd.lib().pd_esc_init(dev.h, 0)
        dt = dev.stable_timestep(0.7)
        dev.force(0.0, dt)
        return body, dev, dt

    body, dev, dt = build(args.precision)
    n_pts, n_bonds, sym = dev.info()
    if args.mapping:
        g_, b_, p_ = (int(x) for x in args.mapping.split(","))
        dev.set_mapping(g_, b_)
        dev.set_pipeline(p_)
    else:
        dev.autotune()
    dev_mapping = dev.mapping()
    step = 1
    dev.run(step, args.warmup, dt)
    step += args.warmup
    # the timed steps run as CUDA graphs of `gsteps` steps; one untimed block captures the graph
    gsteps = min(args.graph, args.steps) if args.graph > 0 else 0
    dev.set_graph(gsteps)
    if gsteps:
        dev.run(step, gsteps, dt)
        step += gsteps

    peak, peak_kind = load_peaks()
    launches0 = dev.launch_count()
    barrier()
    with ClockSampler(local) as clk:
        ms_total = dev.run_timed(step, args.steps, dt, phases=False)
        step += args.steps
        launches = dev.launch_count() - launches0
        # per-kernel durations for the roofline: the following steps (at most EAGER_STEPS),
        # issued eagerly with events around every kernel on the handle's stream
        n_launch = min(args.steps, EAGER_STEPS)
        _, ms_a, ms_b, ms_int = dev.run_timed(step, n_launch, dt)
        step += n_launch
    barrier()
    ms_max = max_over_ranks(ms_total)
    value = n_bonds * args.steps * world / (ms_max / 1e3)
    clocks = clk.summary()

    # roofline of the dominant kernel (per launch, algorithmic bytes)
    prec = args.precision
    per_kernel = {"phase_a": ms_a / n_launch, "phase_b": ms_b / n_launch}
    dom = max(per_kernel, key=per_kernel.get) if mat != "BB" else "phase_a"
    dom_ms = per_kernel[dom]
    # bytes a launch of one force phase must move: every bond once (nbr, geometry, state bit)
    # and its per-point reads / writes
    if prec == "fp32":
        pt_bytes = {"phase_a": 32 + 8 + 16 + 4 + 4, "phase_b": 32 + 8 + 16 + 12 + 4}[dom]
    else:
        pt_bytes = {"phase_a": 64 + 8 + 32 + 4 + 4, "phase_b": 64 + 8 + 32 + 24 + 4}[dom]
    b_bond = B_BOND[prec] + (({"fp32": 4.0, "fp64": 8.0}[prec]) if args.correction == "energy" else 0.0)
    alg_bytes = n_bonds * b_bond + n_pts * pt_bytes
    achieved = alg_bytes / (dom_ms / 1e3) / 1e9
    # DRAM traffic per launch from the committed ncu capture, scaled by the bond count
    traffic = None
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            tb = json.load(f)["dram_bytes_per_bond"]
        key = {"phase_a": f"{mat.lower()}_phase_a", "phase_b": f"{mat.lower()}_phase_b"}[dom]
        if prec == "fp32" and key in tb:
            traffic = tb[key] * n_bonds
    except Exception:
        traffic = None
    step_bytes = n_bonds * b_bond + n_pts * (B_POINT[prec] + B_POINT_EXTRA[mat])
    step_ms = ms_max / args.steps
    step_achieved = step_bytes / (step_ms / 1e3) / 1e9

    # FP64 comparison on the same workload
    fp64 = None
    f64_steps = args.fp64_steps if args.fp64_steps >= 0 else min(max(args.steps // 4, 10), 250)
    if prec == "fp32" and f64_steps > 0:
        dev.close()
        _, d64, dt64 = build("fp64")
        d64.autotune()
        d64.run(1, 3, dt64)
        barrier()
        t64 = d64.run_timed(4, f64_steps, dt64)[0]
        barrier()
        t64 = max_over_ranks(t64)
        fp64 = n_bonds * f64_steps * world / (t64 / 1e3)
        d64.close()
        _, dev, dt = build(prec)
        # the tuned mapping of the timed run, so that e2e runs the same kernels
        dev.set_mapping(dev_mapping[0], dev_mapping[1])
        dev.set_pipeline(dev_mapping[2])
        dev.set_graph(gsteps)

    # end to end through the public API with host buffers: upload the state, run, read back
    # (page-locked host buffers)
    bufs = [pinned(n_pts, 3), pinned(n_pts, 3), pinned(n_pts, 3), pinned(n_pts)]
    h_u, h_v, out_u, out_d = (b[1] for b in bufs)
    # untimed warm-up through the same calls (the rebuilt handle captures its graph here)
    dev.set_state(displacement=h_u, velocity=h_v)
    dev.run(1, max(args.warmup, 3, gsteps), dt)
    dev.field("displacement", out=out_u)
    barrier()
    e2e_steps = min(args.steps, EAGER_STEPS)
    t0 = time.perf_counter()
    dev.set_state(displacement=h_u, velocity=h_v)
    dev.run(1, e2e_steps, dt)
    dev.field("displacement", out=out_u)
    dev.field("damage", out=out_d)
    e2e_s = time.perf_counter() - t0
    e2e_s = max_over_ranks(e2e_s)
    h2d = (h_u.nbytes + h_v.nbytes) / e2e_steps
    d2h = (out_u.nbytes + out_d.nbytes) / e2e_steps
    e2e = n_bonds * e2e_steps * world / e2e_s

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(args.config, os.cpu_count() or 1, correction=args.correction)
    dev.close()
    jfnk = None
    if rank == 0 and world == 1 and args.jfnk_increments > 0:
        jfnk = jfnk_compare(local, args.jfnk_increments,
                            repeats=args.jfnk_repeats if args.jfnk_repeats > 0 else 2)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32" if prec == "fp32" else "f64",
            "data": "synthetic",
            "config": {"workload": f"{args.config}: {mat} {nx}x{ny}x{nz} points, dx={dx}, "
                                   f"horizon 3.015dx, {frac:.0%} pairs broken, VV step"
                                   + (", EnergySurfaceCorrection" if args.correction == "energy" else ""),
                       "points": n_pts, "bonds": n_bonds, "precision": prec,
                       "mapping": dict(zip(("group", "block", "pipe"), dev_mapping)),
                       "symmetric_pairs": bool(sym), "graph_steps": gsteps,
                       "l2": ("inputs larger than L2 (bond arrays of "
                              f"{n_bonds * B_BOND[prec] / 1e9:.1f} GB)" if n_bonds * B_BOND[prec] > 126e6
                              else "inputs smaller than L2: the plate job as stated (L2 not flushed)"),
                       "parallelism": f"replicas x{world}"},
            "roofline": {"bound": "hbm", "kernel": f"{mat.lower()} force {dom}",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "traffic_source": "profiles/traffic.json (ncu DRAM counters of both "
                                           "phases captured on the 8M-point block, per bond)",
                         "alg_bytes_per_launch": alg_bytes, "ms_per_launch": dom_ms},
            "roofline_step": {"achieved": step_achieved, "peak": peak, "frac": step_achieved / peak,
                              "alg_bytes_per_step": step_bytes,
                              "ms": {"phase_a": ms_a / n_launch, "phase_b": ms_b / n_launch,
                                     "integrate": ms_int / n_launch}},
            "fp64_value": fp64, "fp32_over_fp64": (value / fp64) if fp64 else None,
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "steps": e2e_steps},
            "gpu_launches": launches, "clocks": clocks, "cpu_baseline": cpu,
            "jfnk": jfnk,
            "timing": (f"value: the timed steps as CUDA graphs of graph_steps steps between two "
                       f"events; roofline: the next {n_launch} steps issued eagerly with events "
                       f"around every kernel" if gsteps else
                       f"value: eager launches between two events; roofline: the next {n_launch} "
                       f"steps with events around every kernel"),
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
