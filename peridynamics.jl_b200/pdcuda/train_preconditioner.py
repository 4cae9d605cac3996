"""Train the learned block preconditioner on seeded three-point-bending beams.

    python -m pdcuda.train_preconditioner --out weights.npz [--steps 300] [--seed 0]

(run from peridynamics.jl_b200/ with a CUDA device). The beams are bond-based lattices of
100k-300k points at dx = 1 mm with seeded load depths and support positions; each runs two
plain block-Jacobi FGMRES(50) load increments with its Krylov residual directions recorded
(``pd_nk_record``), then the network is trained on the fast end of their preconditioned
spectra (``mpnn.train``). The weights shipped in weights/beam_block_pc.npz were made by this
script with its defaults.
"""
from __future__ import annotations

import argparse
import time

import numpy as np

from . import body as B
from . import mpnn
from .materials import BBMaterial
from .newton_krylov import NewtonKrylov
from .solver import DeviceBody

# (nx, ny, nz) of the training beams: 100k, 200k and 300k points
TRAIN_SHAPES = ((200, 25, 20), (200, 40, 25), (240, 50, 25))


def bending_beam(nx, ny, nz, dx=1e-3, load=-0.5e-3, support=20, E=70e9, rho=2700.0):
    """Three-point bending of a bond-based beam (x span, y height, z width), horizon
    3.015 dx, no fracture: the bottom lines `support` points in from both ends are fixed in
    x, y and z; the top line at mid-span (the points within dx / 2 of x = 0) is displaced by
    `load` in y (reached at the last load increment)."""
    pos, vol = B.uniform_box(nx * dx, ny * dx, nz * dx, dx)
    body = B.Body(BBMaterial(), pos, vol)
    B.material(body, horizon=3.015 * dx, rho=rho, E=E)
    x, y = pos[0], pos[1]
    xl, xr = x.min() + support * dx, x.max() - support * dx
    bottom = np.abs(y - y.min()) < dx / 2
    sup = np.nonzero(bottom & ((np.abs(x - xl) < dx / 2) | (np.abs(x - xr) < dx / 2)))[0]
    top = np.nonzero((np.abs(y - y.max()) < dx / 2) & (np.abs(x) <= dx / 2 + 1e-12))[0]
    B.point_set(body, "support", sup)
    B.point_set(body, "load", top)
    for d in ("x", "y", "z"):
        B.displacement_bc(lambda p: 0.0, body, "support", d)
    B.displacement_bc(lambda p: load, body, "load", "y")
    return body


def plain_solver(n_steps=20):
    return NewtonKrylov(steps=n_steps, tol=1e-8, tol_mode="relative", frechet="forward",
                        gmres_restart=50, gmres_maxiter=50000, maxiter=20,
                        preconditioner="block_jacobi")


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--out", required=True)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    rng = np.random.default_rng(a.seed)
    devs = []
    for shape in TRAIN_SHAPES:
        load = -rng.uniform(0.3e-3, 0.7e-3)
        support = int(rng.integers(10, 31))
        body = bending_beam(*shape, load=load, support=support)
        dev = DeviceBody(body, precision="fp64", device=a.device)
        dev.autotune()
        t0 = time.time()
        nk = plain_solver()
        n = mpnn.collect(dev, nk, 2, 64)
        its = sum(s["gmres_iters"] for s in nk.stats)
        print(f"beam {shape} ({body.n_points} points, load {load * 1e3:.2f} mm, support {support}): "
              f"{n} Krylov directions, {its} block-Jacobi Krylov steps, {time.time() - t0:.1f} s",
              flush=True)
        devs.append(dev)
    net = mpnn.BlockPreconditionerNet(seed=a.seed, device=a.device)
    t0 = time.time()
    mpnn.train(net, devs, a.steps, lr=a.lr, seed=a.seed, log=lambda m: print(m, flush=True))
    print(f"trained {a.steps} steps in {time.time() - t0:.1f} s", flush=True)
    for dev in devs:
        net.infer(dev)
        q = mpnn.top_modes(dev, 2, iters=40, learned=True)
        print(f"top eigenvalue of K0 B on {dev.n} points: "
              f"{max(mpnn.rayleigh(dev, v) for v in q):.3f}", flush=True)
    net.save(a.out)
    return net


if __name__ == "__main__":
    main()
