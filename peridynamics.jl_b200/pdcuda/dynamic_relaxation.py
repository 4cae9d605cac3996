"""DynamicRelaxation: adaptive dynamic relaxation on the device.

Mirrors src/time_solvers/dynamic_relaxation.jl of the reference: the keyword constructor and
its checks (:40-56), and solve! (:92-107) with init_density_matrix! and relaxation_timestep!
running as ``pd_dr_init`` / ``pd_run_dr``: the conditions and drift, the same force kernels
as Velocity Verlet, the global damping coefficient and the velocity update stay on the device.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L


class DynamicRelaxation:
    """Dynamic relaxation (dynamic_relaxation.jl:40-56); ArgumentError -> ValueError."""

    def __init__(self, steps, stepsize=1.0, damping_factor=1.0):
        if steps <= 0:
            raise ValueError("`steps` should be larger than zero!\n")
        if stepsize <= 0:
            raise ValueError("`stepsize` should be larger than zero!\n")
        if damping_factor <= 0:
            raise ValueError("`damping_factor` should be larger than zero!\n")
        self.n_steps = int(steps)
        self.dt = float(stepsize)
        self.damping_factor = float(damping_factor)

    def __repr__(self):
        return (f"DynamicRelaxation(n_steps={self.n_steps}, Δt={self.dt}, "
                f"Λ={self.damping_factor})")


def density_matrix(dev):
    out = np.empty(dev.n)
    L.check(L.lib().pd_dr_density_matrix(dev.h, L.ptr(out)), "pd_dr_density_matrix")
    return out


def run(dev, dr, first_step, n_steps):
    """relaxation_timestep! for n_steps steps from first_step (conditions tabulated first)."""
    dev.tabulate_bcs(first_step, n_steps, dr.dt)
    st = L.lib().pd_run_dr(dev.h, first_step, n_steps)
    if st == L.PD_ERR_NAN:
        step = C.c_int64(-1)
        L.lib().pd_nan_step(dev.h, C.byref(step))
        raise L.NaNError(step.value * dr.dt, step.value)
    L.check(st, "pd_run_dr")


def run_timed(dev, dr, first_step, n_steps):
    """run() with CUDA events around every phase: (total, conditions + drift, force,
    damping + velocity update) milliseconds summed over the steps."""
    dev.tabulate_bcs(first_step, n_steps, dr.dt)
    out = [C.c_double() for _ in range(4)]
    st = L.lib().pd_run_dr_timed(dev.h, first_step, n_steps, *[C.byref(o) for o in out])
    if st == L.PD_ERR_NAN:
        step = C.c_int64(-1)
        L.lib().pd_nan_step(dev.h, C.byref(step))
        raise L.NaNError(step.value * dr.dt, step.value)
    L.check(st, "pd_run_dr_timed")
    return tuple(o.value for o in out)


def init(dev, dr):
    """init_density_matrix! and the force evaluation at t = 0 of initialize!."""
    L.check(L.lib().pd_dr_init(dev.h, dr.dt, dr.damping_factor), "pd_dr_init")
    dev.force(0.0, dr.dt)


def solve(dev, dr, export=None, freq=0):
    """initialize! (a force evaluation at t = 0) and solve! (dynamic_relaxation.jl:92-107),
    exporting at step 0 and after every block of freq steps."""
    init(dev, dr)
    if export is not None:
        export(0, 0.0, dev)
    block = freq if (export is not None and freq > 0) else dr.n_steps
    n = 1
    while n <= dr.n_steps:
        k = min(block, dr.n_steps - n + 1)
        run(dev, dr, n, k)
        n += k
        if export is not None:
            export(n - 1, (n - 1) * dr.dt, dev)
    return dev
