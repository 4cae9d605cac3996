"""NewtonKrylov: the quasi-static Jacobian-free Newton-Krylov solver on the device.

Mirrors src/time_solvers/newton_krylov.jl of the reference: the keyword constructor and its
checks (:47-130), ``newton_krylov_check`` (:256-276), the validation of the body
(validate_chunk_for_newton_krylov!, :219-253) and ``solve!`` (:280-295). Each load increment
runs as one ``pd_nk_step`` call: the Newton iterations, the Frechet Jacobian-vector products
and the (F)GMRES solves all stay on the device.

Beyond the reference's keywords: ``frechet`` ("central", the reference's rule, or "forward":
eps = sqrt(eps_mach) |u| / |v|, one force evaluation per product), ``tol_mode`` ("absolute",
the reference's ``||r|| < tol``, or "relative": ``||r|| <= tol ||r_first||`` per increment) and
``preconditioner`` ("none", the reference's plain GMRES; "block_jacobi"; "block_poly";
"learned_poly" and "learned", which need per-point corrections from a trained
``pdcuda.mpnn`` network or an array of 9 floats per point).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib as L

_PC = {"none": L.PC_NONE, "block_jacobi": L.PC_BLOCK_JACOBI, "block_poly": L.PC_BLOCK_POLY,
       "learned_poly": L.PC_LEARNED_POLY, "learned": L.PC_LEARNED}
_FRECHET = {"central": L.NK_CENTRAL, "forward": L.NK_FORWARD}


class NewtonKrylov:
    """Quasi-static solver (newton_krylov.jl:47-130); ArgumentError -> ValueError."""

    def __init__(self, time=-1.0, steps=-1, stepsize=1.0, maxiter=100, tol=1e-4,
                 perturbation_scale=1.0, gmres_maxiter=200, gmres_reltol=1e-4,
                 gmres_abstol=1e-8, gmres_restart=100, frechet="central", tol_mode="absolute",
                 preconditioner="none", corrections=None):
        if time > 0 and steps > 0:
            raise ValueError("specify either time or number of steps, not both!")
        if time < 0 and steps < 0:
            raise ValueError("specify either time or number of steps!")
        if stepsize <= 0:
            raise ValueError("stepsize has to be larger than zero: stepsize > 0")
        if time > 0:
            self.n_steps = int(math.ceil(time / stepsize))
            self.end_time = float(time)
        else:
            self.n_steps = int(steps)
            self.end_time = steps * float(stepsize)
        self.dt = float(stepsize)
        checks = (("maxiter", maxiter), ("tol", tol), ("gmres_reltol", gmres_reltol),
                  ("gmres_abstol", gmres_abstol), ("gmres_maxiter", gmres_maxiter),
                  ("gmres_restart", gmres_restart), ("perturbation_scale", perturbation_scale))
        for name, v in checks:
            if v <= 0:
                what = "tolerance" if name == "tol" else name
                raise ValueError(f"{what} has to be larger than zero: {name} > 0")
        if frechet not in _FRECHET:
            raise ValueError(f"frechet must be one of {sorted(_FRECHET)}")
        if tol_mode not in ("absolute", "relative"):
            raise ValueError("tol_mode must be 'absolute' or 'relative'")
        if preconditioner not in _PC:
            raise ValueError(f"preconditioner must be one of {sorted(_PC)}")
        self.maxiter = int(maxiter)
        self.tol = float(tol)
        self.perturbation_scale = float(perturbation_scale)
        self.gmres_maxiter = int(gmres_maxiter)
        self.gmres_reltol = float(gmres_reltol)
        self.gmres_abstol = float(gmres_abstol)
        self.gmres_restart = int(gmres_restart)
        self.frechet = frechet
        self.tol_mode = tol_mode
        self.preconditioner = preconditioner
        self.corrections = corrections
        self.stats = []

    def check(self):
        """newton_krylov_check (newton_krylov.jl:256-276); ErrorException -> RuntimeError."""
        for name, label in (("end_time", "end_time"), ("n_steps", "n_steps"), ("dt", "Δt"),
                            ("maxiter", "maxiter"), ("tol", "tol")):
            if getattr(self, name) < 0:
                raise RuntimeError(f"`{label}` of NewtonKrylov smaller than zero!\n")
        if self.perturbation_scale <= 0:
            raise RuntimeError("`perturbation_scale` of NewtonKrylov must be larger than zero!\n")

    def params(self):
        p = L.NKParams()
        p.maxiter = self.maxiter
        p.tol = self.tol
        p.tol_relative = 1 if self.tol_mode == "relative" else 0
        p.perturbation_scale = self.perturbation_scale
        p.frechet = _FRECHET[self.frechet]
        p.gmres_maxiter = self.gmres_maxiter
        p.gmres_reltol = self.gmres_reltol
        p.gmres_abstol = self.gmres_abstol
        p.gmres_restart = self.gmres_restart
        p.precond = _PC[self.preconditioner]
        return p

    def __repr__(self):
        return (f"NewtonKrylov(end_time={self.end_time}, n_steps={self.n_steps}, "
                f"Δt={self.dt}, maxiter={self.maxiter}, tol={self.tol}, "
                f"perturbation_scale={self.perturbation_scale}, "
                f"gmres_maxiter={self.gmres_maxiter}, gmres_reltol={self.gmres_reltol}, "
                f"gmres_abstol={self.gmres_abstol}, gmres_restart={self.gmres_restart})")


def validate_body(body):
    """validate_chunk_for_newton_krylov! (newton_krylov.jl:219-253) on the body."""
    n = len(body.single_dim_bcs) + len(body.posdep_single_dim_bcs) + len(body.data_bcs)
    if n > 0:
        raise ValueError("NewtonKrylov solver does not support all boundary condition types!\n"
                         "Specify only position-dependent boundary conditions!")
    for i in range(body.n_points):
        k = body.params_map[i]
        if k > 0 and body.point_params[k - 1].has_fracture:
            raise ValueError("NewtonKrylov solver currently does not support damage or "
                             f"fracture!\nFracture parameters found at point index {i + 1}!\n")


def condition_table(body):
    """pos_single_dim_bcs evaluated at the reference positions: one pd_nk_condition each
    (the host evaluates f(p); the device scales by beta every increment)."""
    conds, keep = [], []
    for c in body.pos_single_dim_bcs:
        pts = np.ascontiguousarray(body.point_sets[c.point_set], np.int32)
        vals = np.array([float(c.fun(body._pos[i])) for i in pts], np.float64)
        field = L.NKC_DISPLACEMENT if c.field == "displacement" else L.NKC_B_EXT
        k = L.NKCondition(field, c.dim, len(pts), L.ptr(pts), L.ptr(vals))
        conds.append(k)
        keep += [pts, vals]
    return conds, keep


def setup(dev, nk):
    """Upload the conditions (and learned corrections) of the body to the device body."""
    nk.check()
    validate_body(dev.body)
    if dev.precision != "fp64":
        raise ValueError("the Newton-Krylov solve needs precision='fp64'")
    lib = L.lib()
    conds, keep = condition_table(dev.body)
    arr = (L.NKCondition * max(len(conds), 1))(*conds)
    L.check(lib.pd_nk_set_conditions(dev.h, len(conds), C.cast(arr, C.c_void_p)),
            "pd_nk_set_conditions")
    if nk.preconditioner in ("learned", "learned_poly"):
        D = nk.corrections
        if D is None:
            raise ValueError("the learned preconditioner needs corrections (a trained network "
                             "or 9 floats per point)")
        if hasattr(D, "corrections"):
            D = D.corrections(dev)
        D = np.ascontiguousarray(D, np.float32).reshape(dev.n, 9)
        L.check(lib.pd_nk_set_corrections(dev.h, L.ptr(D)), "pd_nk_set_corrections")


def step(dev, nk, n):
    """newton_krylov_step! (newton_krylov.jl:298-332) for load increment n."""
    st = L.NKStats()
    p = nk.params()
    status = L.lib().pd_nk_step(dev.h, n, n / nk.n_steps, C.byref(p), C.byref(st))
    nk.stats.append(st.as_dict())
    if status == L.PD_ERR_NAN:
        raise L.NaNError(n * nk.dt, n)
    L.check(status, "pd_nk_step")
    return st


def solve(dev, nk, export=None, freq=0):
    """solve! (newton_krylov.jl:280-295): every increment, exports at multiples of freq."""
    setup(dev, nk)
    if export is not None:
        export(0, 0.0, dev)
    for n in range(1, nk.n_steps + 1):
        step(dev, nk, n)
        if export is not None and freq > 0 and (n % freq == 0 or n == nk.n_steps):
            export(n, n * nk.dt, dev)
    return dev


_OPS = {"jv": 0, "k0": 1, "precond": 2, "residual": 3}


def apply_operator(dev, nk, op, v=None):
    """One operator of the solve at the current device state (tests and diagnostics):
    "jv" (the Frechet product of nk), "k0", "precond" (nk.preconditioner) or "residual"."""
    out = np.empty(3 * dev.n)
    vv = None if v is None else np.ascontiguousarray(v, np.float64).reshape(-1)
    p = nk.params()
    L.check(L.lib().pd_nk_apply(dev.h, _OPS[op], C.byref(p), L.ptr(vv), L.ptr(out)),
            "pd_nk_apply")
    return out


def record(dev, capacity):
    """Keep the unit residual direction of every Krylov (re)start, up to capacity vectors."""
    L.check(L.lib().pd_nk_record(dev.h, int(capacity)), "pd_nk_record")


def recorded(dev):
    n = C.c_int64()
    L.check(L.lib().pd_nk_recorded(dev.h, C.byref(n)), "pd_nk_recorded")
    return n.value


def recorded_vector(dev, k):
    """Recorded residual direction k (3n floats)."""
    out = np.empty(3 * dev.n, np.float32)
    L.check(L.lib().pd_nk_recorded_vector(dev.h, int(k), L.ptr(out)), "pd_nk_recorded_vector")
    return out
