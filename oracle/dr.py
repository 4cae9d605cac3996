"""CPU restatement of the reference's dynamic relaxation (test infrastructure).

Follows src/time_solvers/dynamic_relaxation.jl of Peridynamics.jl on top of the FP64 force
restatement (``OracleBody.force_density``), in the reference's operation order:
  calc_density_matrix!     :153-164   Lambda_i = f / 4 dt^2 n_i (5 pi delta^2 bc), per dof
  relaxation_timestep!     :191-211   conditions at t = n dt, u += v_half dt, x += v_half dt,
                                      force density, damping (n > 1), velocity update
  damping_terms / combine / finish_damping  :269-317   compensated sums (TwoSum), one chunk
  relaxation_first_step! / relaxation_step! / relaxation_updates!  :337-370
Conditions come as the dictionaries of tests/helpers.oracle_bcs (kinds: 0 = f(t) per step,
1 = f(p, t) per point per step, 2 = constant data), applied as apply_boundary_conditions!
(boundary_conditions.jl:37-51, 98-108, 198-226): finite values overwrite the field.

Only tests/ import this module.
"""
from __future__ import annotations

import math

import numpy as np

FIVE_PI = 5 * math.pi


def density_matrix(ob, dt, factor=1.0):
    """Lambda per point (the reference stores it per dof, the same for x, y, z)."""
    n_b = np.diff(ob.off).astype(np.float64)
    out = np.empty(ob.n)
    for i in range(ob.n):
        p = ob.params_list[ob.pid[i]]
        k = FIVE_PI * (p.delta * p.delta) * p.bc
        out[i] = factor * 1 / 4 * (dt * dt) * n_b[i] * k
    return out


def two_sum(a, b):
    s = a + b
    v = s - a
    return s, (a - (s - v)) + (b - v)


def finish_damping(cn1, cn2):
    cn = 0.0
    if cn2 != 0.0 and cn1 / cn2 > 0.0:
        cn = 2.0 * math.sqrt(cn1 / cn2)
    if cn > 2.0:
        cn = 1.9
    return cn


class OracleDR:
    """fast=True sums the damping terms with numpy (pairwise, not the reference's order): the
    timed CPU baseline of large samples; the parity tests use the ordered loop."""

    def __init__(self, ob, dt, factor=1.0, fast=False):
        self.ob, self.dt, self.fast = ob, float(dt), fast
        self.lam = density_matrix(ob, dt, factor)
        self.vh_old = np.zeros((ob.n, 3))
        self.b_old = np.zeros((ob.n, 3))
        self.last_cn = 0.0

    def damping(self):
        ob, dt = self.ob, self.dt
        u, vh, b = ob.u.reshape(-1), ob.vh.reshape(-1), ob.b_int.reshape(-1)
        vho, bo = self.vh_old.reshape(-1), self.b_old.reshape(-1)
        lam = np.repeat(self.lam, 3)
        with np.errstate(divide="ignore", invalid="ignore"):
            if self.fast:
                m = vh != 0.0
                t1 = -(u[m] * u[m]) * (b[m] - bo[m]) / (dt * lam[m] * vho[m])
                return finish_damping(float(np.sum(t1)), float(np.dot(u, u)))
            return self._damping_sums(u, vh, b, vho, bo, lam, dt)

    @staticmethod
    def _damping_sums(u, vh, b, vho, bo, lam, dt):
        cn1 = cn1c = cn2 = cn2c = 0.0
        for q in range(u.size):
            if vh[q] != 0.0:
                # a dof held by a velocity condition whose previous update gave 0 divides by
                # zero here; the resulting NaN sum makes cn 0, as in the reference
                db = b[q] - bo[q]
                temp = dt * lam[q] * vho[q]
                cn1, e = two_sum(cn1, -(u[q] * u[q]) * db / temp)
                cn1c += e
            cn2, e = two_sum(cn2, u[q] * u[q])
            cn2c += e
        return finish_damping(cn1 + cn1c, cn2 + cn2c)

    def apply_conditions(self, bcs, n):
        ob = self.ob
        for bc in bcs:
            field = ob.vh if bc["field"] == 0 else ob.b_ext
            pts = np.asarray(bc["pts"])
            row = n - bc.get("first_step", 1)
            if bc["kind"] == 0:
                vals = np.full(len(pts), bc["values"][row])
            elif bc["kind"] == 1:
                vals = np.asarray(bc["values"]).reshape(-1, len(pts))[row]
            else:
                vals = np.asarray(bc["values"])
            ok = np.isfinite(vals)
            field[pts[ok], bc["dim"]] = vals[ok]

    def step(self, n, bcs=()):
        """relaxation_timestep! for step n >= 1."""
        ob, dt = self.ob, self.dt
        t = n * dt
        self.apply_conditions(bcs, n)
        du = ob.vh * dt
        ob.u += du
        ob.pos += du
        ob.force_density(t, dt)
        lam = self.lam[:, None]
        b = ob.b_int + ob.b_ext
        if n == 1:
            vh = 0.5 * dt * b / lam
        else:
            cn = self.last_cn = self.damping()
            a = b / lam
            vh = ((2 - cn * dt) * self.vh_old + 2 * dt * a) / (2 + cn * dt)
        ob.vh[:] = vh
        ob.v[:] = 0.5 * (self.vh_old + ob.vh)
        self.vh_old[:] = ob.vh
        self.b_old[:] = ob.b_int
