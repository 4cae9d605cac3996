"""CPU restatement of the reference's quasi-static Newton-Krylov solver (test infrastructure).

Follows src/time_solvers/newton_krylov.jl of Peridynamics.jl on top of the FP64 force
restatement of ``pd_oracle.c`` (``OracleBody.force_density``):
  newton_krylov_step!            :298-332   (``OracleNK.step``)
  apply_incr_boundary_conditions! boundary_conditions.jl:229-236, apply_psdbc! :154-163
  update_position!               :349-357
  calc_residual!                 :371-387
  solve_linear_system!           :415-460   (restarted GMRES, ``gmres``)
  compute_perturbation           :537-567   (central rule; the forward rule is the variant
                                             eps = sqrt(eps_mach) |u| / |v|)
  jacobian_vector_product! and the store / restore helpers :504-532, 569-671
  update_displacement_from_du!   :673-686
GMRES itself comes from IterativeSolvers.jl (``gmres!``, version 0.9 per the reference's
[compat]); its published algorithm -- restarted GMRES with modified Gram-Schmidt Arnoldi,
Givens rotations, stop when the estimated residual <= max(reltol ||b||, abstol) or after
maxiter iterations -- is restated in ``gmres``. The Krylov arithmetic is not pinned by a
golden vector of the reference; the solves are judged by the true nonlinear residual.

Also here, as the checker of the device preconditioners: the analytic 3x3 diagonal blocks of
the bond-based Jacobian (block Jacobi) and the small-strain bond stiffness K0.

Only tests/ and bench.py's CPU baseline import this module.
"""
from __future__ import annotations

import math

import numpy as np

EPS = 2.220446049250313e-16


class OracleNK:
    """The Newton-Krylov solve of one OracleBody with position-dependent conditions.

    conds: list of (field, dim, points, values) with field "displacement" or "b_ext" and
    values = f(p) at the reference positions (full load)."""

    def __init__(self, ob, conds):
        self.ob = ob
        self.n = ob.n
        self.conds = [(f, int(d), np.asarray(p, np.int64), np.asarray(v, np.float64))
                      for f, d, p, v in conds]
        self.cmask = np.zeros(3 * self.n, bool)
        for f, d, p, _ in self.conds:
            if f == "displacement":
                self.cmask[3 * p + d] = True
        self.V = ob.vol

    # -- state ------------------------------------------------------------------------------
    def apply_conditions(self, beta):
        u = self.ob.u
        for f, d, p, v in self.conds:
            val = beta * v
            ok = np.isfinite(val)
            if f == "displacement":
                u[p[ok], d] = val[ok]
            else:
                self.ob.b_ext[p[ok], d] = val[ok]
        # update_position! for the constrained dofs
        pos, X = self.ob.pos.reshape(-1), self.ob.X.reshape(-1)
        q = np.nonzero(self.cmask)[0]
        pos[q] = X[q] + u.reshape(-1)[q]

    def force(self):
        self.ob.force_density()
        return self.ob.b_int.reshape(-1).copy()

    def residual(self):
        b = self.force()
        r = (b + self.ob.b_ext.reshape(-1)) * np.repeat(self.V, 3)
        r[self.cmask] = 0.0
        return r

    def _set_pos(self, udisp):
        self.ob.pos[:] = self.ob.X + udisp.reshape(-1, 3)

    def jv(self, v, rule="central", scale=1.0, Fu=None):
        """J v by finite differences (jacobian_vector_product!, compute_perturbation)."""
        u = self.ob.u.reshape(-1).copy()
        un = math.sqrt(float(np.dot(u, u)))
        vn = math.sqrt(float(np.dot(v, v)))
        if vn < EPS:
            vn = 1.0
        V3 = np.repeat(self.V, 3)
        if rule == "central":
            eps = scale * np.cbrt(EPS) * (un + 1.0) / vn
            self._set_pos(u + eps * v)
            fp = self.force() * V3
            self._set_pos(u - eps * v)
            fm = self.force() * V3
            out = (fp - fm) / (2 * eps)
        else:
            eps = scale * math.sqrt(EPS) * (un if un > 0 else 1.0) / vn
            if Fu is None:
                self._set_pos(u)
                Fu = self.force() * V3
            self._set_pos(u + eps * v)
            out = (self.force() * V3 - Fu) / eps
        out[self.cmask] = v[self.cmask]
        self._set_pos(u)
        return out

    # -- preconditioners (bond-based) -------------------------------------------------------
    def _bonds(self):
        ob = self.ob
        i = np.repeat(np.arange(ob.n), np.diff(ob.off))
        j = ob.nbr.astype(np.int64)
        act = ob.bond_active[: ob.n_bonds].astype(bool)
        bc = np.array([p.bc for p in ob.params_list])
        c = bc[ob.pid[i]]
        if len(ob.params_list) > 1:
            c = 0.5 * (bc[ob.pid[i]] + bc[ob.pid[j]])
        return i[act], j[act], ob.L[act], c[act]

    def bj_blocks(self):
        """P_i = J_ii^-1 with J_ii = -V_i sum_j V_j c [(1/L - 1/l) I + d d^T / l^3]; rows and
        columns of constrained dofs are the identity."""
        ob = self.ob
        i, j, L, c = self._bonds()
        d = ob.pos[j] - ob.pos[i]
        l = np.linalg.norm(d, axis=1)
        s = c * self.V[j] * self.V[i]
        a = s * (1.0 / L - 1.0 / l)
        g = s / l ** 3
        K = a[:, None, None] * np.eye(3) + g[:, None, None] * d[:, :, None] * d[:, None, :]
        J = np.zeros((ob.n, 3, 3))
        np.add.at(J, i, -K)
        cm = self.cmask.reshape(-1, 3)
        for a_ in range(3):
            for b_ in range(3):
                m = cm[:, a_] | cm[:, b_]
                J[m, a_, b_] = 1.0 if a_ == b_ else 0.0
        det = np.linalg.det(J)
        bad = ~(np.abs(det) > 0) | ~np.isfinite(det)
        J[bad] = np.eye(3)
        return np.linalg.inv(J)

    def k0(self, v):
        """K0 v: V_i sum_j c V_j / L^3 (xi . (v_j - v_i)) xi, xi = X_j - X_i; constrained
        rows 0."""
        ob = self.ob
        i, j, L, c = self._bonds()
        xi = ob.X[j] - ob.X[i]
        v3 = v.reshape(-1, 3)
        k = c * self.V[j] / L ** 3
        pr = k * np.einsum("bk,bk->b", xi, v3[j] - v3[i])
        out = np.zeros((ob.n, 3))
        np.add.at(out, i, pr[:, None] * xi)
        out = (out * self.V[:, None]).reshape(-1)
        out[self.cmask] = 0.0
        return out

    def precond(self, kind, v, P=None, D=None):
        """M v of the device preconditioners (block Jacobi, block poly, learned forms)."""
        if kind == "none":
            return v.copy()
        P = self.bj_blocks() if P is None else P
        B = P if D is None else np.einsum("nab,nbc->nac", P, np.eye(3) + D)
        cm = self.cmask

        def bm(w):
            z = np.einsum("nab,nb->na", B, w.reshape(-1, 3)).reshape(-1)
            z[cm] = 0.0
            return z

        if kind in ("block_jacobi", "learned"):
            return bm(v)
        t = bm(v)
        return bm(2.0 * v - self.k0(t))

    # -- linear and nonlinear solves ----------------------------------------------------------
    def gmres(self, rhs, matvec, prec, maxiter, reltol, abstol, restart):
        """Restarted right-preconditioned GMRES from x = 0 (prec = identity: plain GMRES),
        modified Gram-Schmidt Arnoldi, Givens rotations."""
        x = np.zeros_like(rhs)
        r = rhs.copy()
        beta = np.linalg.norm(r)
        tol = max(reltol * beta, abstol)
        it = 0
        if beta <= tol:
            return x, it
        while True:
            m = restart
            Vb = [r / beta]
            Zb = []
            H = np.zeros((m + 1, m))
            cs, sn = np.zeros(m), np.zeros(m)
            g = np.zeros(m + 1)
            g[0] = beta
            cols = 0
            stop = False
            for jj in range(m):
                z = prec(Vb[jj])
                Zb.append(z)
                w = matvec(z)
                it += 1
                for q in range(jj + 1):
                    H[q, jj] = np.dot(Vb[q], w)
                    w = w - H[q, jj] * Vb[q]
                hnext = np.linalg.norm(w)
                H[jj + 1, jj] = hnext
                Vb.append(w / hnext if hnext > 0 else w)
                for q in range(jj):
                    a = cs[q] * H[q, jj] + sn[q] * H[q + 1, jj]
                    H[q + 1, jj] = -sn[q] * H[q, jj] + cs[q] * H[q + 1, jj]
                    H[q, jj] = a
                rho = math.hypot(H[jj, jj], H[jj + 1, jj])
                cs[jj], sn[jj] = (1.0, 0.0) if rho == 0 else (H[jj, jj] / rho, H[jj + 1, jj] / rho)
                H[jj, jj] = rho
                H[jj + 1, jj] = 0.0
                g[jj + 1] = -sn[jj] * g[jj]
                g[jj] = cs[jj] * g[jj]
                cols = jj + 1
                if abs(g[jj + 1]) <= tol or it >= maxiter or not hnext > 0:
                    stop = True
                    break
            y = np.linalg.solve(np.triu(H[:cols, :cols]), g[:cols]) if cols else np.zeros(0)
            for q in range(cols):
                x = x + y[q] * Zb[q]
            if stop:
                return x, it
            r = rhs - matvec(x)
            beta = np.linalg.norm(r)
            if beta <= tol:
                return x, it

    def step(self, n, n_steps, maxiter=100, tol=1e-4, tol_relative=False, scale=1.0,
             rule="central", gmres_maxiter=200, gmres_reltol=1e-4, gmres_abstol=1e-8,
             restart=100, precond="none", D=None):
        """newton_krylov_step!; returns (converged, newton iterations, gmres iterations,
        first and last residual norms)."""
        self.apply_conditions(n / n_steps)
        first = None
        gm = 0
        for it in range(1, maxiter + 1):
            r = self.residual()
            Fu = self.ob.b_int.reshape(-1) * np.repeat(self.V, 3)
            rn = float(np.linalg.norm(r))
            first = rn if first is None else first
            conv = rn <= tol * first if tol_relative else rn < tol
            if conv:
                return True, it, gm, first, rn
            if it == maxiter:
                return False, it, gm, first, rn
            P = None if precond == "none" else self.bj_blocks()
            mv = lambda v: self.jv(v, rule, scale, Fu if rule == "forward" else None)
            pc = lambda v: self.precond(precond, v, P, D)
            du, k = self.gmres(-r, mv, pc, gmres_maxiter, gmres_reltol, gmres_abstol, restart)
            gm += k
            # update_displacement_from_du! on the free dofs
            free = ~self.cmask
            u = self.ob.u.reshape(-1)
            pos = self.ob.pos.reshape(-1)
            u[free] += du[free]
            pos[free] += du[free]
        return False, maxiter, gm, first, rn
