"""The oracle twin of a pdcuda Body (test infrastructure only).

``oracle_body(body)`` builds the FP64 CPU oracle of ``oracle.py`` on the same positions,
volumes, parameter sets, failure permissions, pre-cracks, initial conditions and surface
correction as a ``pdcuda.Body``; ``oracle_bcs`` tabulates the body's boundary conditions for
the oracle's Velocity Verlet run. Only the tests, ``__graft_entry__.smoke()`` and the CPU
baseline / reference legs of ``bench.py`` use it, as the checker.
"""
import numpy as np

import oracle as O
import pdcuda as pd

MAT_ORACLE = {pd.BBMaterial: O.BB, pd.OSBMaterial: O.OSB, pd.CMaterial: O.CMAT}


def oracle_params(p):
    return O.Params(p.delta, p.rho, p.E, p.nu, p.G, p.K, p.lambda_, p.mu, p.Gc, p.epsilon_c, p.bc)


def oracle_body(body, cmodel=None):
    """The oracle twin of a pdcuda Body (same positions, parameters, permissions, cracks)."""
    mat = body.mat
    params = [oracle_params(p) for p in body.point_params]
    cracks = [(np.isin(np.arange(body.n_points), body.point_sets[a]).astype(np.uint8),
               np.isin(np.arange(body.n_points), body.point_sets[b]).astype(np.uint8))
              for a, b, filt in body.point_sets_precracks if filt]
    kernel = {pd.const_one_kernel: O.KERNEL_CONST_ONE, pd.linear_kernel: O.KERNEL_LINEAR,
              pd.cubic_b_spline_kernel: O.KERNEL_CUBIC_BSPLINE}[mat.kernel]
    cm = 0
    if isinstance(mat, pd.CMaterial):
        cm = {pd.SaintVenantKirchhoff: O.SVK, pd.NeoHooke: O.NEOHOOKE,
              pd.NeoHookePenalty: O.NHPENALTY}[type(mat.model)]
    ob = O.OracleBody(MAT_ORACLE[type(mat)], body._pos, body.volume, params,
                      pid=body.params_map - 1, kernel=kernel, cmodel=cm,
                      zem_cs=getattr(getattr(mat, "zem", None), "Cs", 0.5), maxdmg=mat.maxdmg,
                      fp_point=body.fail_permit.astype(np.uint8), cracks=cracks,
                      zem=O.ZEM_WAN if isinstance(getattr(mat, "zem", None), pd.ZEMWan) else O.ZEM_SILLING)
    for a, b, filt in body.point_sets_precracks:
        if not filt:
            ob.break_bonds(body.point_sets[a], body.point_sets[b])
            ob.calc_damage()
    if isinstance(getattr(mat, "correction", None), pd.EnergySurfaceCorrection):
        ob.init_surface_correction()   # initialize! after the pre-cracks
    for ic in body.single_dim_ics:
        ob.v[body.point_sets[ic.point_set], ic.dim] = ic.fun
    for ic in body.posdep_single_dim_ics:
        for i in body.point_sets[ic.point_set]:
            val = float(ic.fun(body._pos[i]))
            if not np.isnan(val):
                ob.v[i, ic.dim] = val
    return ob


def oracle_bcs(body, first, n, dt):
    """The boundary conditions of a body tabulated for the oracle's run_vv."""
    out = []
    for c in body.single_dim_bcs:
        pts = body.point_sets[c.point_set]
        vals = np.array([float(c.fun(s * dt)) for s in range(first, first + n)])
        out.append(dict(field=0 if c.field == "velocity_half" else 1, dim=c.dim, kind=0, pts=pts,
                        values=vals, first_step=first))
    for c in body.posdep_single_dim_bcs:
        pts = body.point_sets[c.point_set]
        vals = np.array([[float(c.fun(body._pos[i], s * dt)) for i in pts]
                         for s in range(first, first + n)]).ravel()
        out.append(dict(field=0 if c.field == "velocity_half" else 1, dim=c.dim, kind=1, pts=pts,
                        values=vals, first_step=first))
    for c in body.data_bcs:
        pts = body.point_sets[c.point_set]
        for row, d in enumerate(c.dim):
            out.append(dict(field=0 if c.field == "velocity_half" else 1, dim=d, kind=2, pts=pts,
                            values=c.data[row, pts], first_step=first))
    return out
