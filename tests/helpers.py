"""Shared builders of the tests: the same bodies for the oracle and the device."""
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
                      fp_point=body.fail_permit.astype(np.uint8), cracks=cracks)
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


def cube_body(mat, n=6, m=3.015, E=210e9, nu=0.25, rho=7850.0, Gc=2.7, fracture=False, **kw):
    """The reference's `cube` fixture (test/setup/fixtures.jl:50-58): unit cube of n^3 points."""
    dx = 1.0 / n
    pos, vol = pd.uniform_box(1.0, 1.0, 1.0, dx)
    body = pd.Body(mat, pos, vol)
    args = dict(horizon=m * dx, rho=rho, E=E, Gc=Gc)
    if not isinstance(mat, pd.BBMaterial):
        args["nu"] = nu
    args.update(kw)
    pd.material(body, **args)
    if not fracture:
        pd.no_failure(body)
    return body


def deform(X, F=((1.01, 0.003, 0.0), (0.0, 0.995, 0.0), (0.0, 0.0, 1.0)), amplitude=1e-4):
    """Inhomogeneous deformation of the reference's deform! fixture (fixtures.jl:123-141):
    returns the displacement (n, 3)."""
    F = np.asarray(F)
    x = X @ F.T
    x[:, 0] += amplitude * np.sin(np.pi * 3 * X[:, 1])
    x[:, 1] += amplitude * np.sin(np.pi * 3 * X[:, 2])
    x[:, 2] += amplitude * np.sin(np.pi * 3 * X[:, 0])
    return x - X


def plate_body(mat, nx=40, ny=20, nz=4, dx=2.5e-3, E=70e9, rho=2700.0, Gc=100.0, v=0.6, nu=None):
    """Mode-I tensile plate: bonds crossing x = 0.5 lx for y < 0.2 ly are filtered, the top
    and bottom two rows are pulled at +-v in y."""
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
