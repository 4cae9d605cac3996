"""VelocityVerlet, Job, submit and the device-resident body.

``DeviceBody`` plays the role of the reference's data handler for one chunk holding every
point (src/core/threads_body_data_handler.jl:31-212): it builds the bond system on the
device, applies pre-cracks and initial conditions, tabulates the boundary-condition
functions on the host and drives the C ABI. ``submit`` follows src/core/submit.jl:14-29 and
src/time_solvers/velocity_verlet.jl:103-179.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib as L
from .body import Body
from .materials import CMaterial, EnergySurfaceCorrection

_FIELDS = {
    "position": (L.F_POSITION, 3, np.float64), "displacement": (L.F_DISPLACEMENT, 3, np.float64),
    "velocity": (L.F_VELOCITY, 3, np.float64), "velocity_half": (L.F_VELOCITY_HALF, 3, np.float64),
    "acceleration": (L.F_ACCELERATION, 3, np.float64), "b_int": (L.F_B_INT, 3, np.float64),
    "b_ext": (L.F_B_EXT, 3, np.float64), "damage": (L.F_DAMAGE, 1, np.float64),
    "n_active_bonds": (L.F_N_ACTIVE_BONDS, 1, np.int64),
    "bond_active": (L.F_BOND_ACTIVE, 0, np.uint8),
    "defgrad": (L.F_DEFGRAD, 9, np.float64), "cauchy_stress": (L.F_CAUCHY_STRESS, 9, np.float64),
    "n_neighbors": (L.F_N_NEIGHBORS, 1, np.int64),
}
_PREC = {"fp64": L.PREC_FP64, "fp32": L.PREC_FP32_KAHAN}


class VelocityVerlet:
    """Velocity Verlet time integration (velocity_verlet.jl:47-71)."""

    def __init__(self, time=-1.0, steps=-1, stepsize=-1.0, safety_factor=0.7):
        if time > 0 and steps > 0:
            raise ValueError("specify either time or number of steps, not both!")
        if time < 0 and steps < 0:
            raise ValueError("specify either time or number of steps!")
        if not (0 < safety_factor < 1):
            raise ValueError("wrong safety factor specified! condition: 0 < safety_factor < 1")
        self.end_time = float(time)
        self.n_steps = int(steps)
        self.dt = float(stepsize)
        self.safety_factor = float(safety_factor)

    def init(self, stable_dt):
        """init_time_solver! (velocity_verlet.jl:103-130)."""
        if self.dt < 0:
            self.dt = stable_dt
        if self.end_time < 0:
            self.end_time = self.n_steps * self.dt
        elif self.n_steps < 0:
            self.n_steps = int(self.end_time // self.dt) + 1
        if self.end_time < 0 or self.n_steps < 0 or self.dt < 0:
            raise RuntimeError("invalid VelocityVerlet state")

    def __repr__(self):
        return f"VelocityVerlet(n_steps={self.n_steps}, dt={self.dt}, safety_factor={self.safety_factor})"


class Job:
    """A simulation job (src/core/job.jl:45-62). With a ``path`` the fields are written as VTK
    files in the reference's layout (``pdcuda.vtk``: `<path>/vtk/timestep_<n>.pvtu` at step 0
    and every ``freq`` steps); ``export`` (a callable export(step, t, sim)) replaces the writer."""

    def __init__(self, body, solver, path="", freq=10, fields=None, export=None,
                 precision="fp64", graph_steps=0, mapping=None, device=0):
        if freq < 0:
            raise ValueError("`freq` should be larger than zero!")
        self.body, self.solver = body, solver
        self.path, self.freq, self.fields = path, int(freq), fields
        if export is None and path:
            from .vtk import VtkExport
            export = VtkExport(path, freq, fields)
        self.export = export
        self.precision, self.graph_steps, self.mapping, self.device = precision, graph_steps, mapping, device


class DeviceBody:
    """One body (all points in one chunk) resident on a CUDA device."""

    def __init__(self, body: Body, precision="fp64", device=0, param_dt=None,
                 independent_params=False, owned=None):
        if precision not in _PREC:
            raise ValueError("precision must be 'fp64' or 'fp32'")
        if np.any(body.params_map == 0):
            raise ValueError("not all points have material parameters: use material!")
        self.body = body
        self.precision = precision
        self.n = body.n_points
        self.h = C.c_void_p()
        lib = L.lib()
        params = (L.PointParams * len(body.point_params))(*[p.to_c() for p in body.point_params])
        self._params = params
        pid = (body.params_map - 1).astype(np.uint16)
        self._pid = pid
        mat = body.mat
        desc = L.BodyDesc()
        desc.n_points = self.n
        desc.position = L.ptr(body._pos)
        desc.volume = L.ptr(body.volume)
        desc.param_id = L.ptr(pid)
        desc.n_params = len(body.point_params)
        desc.params = C.cast(params, C.c_void_p)
        desc.material = mat.material_id
        desc.kernel = mat.kernel_id
        desc.cmodel = mat.model.id if isinstance(mat, CMaterial) else 0
        desc.precision = _PREC[precision]
        # several parameter sets: the reference's ParameterHandler semantics (bond-averaged
        # parameters), unless every bonded pair shares its set (independent specimens)
        desc.multi_params = 1 if (len(body.point_params) > 1 and not independent_params) else 0
        desc.zem_cs = getattr(mat.zem, "Cs", 0.5) if isinstance(mat, CMaterial) else 0.5
        desc.zem = mat.zem.id if isinstance(mat, CMaterial) else L.ZEM_SILLING
        desc.maxdmg = mat.maxdmg
        desc.device = device
        filt = [c for c in body.point_sets_precracks if c[2]]
        nf = len(filt)
        fa = np.zeros((max(nf, 1), self.n), np.uint8)
        fb = np.zeros((max(nf, 1), self.n), np.uint8)
        for k, (a, b, _) in enumerate(filt):
            fa[k, body.point_sets[a]] = 1
            fb[k, body.point_sets[b]] = 1
        fp = body.fail_permit.astype(np.uint8)
        spos = getattr(body, "_search_pos", None)
        if owned is None:
            L.check(lib.pd_create_search(C.byref(desc), L.ptr(spos), L.ptr(fp), nf, L.ptr(fa),
                                         L.ptr(fb), C.byref(self.h)), "pd_create_search")
        else:  # a partition: owned rows and halo rows (pdcuda.halo)
            own = np.ascontiguousarray(owned, np.uint8)
            L.check(lib.pd_create_partition(C.byref(desc), L.ptr(spos), L.ptr(fp), nf, L.ptr(fa),
                                            L.ptr(fb), L.ptr(own), C.byref(self.h)),
                    "pd_create_partition")
        self.n_bonds = self.info()[1]
        # apply_precracks! (predefined_cracks.jl:31-60): damage-mode cracks break bonds
        for a, b, filt_mode in body.point_sets_precracks:
            if filt_mode:
                continue
            ma = np.zeros(self.n, np.uint8)
            mb = np.zeros(self.n, np.uint8)
            ma[body.point_sets[a]] = 1
            mb[body.point_sets[b]] = 1
            L.check(lib.pd_break_bonds(self.h, L.ptr(ma), L.ptr(mb)), "pd_break_bonds")
        # apply_initial_conditions! (initial_conditions.jl:86-94)
        if body.single_dim_ics or body.posdep_single_dim_ics:
            v = np.zeros((self.n, 3))
            for ic in body.single_dim_ics:
                v[body.point_sets[ic.point_set], ic.dim] = ic.fun
            for ic in body.posdep_single_dim_ics:
                for i in body.point_sets[ic.point_set]:
                    val = float(ic.fun(body._pos[i]))
                    if not math.isnan(val):
                        v[i, ic.dim] = val
            self.set_state(velocity=v)
        # initialize! of EnergySurfaceCorrection (bond_system_corrections.jl:78-94) after the
        # pre-cracks; a partition computes it with its neighbours (pdcuda.halo)
        self.esc = isinstance(getattr(mat, "correction", None), EnergySurfaceCorrection)
        if self.esc and owned is None:
            L.check(lib.pd_esc_init(self.h, 0), "pd_esc_init")
        self._setup_bcs()
        self.param_dt = param_dt

    # -- conditions -------------------------------------------------------------------------
    def _setup_bcs(self):
        body = self.body
        self._bcs = []   # (kind, fun, points, dt-source)
        descs = []
        keep = []
        field_id = {"velocity_half": L.BC_VELOCITY_HALF, "b_ext": L.BC_B_EXT}
        for c in body.single_dim_bcs:
            pts = np.ascontiguousarray(body.point_sets[c.point_set], np.int32)
            keep.append(pts)
            descs.append(L.BCDesc(field_id[c.field], c.dim, L.BC_KIND_TIME, len(pts), L.ptr(pts), None))
            self._bcs.append(("time", c.fun, pts))
        for c in body.posdep_single_dim_bcs:
            pts = np.ascontiguousarray(body.point_sets[c.point_set], np.int32)
            keep.append(pts)
            descs.append(L.BCDesc(field_id[c.field], c.dim, L.BC_KIND_POINT_TIME, len(pts), L.ptr(pts), None))
            self._bcs.append(("point_time", c.fun, pts))
        for c in body.data_bcs:
            pts = np.ascontiguousarray(body.point_sets[c.point_set], np.int32)
            for row, d in enumerate(c.dim):
                vals = np.ascontiguousarray(c.data[row, pts], np.float64)
                keep += [pts, vals]
                descs.append(L.BCDesc(field_id[c.field], d, L.BC_KIND_DATA, len(pts), L.ptr(pts), L.ptr(vals)))
        arr = (L.BCDesc * max(len(descs), 1))(*descs)
        L.check(L.lib().pd_set_bcs(self.h, len(descs), C.cast(arr, C.c_void_p)), "pd_set_bcs")
        self.per_step = sum(1 if k == "time" else len(p) for k, _, p in self._bcs)

    def _point_dt(self, points, dt):
        if dt > 0:
            return np.full(len(points), dt)
        return self.param_dt[self._pid[points]]

    def tabulate_bcs(self, first_step, n_steps, dt):
        """Values of the time-dependent conditions at t = step * dt (apply_bc!,
        boundary_conditions.jl:37-51, 91-108) for the next n_steps steps."""
        if not self._bcs or n_steps <= 0:
            return
        vals = np.empty((n_steps, self.per_step))
        steps = np.arange(first_step, first_step + n_steps, dtype=np.float64)
        col = 0
        for kind, f, pts in self._bcs:
            dts = self._point_dt(pts[:1], dt)[0] if len(pts) else max(dt, 0.0)
            if kind == "time":
                vals[:, col] = [float(f(s * dts)) for s in steps]
                col += 1
            else:
                pos = self.body._pos[pts]
                for r, s in enumerate(steps):
                    t = s * dts
                    vals[r, col:col + len(pts)] = [float(f(pos[q], t)) for q in range(len(pts))]
                col += len(pts)
        vals = np.ascontiguousarray(vals)
        L.check(L.lib().pd_set_bc_values(self.h, first_step, n_steps, L.ptr(vals), vals.size),
                "pd_set_bc_values")

    # -- state -------------------------------------------------------------------------------
    def set_state(self, position=None, displacement=None, velocity=None, velocity_half=None,
                  acceleration=None, b_ext=None, bond_active=None):
        """Point fields as 3 x N (or N x 3) arrays; bond_active one byte per bond."""
        def pv(a):
            if a is None:
                return None
            a = np.asarray(a, np.float64)
            if a.shape == (3, self.n) and self.n != 3:
                a = a.T
            return np.ascontiguousarray(a.reshape(self.n, 3))
        args = [pv(a) for a in (position, displacement, velocity, velocity_half, acceleration, b_ext)]
        ba = None if bond_active is None else np.ascontiguousarray(bond_active, np.uint8)
        self._keep = args + [ba]
        L.check(L.lib().pd_set_state(self.h, *[L.ptr(a) for a in args], L.ptr(ba)), "pd_set_state")

    def field(self, name, out=None):
        """A storage field: point vectors / tensors as 3 x N / 9 x N views (the reference's
        layout), scalars as N, bond_active as n_bonds bytes. out: a C-contiguous array of the
        field's size and type to read into (pinned host memory makes the copy faster)."""
        fid, comp, dt = _FIELDS[name]
        shape = (self.n_bonds,) if comp == 0 else (self.n,) if comp == 1 else (self.n, comp)
        if out is None:
            out = np.empty(shape, dt)
        elif out.dtype != dt or out.size != int(np.prod(shape)) or not out.flags.c_contiguous:
            raise ValueError(f"out must be a C-contiguous {np.dtype(dt).name} array of {np.prod(shape)} elements")
        out = out.reshape(shape)
        L.check(L.lib().pd_get_field(self.h, fid, L.ptr(out), out.nbytes), f"pd_get_field({name})")
        return out.T if comp > 1 else out

    def info(self):
        n, nb, sym = C.c_int64(), C.c_int64(), C.c_int32()
        L.check(L.lib().pd_info(self.h, C.byref(n), C.byref(nb), C.byref(sym)))
        return n.value, nb.value, sym.value

    # -- solver entry points ----------------------------------------------------------------
    def stable_timestep(self, safety_factor=0.7, per_param=False):
        dt = C.c_double()
        arr = np.empty(len(self.body.point_params))
        L.check(L.lib().pd_stable_timestep(self.h, safety_factor, C.byref(dt), L.ptr(arr)),
                "pd_stable_timestep")
        return (dt.value, arr) if per_param else dt.value

    def set_param_timesteps(self, dts):
        dts = np.ascontiguousarray(dts, np.float64)
        self.param_dt = dts
        L.check(L.lib().pd_set_param_timesteps(self.h, L.ptr(dts)), "pd_set_param_timesteps")

    def force(self, t=0.0, dt=0.0):
        """calc_force_density!(chunk, t, dt) with the NaN check."""
        st = L.lib().pd_force(self.h, t, dt)
        self._raise(st, t, dt)

    def run(self, first_step, n_steps, dt):
        """n_steps Velocity Verlet steps starting at step number first_step."""
        self.tabulate_bcs(first_step, n_steps, dt)
        st = L.lib().pd_run_vv(self.h, first_step, n_steps, dt)
        self._raise(st, None, dt)

    def run_timed(self, first_step, n_steps, dt, phases=True):
        """run() with CUDA events around every kernel: (total, phase A, phase B, integrate) ms.
        phases=False: the steps as run() issues them (CUDA graphs when set_graph is on), timed
        as a whole; returns the total ms."""
        self.tabulate_bcs(first_step, n_steps, dt)
        out = [C.c_double() for _ in range(4)]
        if not phases:
            st = L.lib().pd_run_vv_timed(self.h, first_step, n_steps, dt, C.byref(out[0]),
                                         None, None, None)
            self._raise(st, None, dt)
            return out[0].value
        st = L.lib().pd_run_vv_timed(self.h, first_step, n_steps, dt, *[C.byref(o) for o in out])
        self._raise(st, None, dt)
        return tuple(o.value for o in out)

    def _raise(self, st, t, dt):
        if st == L.PD_ERR_NAN:
            step = C.c_int64()
            L.lib().pd_nan_step(self.h, C.byref(step))
            tt = t if t is not None else step.value * (dt if dt and dt > 0 else float("nan"))
            raise L.NaNError(tt, step.value)
        L.check(st)

    def set_mapping(self, group, block=256):
        L.check(L.lib().pd_set_mapping(self.h, group, block), "pd_set_mapping")

    def set_pipeline(self, pipe):
        L.check(L.lib().pd_set_pipeline(self.h, pipe), "pd_set_pipeline")

    def mapping(self):
        """(lanes per point, block size, bond-stream variant); 0 lanes = serial order."""
        g, b, p = C.c_int32(), C.c_int32(), C.c_int32()
        L.check(L.lib().pd_get_mapping(self.h, C.byref(g), C.byref(b), C.byref(p)), "pd_get_mapping")
        return g.value, b.value, p.value

    def autotune(self):
        g, b = C.c_int32(), C.c_int32()
        L.check(L.lib().pd_autotune(self.h, C.byref(g), C.byref(b)), "pd_autotune")
        return g.value, b.value

    def set_graph(self, steps):
        L.check(L.lib().pd_set_graph(self.h, steps), "pd_set_graph")

    def launch_count(self):
        c = C.c_int64()
        L.check(L.lib().pd_launch_count(self.h, C.byref(c)))
        return c.value

    def near_critical(self, tol=1e-12):
        """Bonds that may fail with |eps - eps_c| <= tol at the current state."""
        c = C.c_int64()
        L.check(L.lib().pd_count_near_critical(self.h, float(tol), C.byref(c)), "pd_count_near_critical")
        return c.value

    def surface_correction(self):
        """(mfactor (n, 3), scfactor (n_bonds, CSR order)) of EnergySurfaceCorrection."""
        mf = np.empty((self.n, 3))
        sc = np.empty(self.info()[1])
        L.check(L.lib().pd_esc_get(self.h, L.ptr(mf), L.ptr(sc)), "pd_esc_get")
        return mf, sc

    def break_random_pairs(self, fraction, seed):
        L.check(L.lib().pd_break_random_pairs(self.h, float(fraction), int(seed)), "pd_break_random_pairs")

    def close(self):
        if self.h:
            L.lib().pd_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def check_conditions_applicable(body, solver):
    """check_conditions_applicable (discretization/body.jl:287-302): displacement conditions
    are applied only by the Newton-Krylov solver."""
    if body.pos_single_dim_bcs:
        raise ValueError(
            "conditions of this body cannot be applied by the specified time solver!\n"
            f"The body has {len(body.pos_single_dim_bcs)} prescribed displacement condition(s) "
            "defined with\n`displacement_bc!`. These are only applied by the `NewtonKrylov` "
            f"solver, but the job uses\na `{type(solver).__name__}` solver, which would ignore "
            "them completely.\nUse a `NewtonKrylov` solver, or specify the load with "
            "`velocity_bc!` or\n`forcedensity_bc!` instead.\n")


def submit(job: Job, quiet=True):
    """submit (core/submit.jl:14-29) on the device: builds the device body, computes the CFL
    step (velocity_verlet.jl:103-163), runs initialize! (a force evaluation at t = 0) and
    solve! (velocity_verlet.jl:165-179). Returns the DeviceBody with the final state."""
    from .newton_krylov import NewtonKrylov, solve as nk_solve
    if isinstance(job.solver, NewtonKrylov):
        dev = DeviceBody(job.body, precision=job.precision, device=job.device)
        if job.mapping is not None:
            dev.set_mapping(*job.mapping)
        return nk_solve(dev, job.solver, job.export, job.freq if job.export is not None else 0)
    from .dynamic_relaxation import DynamicRelaxation, solve as dr_solve
    check_conditions_applicable(job.body, job.solver)
    if isinstance(job.solver, DynamicRelaxation):
        dev = DeviceBody(job.body, precision=job.precision, device=job.device)
        if job.mapping is not None:
            dev.set_mapping(*job.mapping)
        return dr_solve(dev, job.solver, job.export, job.freq if job.export is not None else 0)
    vv = job.solver
    dev = DeviceBody(job.body, precision=job.precision, device=job.device)
    if job.mapping is not None:
        dev.set_mapping(*job.mapping)
    if job.graph_steps:
        dev.set_graph(job.graph_steps)
    vv.init(dev.stable_timestep(vv.safety_factor) if vv.dt < 0 else vv.dt)
    dt = vv.dt
    dev.force(0.0, dt)
    if job.export is not None:
        job.export(0, 0.0, dev)
    freq = job.freq if (job.export is not None and job.freq > 0) else vv.n_steps
    n = 1
    while n <= vv.n_steps:
        k = min(freq, vv.n_steps - n + 1)
        dev.run(n, k, dt)
        n += k
        if job.export is not None and ((n - 1) % job.freq == 0 or n > vv.n_steps):
            job.export(n - 1, (n - 1) * dt, dev)
    return dev
