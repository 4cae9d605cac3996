"""ctypes binding of the FP64 CPU oracle (test infrastructure only).

The oracle restates Peridynamics.jl's explicit-dynamics hot path in C (``pd_oracle.c``).
Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU baseline / reference
leg import this module, and only as the checker: the product never calls it.

Array layout: positions and every point vector are ``(n, 3)`` float64 C-contiguous, which
is the memory layout of the reference's ``3 x N`` column-major matrices.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

BB, OSB, CMAT = 0, 1, 2
SVK, NEOHOOKE, NHPENALTY = 0, 1, 2
KERNEL_CONST_ONE, KERNEL_LINEAR, KERNEL_CUBIC_BSPLINE = 0, 1, 2
ZEM_SILLING, ZEM_WAN = 0, 1


class Params(C.Structure):
    _fields_ = [(k, C.c_double) for k in
                ("delta", "rho", "E", "nu", "G", "K", "lambda_", "mu", "Gc", "epsc", "bc")]


class Sys(C.Structure):
    _fields_ = [("n", C.c_int64), ("n_bonds", C.c_int64),
                ("X", C.c_void_p), ("vol", C.c_void_p), ("off", C.c_void_p),
                ("nbr", C.c_void_p), ("L", C.c_void_p), ("fail_permit", C.c_void_p),
                ("omega", C.c_void_p), ("pid", C.c_void_p), ("params", C.c_void_p),
                ("n_params", C.c_int32), ("material", C.c_int32), ("cmodel", C.c_int32),
                ("multi", C.c_int32), ("zem_cs", C.c_double), ("maxdmg", C.c_double),
                ("scfactor", C.c_void_p), ("zem", C.c_int32)]


class State(C.Structure):
    _fields_ = [(k, C.c_void_p) for k in
                ("pos", "u", "v", "vh", "a", "b_int", "b_ext", "damage", "n_active",
                 "bond_active", "bond_length", "defgrad", "cauchy")]


class BC(C.Structure):
    _fields_ = [("field", C.c_int32), ("dim", C.c_int32), ("kind", C.c_int32),
                ("n_pts", C.c_int32), ("pts", C.c_void_p), ("values", C.c_void_p),
                ("first_step", C.c_int64)]


def build():
    """Compile liboracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        vp, i64, i32, dbl = C.c_void_p, C.c_int64, C.c_int32, C.c_double
        L.or_find_bonds.restype = i64
        L.or_find_bonds.argtypes = [i64, vp, vp, vp, vp, vp, i32, i64, vp, vp, vp, vp]
        L.or_kernels.argtypes = [vp, i32, vp]
        L.or_init_state.argtypes = [vp, vp]
        L.or_break_bonds.argtypes = [vp, vp, vp, vp]
        L.or_calc_damage.argtypes = [vp, vp]
        L.or_force_density.argtypes = [vp, vp, dbl, dbl]
        L.or_contains_nan.restype = C.c_int
        L.or_contains_nan.argtypes = [vp, vp]
        L.or_stable_timestep.restype = dbl
        L.or_stable_timestep.argtypes = [vp, dbl]
        L.or_run_vv.restype = i64
        L.or_run_vv.argtypes = [vp, vp, vp, i32, i64, i64, dbl]
        L.or_first_piola_kirchhoff.argtypes = [i32, vp, vp, vp]
        L.or_inv3.argtypes = [vp, vp]
        L.or_zem_wan_stiffness.argtypes = [vp, vp, vp]
        L.or_det3.restype = dbl
        L.or_det3.argtypes = [vp]
        L.or_point_params.restype = C.c_int
        L.or_point_params.argtypes = [i32] + [dbl] * 10 + [vp, C.c_char_p, i32]
        L.or_set_threads.argtypes = [i32]
        L.or_set_serial_order.argtypes = [i32]
        L.or_esc_mfactor.argtypes = [vp, vp, vp]
        L.or_esc_scfactor.argtypes = [vp, vp, vp]
        L.or_esc_lame.argtypes = [vp, vp, i64, vp]
        _LIB = L
    return _LIB


def _p(a):
    return None if a is None else a.ctypes.data


def zem_wan_stiffness(params, Kinv):
    """ZEMWan's C_1 = C : K^-1 (zem_stabilization.jl:32-42) for one parameter set and one
    3x3 inverse shape tensor."""
    k = np.asfortranarray(Kinv, dtype=np.float64)
    out = np.zeros((3, 3), np.float64, order="F")
    lib().or_zem_wan_stiffness(C.byref(params), k.ctypes.data, out.ctypes.data)
    return out


def point_params(material, horizon, rho, E=np.nan, nu=np.nan, G=np.nan, K=np.nan,
                 lambda_=np.nan, mu=np.nan, Gc=np.nan, epsilon_c=np.nan):
    out = Params()
    msg = C.create_string_buffer(256)
    rc = lib().or_point_params(material, horizon, rho, E, nu, G, K, lambda_, mu, Gc,
                               epsilon_c, C.byref(out), msg, 256)
    if rc != 0:
        raise ValueError(msg.value.decode())
    return out


def find_bonds(X, delta, fp_point=None, cracks=()):
    """Bond lists in CSR form: (off, nbr, L, fail_permit). ``cracks`` are (mask_a, mask_b)
    pairs of filter-mode pre-cracks."""
    X = np.ascontiguousarray(X, dtype=np.float64)
    n = X.shape[0]
    delta = np.ascontiguousarray(np.broadcast_to(np.asarray(delta, np.float64), (n,)))
    fp = np.ones(n, np.uint8) if fp_point is None else np.ascontiguousarray(fp_point, np.uint8)
    nc = len(cracks)
    ca = np.zeros((max(nc, 1), n), np.uint8)
    cb = np.zeros((max(nc, 1), n), np.uint8)
    for k, (a, b) in enumerate(cracks):
        ca[k] = a
        cb[k] = b
    L_ = lib()
    total = L_.or_find_bonds(n, _p(X), _p(delta), _p(fp), _p(ca), _p(cb), nc, 0, None, None,
                             None, None)
    if total < 0:
        raise ValueError("point duplicate found")
    off = np.zeros(n + 1, np.int64)
    nbr = np.zeros(max(total, 1), np.int32)
    Lb = np.zeros(max(total, 1), np.float64)
    fpb = np.zeros(max(total, 1), np.uint8)
    L_.or_find_bonds(n, _p(X), _p(delta), _p(fp), _p(ca), _p(cb), nc, total, _p(off), _p(nbr),
                     _p(Lb), _p(fpb))
    return off, nbr[:total], Lb[:total], fpb[:total]


class OracleBody:
    """One body (one chunk) of the FP64 oracle with its storage fields."""

    def __init__(self, material, X, vol, params, pid=None, off=None, nbr=None, L=None,
                 fail_permit=None, kernel=KERNEL_LINEAR, cmodel=SVK, multi=None,
                 zem_cs=0.5, maxdmg=0.85, fp_point=None, cracks=(), zem=0):
        self.X = np.ascontiguousarray(X, dtype=np.float64).reshape(-1, 3)
        n = self.X.shape[0]
        self.n = n
        self.vol = np.ascontiguousarray(vol, dtype=np.float64)
        if isinstance(params, Params):
            params = [params]
        self.params_list = list(params)
        self.params = (Params * len(params))(*params)
        self.pid = (np.zeros(n, np.int32) if pid is None
                    else np.ascontiguousarray(pid, dtype=np.int32))
        if off is None:
            delta = np.array([params[k].delta for k in self.pid], np.float64)
            off, nbr, L, fail_permit = find_bonds(self.X, delta, fp_point, cracks)
        self.off = np.ascontiguousarray(off, np.int64)
        self.nbr = np.ascontiguousarray(nbr, np.int32)
        self.L = np.ascontiguousarray(L, np.float64)
        self.fail_permit = np.ascontiguousarray(fail_permit, np.uint8)
        B = int(self.off[-1])
        self.n_bonds = B
        self.material = material
        self.omega = np.zeros(max(B, 1), np.float64)
        if multi is None:
            multi = 1 if len(params) > 1 else 0
        self.sys = Sys(n, B, _p(self.X), _p(self.vol), _p(self.off), _p(self.nbr), _p(self.L),
                       _p(self.fail_permit), _p(self.omega), _p(self.pid),
                       C.cast(self.params, C.c_void_p), len(params), material, cmodel, multi,
                       zem_cs, maxdmg, None, int(zem))
        lib().or_kernels(C.byref(self.sys), kernel, _p(self.omega))
        z3 = lambda: np.zeros((n, 3), np.float64)
        self.pos, self.u, self.v, self.vh, self.a, self.b_int, self.b_ext = (z3() for _ in range(7))
        self.damage = np.zeros(n, np.float64)
        self.n_active = np.zeros(n, np.int64)
        self.bond_active = np.ones(max(B, 1), np.uint8)
        self.bond_length = np.zeros(max(B, 1), np.float64)
        self.defgrad = np.zeros((n, 9), np.float64)
        self.cauchy = np.zeros((n, 9), np.float64)
        self.st = State(*[_p(a) for a in (self.pos, self.u, self.v, self.vh, self.a, self.b_int,
                                            self.b_ext, self.damage, self.n_active,
                                            self.bond_active, self.bond_length, self.defgrad,
                                            self.cauchy)])
        lib().or_init_state(C.byref(self.sys), C.byref(self.st))

    @property
    def n_neighbors(self):
        return np.diff(self.off)

    def break_bonds(self, set_a, set_b):
        a = np.zeros(self.n, np.uint8)
        b = np.zeros(self.n, np.uint8)
        a[np.asarray(set_a, np.int64)] = 1
        b[np.asarray(set_b, np.int64)] = 1
        lib().or_break_bonds(C.byref(self.sys), C.byref(self.st), _p(a), _p(b))

    def init_surface_correction(self):
        """EnergySurfaceCorrection (bond_system_corrections.jl:78-124, 156-204) from the
        current bond states: mfactor (n, 3) and scfactor (n_bonds), then used by the force."""
        self.mfactor = np.zeros((self.n, 3), np.float64)
        self.scfactor = np.ones(max(self.n_bonds, 1), np.float64)
        lib().or_esc_mfactor(C.byref(self.sys), C.byref(self.st), _p(self.mfactor))
        lib().or_esc_scfactor(C.byref(self.sys), _p(self.mfactor), _p(self.scfactor))
        self.sys.scfactor = _p(self.scfactor)

    def esc_lame(self, i):
        """get_averaged_lame_parameters of point i: (lambda, mu)."""
        out = np.zeros(2)
        lib().or_esc_lame(C.byref(self.sys), C.byref(self.st), int(i), _p(out))
        return out

    def calc_damage(self):
        lib().or_calc_damage(C.byref(self.sys), C.byref(self.st))

    def force_density(self, t=0.0, dt=0.0):
        lib().or_force_density(C.byref(self.sys), C.byref(self.st), t, dt)

    def stable_timestep(self, safety_factor=0.7):
        return lib().or_stable_timestep(C.byref(self.sys), safety_factor)

    def run_vv(self, first_step, n_steps, dt, bcs=()):
        """bcs: list of dicts(field, dim, kind, pts, values, first_step)."""
        keep = []
        arr = (BC * max(len(bcs), 1))()
        for k, bc in enumerate(bcs):
            pts = np.ascontiguousarray(bc["pts"], np.int32)
            vals = np.ascontiguousarray(bc["values"], np.float64)
            keep += [pts, vals]
            arr[k] = BC(bc["field"], bc["dim"], bc["kind"], len(pts), _p(pts), _p(vals),
                        bc.get("first_step", first_step))
        return lib().or_run_vv(C.byref(self.sys), C.byref(self.st), C.cast(arr, C.c_void_p),
                               len(bcs), first_step, n_steps, dt)


def set_threads(n):
    lib().or_set_threads(int(n))


def set_serial_order(on):
    """True: the state-based force loops keep the serial loop's summation order on any thread
    count (bit for bit the one-thread result); False: the threads backend's chunked scatter."""
    lib().or_set_serial_order(1 if on else 0)
