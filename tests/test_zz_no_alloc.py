"""pd_osb_force_static: the force evaluation for callers that must not let the library
allocate device memory (a host with its own memory pool, an allocation-free time loop).

All of its inputs and outputs are device arrays that the caller owns (here: torch tensors);
its scratch state lives in a static device array of the library. Two calls in a row must
reproduce the force density, bond states and active-bond counts of the regular entry points
(pd_create + pd_force, FP64 serial-order mapping), within the FP64 tolerance of these tests,
for each of the three influence functions and for bond states that differ between the two
directions of a pair.
"""
import ctypes as C

import numpy as np
import pytest

import pdcuda as pd
from helpers import cube_body, deform

pytestmark = pytest.mark.gpu
RTOL = 1e-12


def csr_bonds(body, delta):
    lib = pd.lib()
    n = body.n_points
    d = np.full(n, delta)
    nb = C.c_int64()
    fp = body.fail_permit.astype(np.uint8)
    assert lib.pd_find_bonds(n, body._pos.ctypes.data, d.ctypes.data, fp.ctypes.data, 0, None, None,
                             0, None, None, None, None, C.byref(nb), 0) == 0
    off = np.zeros(n + 1, np.int64)
    nbr = np.zeros(nb.value, np.int32)
    L = np.zeros(nb.value)
    fpb = np.zeros(nb.value, np.uint8)
    assert lib.pd_find_bonds(n, body._pos.ctypes.data, d.ctypes.data, fp.ctypes.data, 0, None, None,
                             nb.value, off.ctypes.data, nbr.ctypes.data, L.ctypes.data,
                             fpb.ctypes.data, C.byref(nb), 0) == 0
    return off, nbr, L, fpb


def regular_force(body, off, nbr, L, fpb, x, kernel, bond_active=None):
    """The regular entry points: pd_create on the same CSR bonds, pd_force (FP64, serial
    order), from the given bond states (all active when None)."""
    lib = pd.lib()
    p = body.point_params[0].to_c()
    desc = pd._lib.BodyDesc()
    desc.n_points = body.n_points
    desc.position = body._pos.ctypes.data
    desc.volume = body.volume.ctypes.data
    desc.n_bonds = len(nbr)
    desc.bond_offsets = off.ctypes.data
    desc.neighbors = nbr.ctypes.data
    desc.bond_length = L.ctypes.data
    desc.fail_permit = fpb.ctypes.data
    desc.n_params = 1
    desc.params = C.cast(C.pointer(p), C.c_void_p)
    desc.material = pd._lib.MAT_OSB
    desc.kernel = kernel
    desc.precision = pd._lib.PREC_FP64
    desc.zem_cs = 0.5
    desc.maxdmg = 0.85
    h = C.c_void_p()
    assert lib.pd_create(C.byref(desc), C.byref(h)) == 0, pd._lib.last_error()
    try:
        assert lib.pd_set_mapping(h, 0, 128) == 0
        xs = np.ascontiguousarray(x)
        ba0 = None if bond_active is None else np.ascontiguousarray(bond_active, np.uint8)
        assert lib.pd_set_state(h, xs.ctypes.data, None, None, None, None, None,
                                None if ba0 is None else ba0.ctypes.data) == 0
        assert lib.pd_force(h, 0.0, 0.0) == 0
        n = body.n_points
        b = np.zeros((n, 3))
        na = np.zeros(n, np.int64)
        ba = np.zeros(len(nbr), np.uint8)
        assert lib.pd_get_field(h, pd._lib.F_B_INT, b.ctypes.data, b.nbytes) == 0
        assert lib.pd_get_field(h, pd._lib.F_N_ACTIVE_BONDS, na.ctypes.data, na.nbytes) == 0
        assert lib.pd_get_field(h, pd._lib.F_BOND_ACTIVE, ba.ctypes.data, ba.nbytes) == 0
    finally:
        lib.pd_destroy(h)
    return b, na, ba


KERNELS = {"linear": pd._lib.KERNEL_LINEAR, "const_one": pd._lib.KERNEL_CONST_ONE,
           "cubic_b_spline": pd._lib.KERNEL_CUBIC_BSPLINE}


@pytest.mark.parametrize("states", ["symmetric", "one_direction"])
@pytest.mark.parametrize("kernel", list(KERNELS))
def test_static_scratch_entry_point_matches_regular_entry_points(kernel, states):
    """Each influence function, from all bonds active and from bond states that differ in the
    two directions of some pairs (the term of a neighbour then uses its own bond)."""
    import torch
    body = cube_body(pd.OSBMaterial(), n=10, fracture=True, Gc=6e6)
    delta = body.point_params[0].delta
    off, nbr, L, fpb = csr_bonds(body, delta)
    x = body._pos + deform(body._pos, amplitude=4e-3)
    ba0 = np.ones(len(nbr), np.uint8)
    if states == "one_direction":
        ba0 = (np.random.default_rng(7).random(len(nbr)) > 0.15).astype(np.uint8)
    b_ref, na_ref, ba_ref = regular_force(body, off, nbr, L, fpb, x, KERNELS[kernel], ba0)
    assert 0 < np.count_nonzero(ba_ref == 0) < len(ba_ref)  # some bonds broke, not all

    dev = torch.device("cuda:0")
    t = lambda a, dt: torch.tensor(np.ascontiguousarray(a), dtype=dt, device=dev)
    X_d, x_d = t(body._pos, torch.float64), t(x, torch.float64)
    vol_d = t(body.volume, torch.float64)
    off_d, nbr_d = t(off, torch.int64), t(nbr, torch.int32)
    L_d, fp_d = t(L, torch.float64), t(fpb, torch.uint8)
    n = body.n_points
    p = body.point_params[0].to_c()
    lib = pd.lib()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call in range(2):
        ba_d = t(ba0, torch.uint8)
        b_d = torch.full((n, 3), float("nan"), dtype=torch.float64, device=dev)
        na_d = torch.full((n,), -1, dtype=torch.int64, device=dev)
        st = lib.pd_osb_force_static(n, X_d.data_ptr(), x_d.data_ptr(), vol_d.data_ptr(),
                                     off_d.data_ptr(), nbr_d.data_ptr(), L_d.data_ptr(),
                                     fp_d.data_ptr(), ba_d.data_ptr(), C.byref(p),
                                     KERNELS[kernel], b_d.data_ptr(), na_d.data_ptr(), stream)
        assert st == 0, lib.pd_static_last_error()
        torch.cuda.synchronize()
        b = b_d.cpu().numpy()
        scale = np.abs(b_ref).max()
        assert scale > 0
        assert np.abs(b - b_ref).max() <= RTOL * scale, f"call {call}"
        assert np.array_equal(na_d.cpu().numpy(), na_ref), f"call {call}"
        assert np.array_equal(ba_d.cpu().numpy(), ba_ref), f"call {call}"


def test_static_scratch_entry_point_rejects_too_many_points():
    lib = pd.lib()
    p = pd.point_parameters(pd.OSBMaterial(), horizon=1.0, rho=1.0, E=1.0, nu=0.25).to_c()
    one = C.c_void_p(1)  # never dereferenced: the size check comes first
    st = lib.pd_osb_force_static((1 << 18) + 1, one, one, one, one, one, one, one, one,
                                 C.byref(p), pd._lib.KERNEL_LINEAR, one, one, None)
    assert st == pd._lib.PD_ERR_ARG
    assert b"at most 262144 points" in lib.pd_static_last_error()
