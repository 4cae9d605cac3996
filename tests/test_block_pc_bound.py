"""What a per-point 3x3 block preconditioner can gain in the block-polynomial Krylov solve of
the bending beam, on the CPU (the learned preconditioner predicts such blocks).

The bond-based small-strain stiffness A = -K0 of a three-point-bending beam (the reference's
Newton systems, newton_krylov.jl:415-460, linearised at the reference configuration) is
assembled as a sparse matrix over the free dofs; restarted GMRES(50) with the block
polynomial M = B (2 I - A B) solves A x = b to 1e-8 for several per-point block choices B:
block Jacobi B_i = (A_ii)^-1 scaled uniformly, and the exact diagonal 3x3 blocks of A^-1 (the
natural per-point target: what the blocks of the inverse are), at several scales and mixed
with block Jacobi's magnitude or shape. Every per-point choice needs more iterations than the
best uniform scaling of block Jacobi: the gain of a per-point block preconditioner over the
uniformly scaled block Jacobi is bounded by what a uniform scale gives, which is what the
shipped readout (one learned scale per body) learns.
"""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from jfnk import OracleNK
from helpers import oracle_body
from test_nk_host import nk_conditions, small_beam


def beam_system(nx, ny, nz):
    body = small_beam(nx=nx, ny=ny, nz=nz)
    ob = oracle_body(body)
    nk = OracleNK(ob, nk_conditions(body))
    i, j, L, c = nk._bonds()
    xi = ob.X[j] - ob.X[i]
    k = c * nk.V[j] * nk.V[i] / L ** 3
    blk = k[:, None, None] * xi[:, :, None] * xi[:, None, :]
    rows, cols, vals = [], [], []
    for a in range(3):
        for b in range(3):   # K0 v_i = sum_j k xi (xi . (v_j - v_i)); A = -K0
            rows += [3 * i + a, 3 * i + a]
            cols += [3 * j + b, 3 * i + b]
            vals += [-blk[:, a, b], blk[:, a, b]]
    A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(3 * ob.n, 3 * ob.n))
    free = np.nonzero(~nk.cmask)[0]
    return A[free][:, free].tocsr(), free // 3, ob.n


def blocks_of(M, pt, n):
    """Per point the square block of M on its free dofs (dense M or sparse)."""
    starts = np.searchsorted(pt, np.arange(n))
    ends = np.searchsorted(pt, np.arange(n), side="right")
    out = []
    for s, e in zip(starts, ends):
        blk = M[s:e, s:e]
        out.append(np.asarray(blk.todense() if sp.issparse(blk) else blk) if e > s else None)
    return out, starts, ends


def iterations(A, blocks, starts, ends, w, b):
    m = A.shape[0]

    def Bm(v):
        z = np.zeros(m)
        for Bp, s, e in zip(blocks, starts, ends):
            if Bp is not None:
                z[s:e] = w * (Bp @ v[s:e])
        return z

    M = spla.LinearOperator((m, m), matvec=lambda v: Bm(2 * v - A @ Bm(v)))
    it = [0]

    def count(_):
        it[0] += 1
    _, info = spla.gmres(A, b, M=M, restart=50, rtol=1e-8, maxiter=40, callback=count,
                         callback_type="pr_norm")
    return it[0] if info == 0 else np.inf


def test_per_point_blocks_do_not_beat_uniformly_scaled_block_jacobi():
    A, pt, n = beam_system(24, 6, 4)
    m = A.shape[0]
    b = A @ np.random.default_rng(0).standard_normal(m)
    P, starts, ends = blocks_of(A, pt, n)
    P = [None if p is None else np.linalg.inv(p) for p in P]
    ideal, _, _ = blocks_of(np.linalg.inv(A.toarray()), pt, n)
    shape = [None if q is None else q * (np.trace(p) / np.trace(q)) for p, q in zip(P, ideal)]
    mag = [None if q is None else p * (np.trace(q) / np.trace(p)) for p, q in zip(P, ideal)]
    best_bj = min(iterations(A, P, starts, ends, w, b) for w in (0.8, 1.0, 1.2))
    per_point = {
        "inverse blocks": min(iterations(A, ideal, starts, ends, w, b)
                              for w in (0.005, 0.02, 0.05, 0.1, 0.2, 0.5)),
        "inverse shape, Jacobi magnitude": min(iterations(A, shape, starts, ends, w, b)
                                               for w in (0.6, 0.8, 1.0)),
        "Jacobi shape, inverse magnitude": min(iterations(A, mag, starts, ends, w, b)
                                               for w in (0.005, 0.02, 0.05)),
    }
    print(f"{m} free dofs: scaled block Jacobi {best_bj} iterations; per-point {per_point}")
    assert np.isfinite(best_bj)
    for name, its in per_point.items():
        assert its > best_bj, name
