"""The learned block preconditioner of the Newton-Krylov solve (no reference counterpart).

``BlockPreconditionerNet`` holds a two-layer message-passing network on the device
(``pd_mpnn_*`` of libpdcuda): 16 features per point, hidden width 64, BF16 tensor-core
layers with FP32 accumulation. It predicts per-point corrections D_i of the block-Jacobi
blocks, B_i = P_i (I + D_i), read out over the body as one isotropic scale (D_i = s I; full
3x3 corrections and per-point scalings made the Krylov solves slower), which ``NewtonKrylov(preconditioner="learned_poly")`` applies
inside FGMRES as z = B (2 v - K0 B v). The untrained network (zero output layer) is the
block-Jacobi polynomial.

With the polynomial the preconditioned spectrum is mu = lambda (2 - lambda) for the
eigenvalues lambda of K0 B: the slow end gains from scaling B up, until the fast end reaches 2
and the polynomial turns it negative. Training (``train``) uses the spectral loss
-mean rho(r) + w mean max(rho(q) - tau, 0)^2 with rho(v) = v . K0 B v: r are the Krylov
residual directions recorded at every restart of plain block-Jacobi runs (``collect``,
``pd_nk_record``: the slow end, where those runs stall), q the top eigenvectors of K0 B under
the current network (power iteration). Adam minimises it with the device's own forward and
backward kernels.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from . import newton_krylov as nkm

N_FEAT, HID, N_OUT = 16, 64, 9
SHAPES = [("W0", (HID, N_FEAT)), ("b0", (HID,)), ("W1", (HID, 2 * HID)), ("b1", (HID,)),
          ("W2", (HID, 2 * HID)), ("b2", (HID,)), ("Wo", (N_OUT, HID)), ("bo", (N_OUT,))]
N_PARAMS = sum(int(np.prod(s)) for _, s in SHAPES)
assert N_PARAMS == L.MPNN_N_PARAMS


def init_params(seed=0):
    """He-scaled random hidden weights, zero biases and output layer."""
    rng = np.random.default_rng(seed)
    parts = []
    for name, s in SHAPES:
        if name.startswith("W") and name != "Wo":
            parts.append((rng.standard_normal(s) * np.sqrt(2.0 / s[1])).astype(np.float32))
        else:
            parts.append(np.zeros(s, np.float32))
    return np.concatenate([p.reshape(-1) for p in parts])


class BlockPreconditionerNet:
    def __init__(self, theta=None, device=0, seed=0):
        self.h = C.c_void_p()
        self.device = device
        L.check(L.lib().pd_mpnn_create(device, C.byref(self.h)), "pd_mpnn_create")
        self.set_params(init_params(seed) if theta is None else theta)

    # -- parameters ---------------------------------------------------------------------------
    def set_params(self, theta):
        theta = np.ascontiguousarray(theta, np.float32)
        if theta.size != N_PARAMS:
            raise ValueError(f"expected {N_PARAMS} parameters")
        L.check(L.lib().pd_mpnn_set_params(self.h, L.ptr(theta)), "pd_mpnn_set_params")

    def params(self):
        out = np.empty(N_PARAMS, np.float32)
        L.check(L.lib().pd_mpnn_get_params(self.h, L.ptr(out)), "pd_mpnn_get_params")
        return out

    def save(self, path):
        np.savez(path, theta=self.params())

    @classmethod
    def load(cls, path, device=0):
        return cls(np.load(path)["theta"], device=device)

    # -- inference ----------------------------------------------------------------------------
    def infer(self, dev):
        """Features [n x 16] and corrections D [n x 9] of a device body (whose conditions are
        set); D is also installed as the body's corrections."""
        x = np.empty((dev.n, N_FEAT), np.float32)
        D = np.empty((dev.n, N_OUT), np.float32)
        L.check(L.lib().pd_mpnn_infer(self.h, dev.h, L.ptr(x), L.ptr(D)), "pd_mpnn_infer")
        return x, D

    def corrections(self, dev):
        return self.infer(dev)[1]

    # -- training -----------------------------------------------------------------------------
    def loss_grad(self, dev, rec_ids=(), samples=None, alpha=1.0, weight=1.0):
        """Loss over recorded directions (indices) and host samples [k x 3n] (scale alpha of
        K0 and weight inside the loss); the gradient is accumulated on the device and
        returned."""
        ids = np.ascontiguousarray(rec_ids, np.int64)
        smp = None if samples is None else np.ascontiguousarray(samples, np.float32).reshape(-1, 3 * dev.n)
        n_host = 0 if smp is None else smp.shape[0]
        loss = C.c_double()
        grad = np.empty(N_PARAMS, np.float32)
        L.check(L.lib().pd_mpnn_loss_grad(self.h, dev.h, len(ids), L.ptr(ids) if len(ids) else None,
                                          n_host, L.ptr(smp), float(alpha), float(weight),
                                          C.byref(loss),
                                          L.ptr(grad)),
                "pd_mpnn_loss_grad")
        return loss.value, grad

    def spectral_grad(self, dev, rec_ids=(), fast=None, tau=1.85, weight=100.0):
        """Spectral loss over recorded directions (the slow end, pulled up) and fast samples
        [k x 3n] (held below tau); the gradient is accumulated on the device and returned."""
        ids = np.ascontiguousarray(rec_ids, np.int64)
        smp = None if fast is None else np.ascontiguousarray(fast, np.float32).reshape(-1, 3 * dev.n)
        n_host = 0 if smp is None else smp.shape[0]
        loss = C.c_double()
        grad = np.empty(N_PARAMS, np.float32)
        L.check(L.lib().pd_mpnn_spectral_grad(self.h, dev.h, len(ids), L.ptr(ids) if len(ids) else None,
                                              n_host, L.ptr(smp), float(tau), float(weight),
                                              C.byref(loss), L.ptr(grad)),
                "pd_mpnn_spectral_grad")
        return loss.value, grad

    def zero_grad(self):
        L.check(L.lib().pd_mpnn_zero_grad(self.h), "pd_mpnn_zero_grad")

    def adam(self, lr):
        L.check(L.lib().pd_mpnn_adam(self.h, float(lr)), "pd_mpnn_adam")

    def close(self):
        if self.h:
            L.lib().pd_mpnn_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def constrained_mask(body):
    """Displacement-constrained dofs of a body (3 n bools)."""
    m = np.zeros(3 * body.n_points, bool)
    for c in body.pos_single_dim_bcs:
        if c.field == "displacement":
            m[3 * np.asarray(body.point_sets[c.point_set]) + c.dim] = True
    return m


def random_probes(mask, k, rng):
    """k unit vectors of uniform entries, zero at the constrained dofs (fast modes)."""
    p = rng.uniform(-1.0, 1.0, (k, mask.size)).astype(np.float32)
    p[:, mask] = 0.0
    p /= np.linalg.norm(p, axis=1, keepdims=True)
    return p


def top_modes(dev, k=4, iters=30, seed=0, start=None, learned=False):
    """k approximate top eigenvectors of K0 B by power iteration: B = P (block Jacobi at the
    current state), or the learned blocks installed on dev (learned=True). Starts from
    `start` (k x 3n) or random vectors. The fast end of the preconditioned spectrum."""
    rng = np.random.default_rng(seed)
    nk = nkm.NewtonKrylov(steps=1, preconditioner="learned" if learned else "block_jacobi")
    mask = constrained_mask(dev.body)
    out = []
    for m in range(k):
        if start is not None:
            q = np.asarray(start[m], np.float64).copy()
        else:
            q = rng.uniform(-1.0, 1.0, 3 * dev.n)
            q[mask] = 0.0
        q /= np.linalg.norm(q)
        for _ in range(iters):
            q = nkm.apply_operator(dev, nk, "k0", nkm.apply_operator(dev, nk, "precond", q))
            q /= np.linalg.norm(q)
        out.append(q.astype(np.float32))
    return np.array(out)


def rayleigh(dev, q, learned=True):
    """q . K0 B q for unit q (B learned or block Jacobi)."""
    nk = nkm.NewtonKrylov(steps=1, preconditioner="learned" if learned else "block_jacobi")
    q = np.asarray(q, np.float64)
    return float(q @ nkm.apply_operator(dev, nk, "k0", nkm.apply_operator(dev, nk, "precond", q)))


def collect(dev, nk, increments, capacity):
    """Run plain solves of the first `increments` load steps of `nk` on dev, recording up to
    `capacity` residual directions; returns how many were recorded."""
    nkm.record(dev, capacity)
    nkm.setup(dev, nk)
    for n in range(1, increments + 1):
        try:
            nkm.step(dev, nk, n)
        except L.NotConvergedError:
            break  # the directions recorded so far are the data
    return nkm.recorded(dev)


def train(net, devs, steps, lr=1e-3, batch=16, n_fast=8, tau=1.85, weight=100.0, refresh=5,
          power_iters=6, seed=0, log=None):
    """Adam on the bodies in turn with the spectral loss: every step takes `batch` recorded
    Krylov directions of one body (the slow end of its preconditioned spectrum, pulled up) and
    its `n_fast` top eigenvectors of K0 B under the current network (recomputed by a few power
    iterations every `refresh` visits), held below tau. Returns the loss history."""
    rng = np.random.default_rng(seed)
    counts = [nkm.recorded(d) for d in devs]
    fast = [top_modes(d, n_fast, seed=seed + k) for k, d in enumerate(devs)]
    hist = []
    for s in range(steps):
        k = s % len(devs)
        visit = s // len(devs)
        if visit > 0 and visit % refresh == 0:
            net.infer(devs[k])
            fast[k] = top_modes(devs[k], n_fast, iters=power_iters, start=fast[k], learned=True)
        ids = rng.choice(counts[k], size=min(batch, counts[k]), replace=False)
        loss, _ = net.spectral_grad(devs[k], ids, fast[k], tau, weight)
        net.adam(lr)
        hist.append(loss)
        if log and (s % 20 == 0 or s == steps - 1):
            log(f"step {s:4d} body {k} loss {loss:.4e}")
    return hist
