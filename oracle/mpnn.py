"""CPU restatement of the learned block preconditioner (test infrastructure).

The network is this project's own part (the reference solves its Newton systems with plain
GMRES); this file is the checker of the device kernels of ``pd_mpnn.cu``: point features,
the two-layer message-passing network with BF16 operands and FP32 accumulation, the Krylov
training loss and its gradient. ``exact=True`` runs the same algebra in FP64 without BF16
rounding; its gradient is checked against finite differences, which pins this restatement.

Network (per point i, bonds j of i that are active):
  x_i  16 features of the point (``features``)
  h0 = relu(W0 x + b0)                                  64
  m_l = mean_j h_{l-1, j};  h_l = h_{l-1} + relu(W_l [h_{l-1}; m_l] + b_l),  l = 1, 2
  D_i = iso(Wo h2 + bo)     3x3 column-major; iso: every block s I, s = mean_j tr(A_j) / 3
The preconditioner blocks are B_i = P_i (I + D_i) = (1 + s) P_i with P_i the block-Jacobi
inverse: one learned scale per body keeps the blocks symmetric positive definite and K0 B
similar to a symmetric operator.

Loss over unit sample vectors r (recorded Krylov residual directions, alpha = 1, and top
eigenvectors of K0 P, alpha = 1 / tau):
  L = mean_s || (I - alpha_s K0 B)^2 r_s ||^2
with alpha = 1 the residual after one step of the block polynomial M = B (2 I - K0 B), the
small-strain stiffness K0 standing in for J.
"""
from __future__ import annotations

import numpy as np

N_FEAT, HID, N_OUT = 16, 64, 9
SHAPES = [("W0", (HID, N_FEAT)), ("b0", (HID,)), ("W1", (HID, 2 * HID)), ("b1", (HID,)),
          ("W2", (HID, 2 * HID)), ("b2", (HID,)), ("Wo", (N_OUT, HID)), ("bo", (N_OUT,))]
N_PARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def unpack(theta):
    out, o = {}, 0
    for name, s in SHAPES:
        k = int(np.prod(s))
        out[name] = theta[o:o + k].reshape(s)
        o += k
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], np.float32).reshape(-1) for name, _ in SHAPES])


def init_params(seed=0):
    """He-scaled random weights, zero output layer (the untrained network is block Jacobi)."""
    rng = np.random.default_rng(seed)
    d = {}
    for name, s in SHAPES:
        if name.startswith("W") and name != "Wo":
            d[name] = rng.standard_normal(s).astype(np.float32) * np.sqrt(2.0 / s[1])
        else:
            d[name] = np.zeros(s, np.float32)
    return pack(d)


def bf16(a):
    """Round float32 to bfloat16 (nearest, ties to even), returned as float32."""
    a = np.ascontiguousarray(a, np.float32)
    b = a.view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).reshape(a.shape)


class Graph:
    """Active bonds of an OracleBody: bond i -> j lists and counts."""

    def __init__(self, ob):
        i = np.repeat(np.arange(ob.n), np.diff(ob.off))
        act = ob.bond_active[: ob.n_bonds].astype(bool)
        self.i = i[act]
        self.j = ob.nbr.astype(np.int64)[act]
        self.n = ob.n
        self.cnt = np.bincount(self.i, minlength=ob.n).astype(np.float32)

    def mean(self, h):
        acc = np.zeros((self.n, h.shape[1]), np.float64)
        np.add.at(acc, self.i, h[self.j].astype(np.float64))
        acc = acc.astype(np.float32)
        with np.errstate(invalid="ignore", divide="ignore"):
            m = np.where(self.cnt[:, None] > 0, acc / self.cnt[:, None], 0.0)
        return m.astype(np.float32)

    def mean_adjoint(self, dm):
        """d h_j = sum over bonds (i -> j) of dm_i / n_i (the bonds are symmetric)."""
        with np.errstate(invalid="ignore", divide="ignore"):
            s = np.where(self.cnt[:, None] > 0, dm / self.cnt[:, None], 0.0).astype(np.float32)
        out = np.zeros(dm.shape, np.float64)
        np.add.at(out, self.j, s[self.i].astype(np.float64))
        return out.astype(np.float32)


def features(onk):
    """16 features per point from the reference configuration (OracleNK of oracle/jfnk.py):
    0-5  the K0 diagonal block K_ii = V_i sum_j c V_j / L^3 xi xi^T scaled by 3 / tr, minus I
         (xx, yy, zz, xy, xz, yz)
    6    tr(K_ii) / max tr - 1;  7  n_i / max n - 1
    8-10 displacement-constrained flags of the three dofs
    11-13 sum_j xi_j / (max n * delta_i);  14  its norm;  15  0"""
    ob = onk.ob
    i, j, L, c = onk._bonds()
    xi = ob.X[j] - ob.X[i]
    k = c * onk.V[j] * onk.V[i] / L ** 3
    K = np.zeros((ob.n, 3, 3))
    np.add.at(K, i, k[:, None, None] * xi[:, :, None] * xi[:, None, :])
    cnt = np.bincount(i, minlength=ob.n).astype(np.float64)
    sx = np.zeros((ob.n, 3))
    np.add.at(sx, i, xi)
    t = K[:, 0, 0] + K[:, 1, 1] + K[:, 2, 2]
    s = np.where(t > 0, 3.0 / np.where(t > 0, t, 1.0), 0.0)
    delta = np.array([p.delta for p in ob.params_list])[ob.pid]
    x = np.zeros((ob.n, N_FEAT))
    x[:, 0] = s * K[:, 0, 0] - 1
    x[:, 1] = s * K[:, 1, 1] - 1
    x[:, 2] = s * K[:, 2, 2] - 1
    x[:, 3] = s * K[:, 0, 1]
    x[:, 4] = s * K[:, 0, 2]
    x[:, 5] = s * K[:, 1, 2]
    x[:, 6] = t / t.max() - 1
    x[:, 7] = cnt / cnt.max() - 1
    x[:, 8:11] = onk.cmask.reshape(-1, 3)
    x[:, 11:14] = sx / (cnt.max() * delta[:, None])
    x[:, 14] = np.linalg.norm(x[:, 11:14], axis=1)
    return x.astype(np.float32)


def forward(theta, x, g, exact=False):
    """Activations of the network; D (n x 9, column-major 3x3 blocks)."""
    rd = (lambda a: np.asarray(a, np.float64)) if exact else bf16
    p = {k: np.asarray(v, np.float64 if exact else np.float32) for k, v in unpack(theta).items()}
    W = {k: rd(v) for k, v in p.items() if k.startswith("W")}
    act = {"x": rd(x)}
    z0 = act["x"] @ W["W0"].T + p["b0"]
    act["h0"] = rd(np.maximum(z0, 0))
    h = act["h0"]
    for l in (1, 2):
        m = _mean64(g, h) if exact else bf16(g.mean(h))
        z = np.concatenate([h, m], axis=1) @ W[f"W{l}"].T + p[f"b{l}"]
        a = rd(np.maximum(z, 0))
        hn = rd(h + a)
        act[f"m{l}"], act[f"a{l}"], act[f"h{l}"] = m, a, hn
        h = hn
    act["D"] = iso(h @ W["Wo"].T + p["bo"])
    return act


def iso(D):
    """Body-wide isotropic readout of n x 9 blocks: every block becomes s I with
    s = mean tr / 3. Applied to a gradient it gives the adjoint (sum tr / (3 n)) I."""
    t = (D[:, 0] + D[:, 4] + D[:, 8]).mean() / 3
    out = np.zeros_like(D)
    out[:, 0] = out[:, 4] = out[:, 8] = t
    return out


def _mean64(g, h):
    acc = np.zeros((g.n, h.shape[1]))
    np.add.at(acc, g.i, h[g.j])
    return np.where(g.cnt[:, None] > 0, acc / np.maximum(g.cnt[:, None], 1), 0.0)


def _mean_adj64(g, dm):
    s = np.where(g.cnt[:, None] > 0, dm / np.maximum(g.cnt[:, None], 1), 0.0)
    out = np.zeros(dm.shape)
    np.add.at(out, g.j, s[g.i])
    return out


def backward(theta, act, dD, g, exact=False):
    """Gradient of a scalar with respect to theta, given dD = d scalar / d D."""
    rd = (lambda a: np.asarray(a, np.float64)) if exact else bf16
    p = unpack(theta)
    W = {k: rd(np.asarray(v, np.float64 if exact else np.float32)) for k, v in p.items()
         if k.startswith("W")}
    grads = {}
    dD = iso(dD)
    dDb = rd(dD)
    grads["Wo"] = dDb.T @ act["h2"]
    grads["bo"] = dD.sum(axis=0)
    dh = dDb @ W["Wo"]
    for l in (2, 1):
        hp = act["h0"] if l == 1 else act["h1"]
        dz = rd(dh * (act[f"a{l}"] > 0))
        X = np.concatenate([hp, act[f"m{l}"]], axis=1)
        grads[f"W{l}"] = dz.T @ X
        grads[f"b{l}"] = dz.sum(axis=0)
        dX = dz @ W[f"W{l}"]
        dm = dX[:, HID:]
        adj = _mean_adj64(g, dm) if exact else g.mean_adjoint(dm.astype(np.float32))
        dh = dh + dX[:, :HID] + adj
    dz0 = rd(dh * (act["h0"] > 0))
    grads["W0"] = dz0.T @ act["x"]
    grads["b0"] = dz0.sum(axis=0)
    return np.concatenate([np.asarray(grads[name], np.float64).reshape(-1) for name, _ in SHAPES])


def loss_and_dD(onk, P, D, samples, alphas=None):
    """L = mean_s ||(I - alpha_s K0 B)^2 r_s||^2 with B = P (I + D) (constrained rows zero)
    and its gradient with respect to D (n x 9, column-major blocks)."""
    n = onk.n
    Dm = D.reshape(n, 3, 3).transpose(0, 2, 1)  # column-major -> [n, row, col]
    B = np.einsum("nab,nbc->nac", P, np.eye(3) + Dm)
    cm = onk.cmask

    def Bm(w):
        z = np.einsum("nab,nb->na", B, w.reshape(-1, 3)).reshape(-1)
        z[cm] = 0.0
        return z

    def BTm(w):
        return np.einsum("nba,nb->na", B, w.reshape(-1, 3)).reshape(-1)

    G = np.zeros((n, 3, 3))
    L = 0.0
    S = len(samples)
    alphas = [1.0] * S if alphas is None else alphas
    for r, al in zip(samples, alphas):
        r = np.asarray(r, np.float64)
        K = lambda v: al * onk.k0(v)
        y1 = r - K(Bm(r))
        y2 = y1 - K(Bm(y1))
        L += float(np.dot(y2, y2)) / S
        w = K(y2)
        q = y2 - BTm(w)
        q[cm] = 0.0  # K0 with masked rows has the adjoint K0 with masked columns
        g1 = K(q)
        a = (-2.0 / S) * (g1.reshape(-1, 3)[:, :, None] * r.reshape(-1, 3)[:, None, :]
                          + w.reshape(-1, 3)[:, :, None] * y1.reshape(-1, 3)[:, None, :])
        a[cm.reshape(-1, 3)] = 0.0  # rows of constrained dofs do not reach B v
        G += a
    dDm = np.einsum("nba,nbc->nac", P, G)  # P^T G
    return L, dDm.transpose(0, 2, 1).reshape(n, 9)


def spectral_loss_and_dD(onk, P, D, slow, fast, tau, weight):
    """L = -mean_slow rho(r) + weight mean_fast max(rho(q) - tau, 0)^2, rho(v) = v . K0 B v,
    and its gradient with respect to D (n x 9, column-major)."""
    n = onk.n
    Dm = D.reshape(n, 3, 3).transpose(0, 2, 1)
    B = np.einsum("nab,nbc->nac", P, np.eye(3) + Dm)
    cm = onk.cmask

    def Bm(w):
        z = np.einsum("nab,nb->na", B, w.reshape(-1, 3)).reshape(-1)
        z[cm] = 0.0
        return z

    G = np.zeros((n, 3, 3))
    L = 0.0
    for v, f_of in [(r, None) for r in slow] + [(q, True) for q in fast]:
        v = np.asarray(v, np.float64)
        rho = float(v @ onk.k0(Bm(v)))
        if f_of is None:
            L -= rho / len(slow)
            f = -1.0 / len(slow)
        elif rho > tau:
            L += weight * (rho - tau) ** 2 / len(fast)
            f = weight * 2.0 * (rho - tau) / len(fast)
        else:
            continue
        a = f * onk.k0(v).reshape(-1, 3)[:, :, None] * v.reshape(-1, 3)[:, None, :]
        a[cm.reshape(-1, 3)] = 0.0
        G += a
    dDm = np.einsum("nba,nbc->nac", P, G)
    return L, dDm.transpose(0, 2, 1).reshape(n, 9)


def loss_grad(theta, onk, P, samples, x=None, g=None, exact=False, alphas=None):
    """Loss and d loss / d theta of the network on one body."""
    g = g or Graph(onk.ob)
    x = features(onk) if x is None else x
    act = forward(theta, x, g, exact)
    L, dD = loss_and_dD(onk, P, act["D"].astype(np.float64), samples, alphas)
    return L, backward(theta, act, dD if exact else dD.astype(np.float32), g, exact)
