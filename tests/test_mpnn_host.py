"""The CPU restatement of the learned preconditioner (oracle/mpnn.py), pinned by finite
differences: its exact FP64 gradient of the Krylov loss with respect to the corrections D and
to every parameter block of the network. No GPU."""
import numpy as np

from helpers import oracle_body
from jfnk import OracleNK
import mpnn as M
from pdcuda import mpnn as P
from test_nk_host import nk_conditions, small_beam


def _problem(seed=0):
    body = small_beam(nx=12, ny=5, nz=4)
    onk = OracleNK(oracle_body(body), nk_conditions(body))
    P_blocks = onk.bj_blocks()
    rng = np.random.default_rng(seed)
    samples = []
    for _ in range(2):
        r = rng.standard_normal(3 * onk.n)
        r[onk.cmask] = 0.0
        samples.append(r / np.linalg.norm(r))
    return onk, P_blocks, samples, rng


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.0e-5, 65504.0], np.float32)
    # 1 + 2^-8 is a tie: rounds to even (1.0); 1 + 1.5 * 2^-8 rounds up to 1 + 2^-7
    assert list(M.bf16(x)[:3]) == [1.0, 1.0, 1.0078125]
    assert M.bf16(x)[3] < 0 and abs(M.bf16(x)[3] + 3.0e-5) < 3.0e-5 / 128


def test_loss_gradient_in_D_matches_finite_differences():
    onk, Pb, samples, rng = _problem()
    D = rng.uniform(-0.1, 0.1, (onk.n, 9))
    al = [1.0, 0.55]
    L0, dD = M.loss_and_dD(onk, Pb, D, samples, al)
    h = 1e-6
    for _ in range(8):
        i, k = rng.integers(onk.n), rng.integers(9)
        Dp, Dm = D.copy(), D.copy()
        Dp[i, k] += h
        Dm[i, k] -= h
        fd = (M.loss_and_dD(onk, Pb, Dp, samples, al)[0]
              - M.loss_and_dD(onk, Pb, Dm, samples, al)[0]) / (2 * h)
        assert abs(dD[i, k] - fd) <= 1e-6 * max(abs(fd), 1e-3), (i, k, dD[i, k], fd)


def test_network_gradient_matches_finite_differences():
    onk, Pb, samples, rng = _problem(1)
    theta = P.init_params(3).astype(np.float64)
    d = M.unpack(theta.copy())
    d["Wo"] = rng.standard_normal(d["Wo"].shape) * 0.05
    d["bo"] = rng.standard_normal(9) * 0.05
    theta = np.concatenate([np.asarray(d[name], np.float64).reshape(-1) for name, _ in M.SHAPES])
    x = M.features(onk).astype(np.float64)
    g = M.Graph(onk.ob)
    _, grad = M.loss_grad(theta, onk, Pb, samples, x=x, g=g, exact=True)
    h = 1e-6
    o = 0
    for name, s in M.SHAPES:
        size = int(np.prod(s))
        idx = o + rng.integers(size, size=2)
        for k in idx:
            tp, tm = theta.copy(), theta.copy()
            tp[k] += h
            tm[k] -= h
            fd = (M.loss_grad(tp, onk, Pb, samples, x=x, g=g, exact=True)[0]
                  - M.loss_grad(tm, onk, Pb, samples, x=x, g=g, exact=True)[0]) / (2 * h)
            assert abs(grad[k] - fd) <= 1e-5 * max(abs(fd), 1e-4), (name, k, grad[k], fd)
        o += size


def test_untrained_network_is_block_jacobi():
    onk, _, _, _ = _problem()
    act = M.forward(P.init_params(0), M.features(onk), M.Graph(onk.ob))
    assert np.all(act["D"] == 0.0)


def test_spectral_loss_gradient_matches_finite_differences():
    onk, Pb, slow, rng = _problem(2)
    fast = []
    for _ in range(2):
        q = rng.standard_normal(3 * onk.n)
        q[onk.cmask] = 0.0
        fast.append(q / np.linalg.norm(q))
    D = rng.uniform(-0.1, 0.1, (onk.n, 9))
    _, dD = M.spectral_loss_and_dD(onk, Pb, D, slow, fast, 0.5, 3.0)
    h = 1e-6
    for _ in range(8):
        i, k = rng.integers(onk.n), rng.integers(9)
        Dp, Dm = D.copy(), D.copy()
        Dp[i, k] += h
        Dm[i, k] -= h
        fd = (M.spectral_loss_and_dD(onk, Pb, Dp, slow, fast, 0.5, 3.0)[0]
              - M.spectral_loss_and_dD(onk, Pb, Dm, slow, fast, 0.5, 3.0)[0]) / (2 * h)
        assert abs(dD[i, k] - fd) <= 1e-6 * max(abs(fd), 1e-4), (i, k, dD[i, k], fd)
