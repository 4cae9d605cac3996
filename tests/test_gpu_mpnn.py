"""The learned block preconditioner on the device against its CPU restatement
(oracle/mpnn.py): features, the BF16 forward pass, the training loss and the gradient of
every parameter; then what the trained network gains in a Newton-Krylov solve."""
import numpy as np
import pytest

import pdcuda as pd
from pdcuda import mpnn as P
from pdcuda import newton_krylov as nkm
from helpers import oracle_body
from jfnk import OracleNK
import mpnn as M
from test_nk_host import nk_conditions, small_beam

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))


def setup_pair(nx=14, ny=6, nz=4, seed=0):
    body = small_beam(nx=nx, ny=ny, nz=nz)
    dev = pd.DeviceBody(body, precision="fp64")
    nkm.setup(dev, pd.NewtonKrylov(steps=1))
    onk = OracleNK(oracle_body(body), nk_conditions(body))
    rng = np.random.default_rng(seed)
    theta = P.init_params(seed)
    d = M.unpack(theta.copy())
    d["Wo"] = (rng.standard_normal(d["Wo"].shape) * 0.05).astype(np.float32)
    d["bo"] = (rng.standard_normal(9) * 0.05).astype(np.float32)
    for l in ("b0", "b1", "b2"):
        d[l] = (rng.standard_normal(d[l].shape) * 0.1).astype(np.float32)
    return body, dev, onk, M.pack(d)


def test_features_and_forward_match_oracle():
    body, dev, onk, theta = setup_pair()
    net = P.BlockPreconditionerNet(theta)
    x, D = net.infer(dev)
    xo = M.features(onk)
    assert np.max(np.abs(x - xo)) <= 1e-5
    act = M.forward(theta, xo, M.Graph(onk.ob))
    # BF16 activations: the device and the oracle round the same values, summed in a
    # different order
    assert rel(D, act["D"]) <= 1e-2
    # the exact FP64 network: BF16 costs about a percent
    exact = M.forward(theta.astype(np.float64), xo.astype(np.float64), M.Graph(onk.ob), exact=True)
    assert rel(D, exact["D"]) <= 3e-2


def test_loss_and_gradient_match_oracle():
    body, dev, onk, theta = setup_pair(seed=1)
    net = P.BlockPreconditionerNet(theta)
    rng = np.random.default_rng(4)
    samples = P.random_probes(onk.cmask, 3, rng)
    loss, grad = net.loss_grad(dev, (), samples, alpha=0.6, weight=3.0)
    P_blocks = onk.bj_blocks().astype(np.float32).astype(np.float64)
    Lo, go = M.loss_grad(theta, onk, P_blocks, [s.astype(np.float64) for s in samples],
                         alphas=[0.6] * len(samples))
    Lo, go = 3.0 * Lo, 3.0 * go
    assert abs(loss - Lo) <= 1e-3 * Lo
    assert rel(grad, go) <= 3e-2
    # every parameter block receives its gradient
    o = 0
    for name, s in M.SHAPES:
        k = int(np.prod(s))
        assert rel(grad[o:o + k], go[o:o + k]) <= 6e-2, name
        o += k


def test_gradient_with_several_point_chunks_per_block_matches_oracle():
    """45,600 points: more 128-point chunks (357, the last one ragged) than the 296 blocks of
    the weight-gradient kernels, so blocks accumulate two chunks in tensor memory."""
    body, dev, onk, theta = setup_pair(nx=100, ny=24, nz=19, seed=5)
    net = P.BlockPreconditionerNet(theta)
    rng = np.random.default_rng(6)
    samples = P.random_probes(onk.cmask, 2, rng)
    loss, grad = net.loss_grad(dev, (), samples, alpha=0.6, weight=1.0)
    P_blocks = onk.bj_blocks().astype(np.float32).astype(np.float64)
    Lo, go = M.loss_grad(theta, onk, P_blocks, [s.astype(np.float64) for s in samples],
                         alphas=[0.6] * len(samples))
    assert abs(loss - Lo) <= 1e-3 * Lo
    assert rel(grad, go) <= 3e-2
    o = 0
    for name, s in M.SHAPES:
        k = int(np.prod(s))
        assert rel(grad[o:o + k], go[o:o + k]) <= 6e-2, name
        o += k


def test_spectral_gradient_matches_oracle():
    body, dev, onk, theta = setup_pair(seed=2)
    plain = pd.NewtonKrylov(steps=1, tol=1e-8, tol_mode="relative", frechet="forward",
                            gmres_restart=8, gmres_maxiter=400, maxiter=3,
                            preconditioner="block_jacobi")
    P.collect(dev, plain, 1, 3)
    assert nkm.recorded(dev) == 3
    slow = [nkm.recorded_vector(dev, k).astype(np.float64) for k in range(3)]
    rng = np.random.default_rng(6)
    fast = P.random_probes(onk.cmask, 2, rng)
    net = P.BlockPreconditionerNet(theta)
    loss, grad = net.spectral_grad(dev, [0, 1, 2], fast, tau=0.3, weight=4.0)
    # the oracle at the device body's state (the solve moved it)
    u = dev.field("displacement").T
    onk.ob.u[:] = u
    onk.ob.pos[:] = onk.ob.X + u
    Pb = onk.bj_blocks().astype(np.float32).astype(np.float64)
    x = M.features(onk)
    g = M.Graph(onk.ob)
    act = M.forward(theta, x, g)
    Lo, dD = M.spectral_loss_and_dD(onk, Pb, act["D"].astype(np.float64), slow,
                                    [f.astype(np.float64) for f in fast], 0.3, 4.0)
    go = M.backward(theta, act, dD.astype(np.float32), g)
    assert abs(loss - Lo) <= 1e-3 * abs(Lo)
    assert rel(grad, go) <= 3e-2


def test_training_moves_the_fast_end_and_beats_block_jacobi():
    body = small_beam(nx=48, ny=10, nz=8, load=-0.1e-3)
    dev = pd.DeviceBody(body, precision="fp64")
    plain = pd.NewtonKrylov(steps=2, tol=1e-8, tol_mode="relative", frechet="forward",
                            gmres_restart=20, gmres_maxiter=5000, maxiter=20,
                            preconditioner="block_jacobi")
    assert P.collect(dev, plain, 2, 64) > 8
    net = P.BlockPreconditionerNet(seed=0)
    lam0 = max(P.rayleigh(dev, q, learned=False) for q in P.top_modes(dev, 2, iters=40))
    P.train(net, [dev], steps=60, lr=2e-3, refresh=5)
    net.infer(dev)
    lam1 = max(P.rayleigh(dev, q) for q in P.top_modes(dev, 2, iters=40, learned=True))
    # the trained scale lifts the preconditioned spectrum, its top held near tau = 1.85 < 2
    assert lam0 < lam1 < 2.0
    its = {}
    for pc in ("block_jacobi", "block_poly", "learned_poly"):
        nk = pd.NewtonKrylov(steps=2, tol=1e-8, tol_mode="relative", frechet="forward",
                             gmres_restart=20, gmres_maxiter=5000, maxiter=20, preconditioner=pc,
                             corrections=net)
        pd.submit(pd.Job(body, nk))
        assert all(s["converged"] for s in nk.stats)
        its[pc] = sum(s["gmres_iters"] for s in nk.stats)
    print("Krylov steps", its, "top eigenvalue", lam0, "->", lam1)
    assert its["learned_poly"] < its["block_jacobi"]
    assert its["learned_poly"] <= 1.05 * its["block_poly"]
