"""The CPU restatement of dynamic relaxation (oracle/dr.py), pinned on the reference's tests:
the density matrix and the two-step relaxation of test_dynamic_relaxation.jl:24-43, 59-82,
the damping clamp of :120-144, and the uniform-tension bands of
test_analytic_solutions.jl:78-84 and verification.jl:374-378. No GPU."""
import numpy as np
import pytest

import pdcuda as pd
from dr import OracleDR, density_matrix, finish_damping
from helpers import oracle_bcs, oracle_body
from test_nk_host import EBAR, FBAR, HBAR, LBAR, WBAR


def four_points(horizon_a=1.5):
    pos = np.array([[0.0, 1.0, 0.0, 0.0], [0.0, 0.0, 0.0, 1.0], [0.0, 0.0, 1.0, 0.0]])
    body = pd.Body(pd.BBMaterial(), pos, np.ones(4))
    pd.material(body, horizon=1.5, rho=8e-6, E=210e3)
    pd.point_set(body, "a", [0, 1])
    pd.material(body, "a", horizon=horizon_a, rho=7.8e-6, E=200e3)
    return body


def test_density_matrix_golden():
    lam = density_matrix(oracle_body(four_points()), 1.0)
    assert np.allclose(lam, [4.0e6, 4.0e6, 4.2e6, 4.2e6], rtol=1e-12)


def two_step_body():
    body = four_points(horizon_a=3.0)
    pd.forcedensity_bc(lambda p, t: 1e5 * p[0], body, "a", "x")
    return body


def test_two_relaxation_steps_golden():
    body = two_step_body()
    ob = oracle_body(body)
    dr = OracleDR(ob, 1.0)
    bcs = oracle_bcs(body, 1, 2, 1.0)
    dr.step(1, bcs)
    dr.step(2, bcs)
    assert ob.pos[1, 0] == pytest.approx(1.05, rel=1e-6)


def test_damping_clamp():
    assert finish_damping(-1.0, 2.0) == 0.0
    assert finish_damping(1.0, 0.0) == 0.0
    assert finish_damping(8.0, 1.0) == 1.9      # 2 sqrt(8) > 2 is clamped
    assert finish_damping(0.25, 1.0) == 1.0


def relaxation_bar(dx):
    """`relaxation_bar` of test_analytic_solutions.jl: CMaterial, epsilon_c = 1, left end held by
    zero velocity conditions, the force spread over the right layer."""
    pos, vol = pd.uniform_box(LBAR + 3 * dx, WBAR, HBAR, dx, center=(-1.5 * dx, 0, 0))
    body = pd.Body(pd.CMaterial(), pos, vol)
    pd.material(body, horizon=3.015 * dx, rho=7850.0, E=EBAR, nu=0.25, epsilon_c=1.0)
    pd.point_set(body, "left", where=lambda p: p[0] < -LBAR / 2)
    pd.point_set(body, "right", where=lambda p: p[0] > LBAR / 2 - dx)
    b_right = FBAR / vol[body.point_sets["right"]].sum()
    for d in ("x", "y", "z"):
        pd.velocity_bc(lambda t: 0.0, body, "left", d)
    pd.forcedensity_bc(lambda t: b_right, body, "right", "x")
    return body


def elongation_error(u, body):
    right = body.point_sets["right"]
    exact = FBAR / (EBAR * WBAR * HBAR) * LBAR
    return abs(u[right, 0].mean() - exact) / exact


def test_oracle_uniform_tension_band():
    body = relaxation_bar(1 / 30)
    ob = oracle_body(body)
    dr = OracleDR(ob, 1.0)
    n = 2000
    bcs = oracle_bcs(body, 1, n, 1.0)
    ob.force_density(0.0, 1.0)
    errs = {}
    for k in range(1, n + 1):
        dr.step(k, bcs)
        if k in (1000, 2000):
            errs[k] = elongation_error(ob.u, body)
    # the reference's bands: < 5 % after 1000 steps (per-commit test), < 2 % after 2000 steps
    # (verification suite: "2000 steps give 0.5 %"; this restatement: 3.0 % and 0.51 %)
    assert errs[1000] < 0.05 and errs[2000] < 0.02
