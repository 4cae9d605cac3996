"""Shared builders of the tests: the same bodies for the oracle and the device."""
import numpy as np

import pdcuda as pd

from bench import make_plate as plate_body  # noqa: F401  (the mode-I plate of the benchmarks)
from twin import MAT_ORACLE, oracle_bcs, oracle_body, oracle_params  # noqa: F401


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
