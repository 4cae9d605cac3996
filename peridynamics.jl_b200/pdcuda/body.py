"""Body, point sets, conditions and pre-cracks: the reference's setup surface.

Mirrors src/discretization/body.jl:83-124 (Body), point_sets.jl:73-135 (point_set!),
point_generators.jl:45-60 (uniform_box), physics/material_parameters.jl:64-84 (material!),
physics/boundary_conditions.jl:422-688 (velocity_bc!, forcedensity_bc!, displacement_bc!,
velocity_databc!), physics/initial_conditions.jl:180-195 (velocity_ic!),
discretization/predefined_cracks.jl:106-112 (precrack!) and physics/fracture.jl:38-96
(failure_permit!, no_failure!).

Positions follow the reference's 3 x N convention at the interface (``position[:, i]`` is
point i) and are stored as (N, 3) C-contiguous arrays, which is the same memory layout.
"""
from __future__ import annotations

import inspect

import numpy as np

from .materials import point_parameters, AbstractMaterial

_DIMS = {"x": 0, "y": 1, "z": 2, 1: 0, 2: 1, 3: 2}


def get_dim(dim):
    """get_dim (boundary_conditions.jl:257-268): 1-based integer or :x/:y/:z -> 0-based."""
    if isinstance(dim, str) and dim.startswith(":"):
        dim = dim[1:]
    if isinstance(dim, (bool, np.bool_)) or dim not in _DIMS:
        raise ValueError(f"unknown dimension `{dim}`!\nThe dimension should either be a Symbol "
                         "or Integer indicating the direction of the condition!")
    return _DIMS[dim]


def uniform_box(lx, ly, lz, dx, center=(0.0, 0.0, 0.0)):
    """Regular lattice of a box (point_generators.jl:45-60): x fastest, then y, then z,
    centred on ``center``. Coordinates are (k - (n - 1) / 2) * dx + center per axis.
    Returns (position 3 x N, volume N)."""
    def axis(l):
        n = int(round(l / dx))
        return (np.arange(n, dtype=np.float64) - (n - 1) / 2.0) * dx
    gx, gy, gz = axis(lx), axis(ly), axis(lz)
    Z, Y, X = np.meshgrid(gz, gy, gx, indexing="ij")
    pos = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=0)
    for k in range(3):
        if abs(center[k]) > 2.220446049250313e-16:
            pos[k] += center[k]
    vol = np.full(pos.shape[1], dx ** 3)
    return pos, vol


def _condition_kind(f):
    """check_boundary_condition_function (boundary_conditions.jl:336-356): by argument names."""
    try:
        names = list(inspect.signature(f).parameters)
    except (TypeError, ValueError):
        names = []
    if names == ["t"]:
        return "sdbc"
    if names == ["p"]:
        return "psdbc"
    if names == ["p", "t"]:
        return "pdsdbc"
    raise ValueError("wrong arguments or argument names for condition function!\n"
                     "Boundary conditions support only three type of functions:\n"
                     "  `f(p, t)`\n  `f(t)`\n  `f(p)`\n")


class Condition:
    def __init__(self, kind, fun, field, point_set, dim, data=None):
        self.kind, self.fun, self.field, self.point_set, self.dim = kind, fun, field, point_set, dim
        self.data = data

    def __repr__(self):
        return f"{self.kind} on {self.field}: point_set={self.point_set}, dim={self.dim + 1}"


class Body:
    """A peridynamic body (body.jl:83-124)."""

    def __init__(self, mat, position, volume):
        if not isinstance(mat, AbstractMaterial):
            raise TypeError("mat must be a material (BBMaterial, OSBMaterial, CMaterial)")
        position = np.asarray(position, dtype=np.float64)
        volume = np.asarray(volume, dtype=np.float64).ravel()
        n = volume.shape[0]
        if position.shape != (3, n):
            raise ValueError("dimension of position must be 3 x n_points matching the volume")
        self.mat = mat
        self.n_points = n
        self._pos = np.ascontiguousarray(position.T)  # (n, 3): the 3 x N column-major memory
        self.volume = np.ascontiguousarray(volume)
        self.fail_permit = np.ones(n, dtype=bool)
        self.point_sets = {"all_points": np.arange(n)}
        self.point_params = []
        self.params_map = np.zeros(n, dtype=np.int64)  # 1-based parameter id, 0 = none
        self.single_dim_bcs = []
        self.posdep_single_dim_bcs = []
        self.pos_single_dim_bcs = []
        self.data_bcs = []
        self.single_dim_ics = []
        self.posdep_single_dim_ics = []
        self.point_sets_precracks = []

    @property
    def position(self):
        """3 x N view of the reference positions."""
        return self._pos.T

    def __repr__(self):
        return f"{self.n_points}-point Body{{{type(self.mat).__name__}}}"

    def _check_set(self, name):
        if name not in self.point_sets:
            raise ValueError(f"there is no point set with name `{name}`!")
        return self.point_sets[name]


def point_set(body, name, points=None, *, where=None):
    """point_set! (point_sets.jl:73-92): by 0-based indices, a boolean mask, or a predicate
    ``where(p)`` on the 3-vector of a reference position (or vectorised over 3 x N)."""
    if callable(points) and where is None:
        points, where = None, points
    if name in body.point_sets:
        raise ValueError(f"there is already a point set with name {name}!")
    if where is not None:
        try:
            mask = np.asarray(where(body.position), dtype=bool)
            if mask.shape != (body.n_points,):
                raise ValueError
        except Exception:
            mask = np.array([bool(where(body._pos[i])) for i in range(body.n_points)])
        pts = np.nonzero(mask)[0]
    else:
        pts = np.asarray(points)
        if pts.dtype == bool:
            pts = np.nonzero(pts)[0]
        pts = pts.astype(np.int64).ravel()
        if pts.size and (pts.min() < 0 or pts.max() >= body.n_points):
            raise IndexError("point index out of bounds")
    body.point_sets[name] = pts


def material(body, set_name=None, **kwargs):
    """material! (material_parameters.jl:64-90)."""
    if set_name is None:
        body.point_params.clear()
        set_name = "all_points"
    pts = body._check_set(set_name)
    params = point_parameters(body.mat, **kwargs)
    body.point_params.append(params)
    body.params_map[pts] = len(body.point_params)
    body.fail_permit[pts] = params.has_fracture


def failure_permit(body, set_name, permit):
    """failure_permit! (fracture.jl:38-42)."""
    body.fail_permit[body._check_set(set_name)] = bool(permit)


def no_failure(body, set_name="all_points"):
    """no_failure! (fracture.jl:78-96)."""
    pts = body._check_set(set_name)
    if np.any(body.params_map[pts] == 0):
        raise ValueError(f'Not all points of point set ":{set_name}" have material parameters!')
    failure_permit(body, set_name, False)


def _check_conflict(body, new):
    """check_boundary_condition_conflicts (boundary_conditions.jl:285-334)."""
    for lst in (body.single_dim_bcs, body.posdep_single_dim_bcs, body.pos_single_dim_bcs,
                body.data_bcs):
        for c in lst:
            dims_a = c.dim if isinstance(c.dim, list) else [c.dim]
            dims_b = new.dim if isinstance(new.dim, list) else [new.dim]
            if c.field == new.field and set(dims_a) & set(dims_b):
                if np.intersect1d(body.point_sets[c.point_set],
                                  body.point_sets[new.point_set]).size:
                    raise ValueError("the specified condition conflicts with already existing "
                                     "conditions!")


def velocity_bc(f, body, set_name, dim):
    """velocity_bc! (boundary_conditions.jl:422-435): f(t) or f(p, t), writes velocity_half."""
    body._check_set(set_name)
    kind = _condition_kind(f)
    d = get_dim(dim)
    if kind == "sdbc":
        c = Condition("sdbc", f, "velocity_half", set_name, d)
        _check_conflict(body, c)
        body.single_dim_bcs.append(c)
    elif kind == "pdsdbc":
        c = Condition("pdsdbc", f, "velocity_half", set_name, d)
        _check_conflict(body, c)
        body.posdep_single_dim_bcs.append(c)
    else:
        raise ValueError("velocity_bc! takes f(t) or f(p, t)")


def forcedensity_bc(f, body, set_name, dim):
    """forcedensity_bc! (boundary_conditions.jl:559-575): f(t), f(p, t) or f(p) on b_ext."""
    body._check_set(set_name)
    kind = _condition_kind(f)
    d = get_dim(dim)
    c = Condition(kind, f, "b_ext", set_name, d)
    _check_conflict(body, c)
    {"sdbc": body.single_dim_bcs, "pdsdbc": body.posdep_single_dim_bcs,
     "psdbc": body.pos_single_dim_bcs}[kind].append(c)


def displacement_bc(f, body, set_name, dim):
    """displacement_bc! (boundary_conditions.jl:675-688): f(p), quasi-static solver only."""
    body._check_set(set_name)
    if _condition_kind(f) != "psdbc":
        raise ValueError("the function for a displacement boundary condition must be of the "
                         "form\n`f(p)`!")
    c = Condition("psdbc", f, "displacement", set_name, get_dim(dim))
    _check_conflict(body, c)
    body.pos_single_dim_bcs.append(c)


def velocity_databc(body, data, set_name, dims):
    """velocity_databc! (boundary_conditions.jl:482-490): data is len(dims) x n_points."""
    body._check_set(set_name)
    data = np.asarray(data, dtype=np.float64)
    if data.shape != (len(dims), body.n_points):
        raise ValueError("the data matrix must be length(dims) x n_points")
    ds = [get_dim(x) for x in dims]
    c = Condition("databc", None, "velocity_half", set_name, ds, data=data)
    _check_conflict(body, c)
    body.data_bcs.append(c)


def forcedensity_databc(body, data, set_name, dims):
    """forcedensity_databc! (boundary_conditions.jl:612-620)."""
    body._check_set(set_name)
    data = np.asarray(data, dtype=np.float64)
    if data.shape != (len(dims), body.n_points):
        raise ValueError("the data matrix must be length(dims) x n_points")
    c = Condition("databc", None, "b_ext", set_name, [get_dim(x) for x in dims], data=data)
    _check_conflict(body, c)
    body.data_bcs.append(c)


def velocity_ic(body_or_f, *args):
    """velocity_ic! (initial_conditions.jl:180-195): velocity_ic(body, set, dim, value) or
    velocity_ic(f, body, set, dim) with f(p)."""
    if callable(body_or_f):
        f, (body, set_name, dim) = body_or_f, args
        if _condition_kind(f) != "psdbc":
            raise ValueError("wrong arguments for position dependent initial condition "
                             "function!")
        body._check_set(set_name)
        body.posdep_single_dim_ics.append(Condition("pdic", f, "velocity", set_name, get_dim(dim)))
    else:
        body, (set_name, dim, value) = body_or_f, args
        body._check_set(set_name)
        body.single_dim_ics.append(Condition("ic", float(value), "velocity", set_name,
                                             get_dim(dim)))


def precrack(body, set_a, set_b, update_dmg=True):
    """precrack! (predefined_cracks.jl:106-112)."""
    a, b = body._check_set(set_a), body._check_set(set_b)
    if np.intersect1d(a, b).size:
        raise ValueError(f"point set `:{set_a}` and `:{set_b}` intersect!")
    body.point_sets_precracks.append((set_a, set_b, not update_dmg))
