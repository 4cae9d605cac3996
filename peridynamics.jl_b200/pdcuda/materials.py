"""Materials, constitutive models, influence functions and material parameters.

Host-side restatement of the parameter logic of Peridynamics.jl that feeds the device
parameter table: ``material!`` keyword handling (src/physics/material_parameters.jl:64-231),
the critical stretch (src/physics/fracture.jl:110-175), the bond constant
(src/physics/bond_based.jl:86-113) and the material types (bond_based.jl:74-84,
ordinary_state_based.jl:82-94, correspondence.jl:111-128).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

from . import _lib as L


# ----------------------------------------------------------------------------------------
# influence functions (src/discretization/kernels.jl:10-52)
# ----------------------------------------------------------------------------------------
def const_one_kernel(delta, L_):
    return 1.0


def linear_kernel(delta, L_):
    return delta / L_


def cubic_b_spline_kernel(delta, L_):
    xi = L_ / delta
    if 0 < xi <= 0.5:
        return 2 / 3 - 4 * xi ** 2 + 4 * xi ** 3
    if 0.5 < xi <= 1:
        return 4 / 3 - 4 * xi + 4 * xi ** 2 - 4 / 3 * xi ** 3
    return 0.0


_KERNEL_IDS = {const_one_kernel: L.KERNEL_CONST_ONE, linear_kernel: L.KERNEL_LINEAR,
               cubic_b_spline_kernel: L.KERNEL_CUBIC_BSPLINE}


# ----------------------------------------------------------------------------------------
# damage model, constitutive models, zero-energy-mode stabilisation
# ----------------------------------------------------------------------------------------
class CriticalStretch:
    """Bond failure when the stretch exceeds the critical stretch (fracture.jl:10)."""

    def __repr__(self):
        return "CriticalStretch()"


class SaintVenantKirchhoff:
    """constitutive_models.jl:33-48"""
    id = L.CM_SVK


class NeoHooke:
    """constitutive_models.jl:167-185"""
    id = L.CM_NEOHOOKE


class NeoHookePenalty:
    """constitutive_models.jl:231-255"""
    id = L.CM_NEOHOOKE_PENALTY


@dataclass
class ZEMSilling:
    """Zero-energy mode stabilisation of Silling (zem_stabilization.jl:16-21)."""
    Cs: float = 0.5
    id = L.ZEM_SILLING


class ZEMWan:
    """Zero-energy mode stabilisation of Wan et al. (2019) (zem_stabilization.jl:23-42): the
    stabilising stiffness of every point is C : K^-1, the Hooke tensor of its parameter set
    contracted with its inverse shape tensor; no stabilisation parameter."""
    id = L.ZEM_WAN

    def __repr__(self):
        return "ZEMWan()"


# ----------------------------------------------------------------------------------------
# material types
# ----------------------------------------------------------------------------------------
class AbstractMaterial:
    material_id = -1
    kernel = linear_kernel
    model = None
    zem = None
    maxdmg = 0.85

    @property
    def kernel_id(self):
        try:
            return _KERNEL_IDS[self.kernel]
        except KeyError as e:
            raise ValueError("only const_one_kernel, linear_kernel and cubic_b_spline_kernel "
                             "are available on the device") from e


class NoCorrection:
    """No surface correction (bond_system_corrections.jl:1-10): every bond factor is 1."""

    def __repr__(self):
        return "NoCorrection"


class EnergySurfaceCorrection:
    """The energy based surface correction of Le and Bobaru (2018)
    (bond_system_corrections.jl:50-64): per-bond factors from the strain energy of every
    point under uniform stretches, computed when the body is set up on the device."""

    def __repr__(self):
        return "EnergySurfaceCorrection"


def _correction(c):
    if c is None or c is NoCorrection or isinstance(c, NoCorrection):
        return NoCorrection()
    if c is EnergySurfaceCorrection or isinstance(c, EnergySurfaceCorrection):
        return EnergySurfaceCorrection()
    raise ValueError("correction must be NoCorrection or EnergySurfaceCorrection")


class BBMaterial(AbstractMaterial):
    """Bond-based peridynamics (bond_based.jl:74-84); nu is fixed to 1/4. correction: the
    material's type parameter of the reference (BBMaterial{EnergySurfaceCorrection}())."""
    material_id = L.MAT_BB

    def __init__(self, dmgmodel=None, correction=None):
        self.dmgmodel = dmgmodel or CriticalStretch()
        self.kernel = const_one_kernel
        self.correction = _correction(correction)

    def __repr__(self):
        return f"BBMaterial{{{self.correction!r}}}()"


class OSBMaterial(AbstractMaterial):
    """Ordinary state-based peridynamics (ordinary_state_based.jl:82-94); correction as for
    BBMaterial."""
    material_id = L.MAT_OSB

    def __init__(self, kernel=linear_kernel, dmgmodel=None, correction=None):
        self.kernel = kernel
        self.dmgmodel = dmgmodel or CriticalStretch()
        self.correction = _correction(correction)

    def __repr__(self):
        return f"OSBMaterial{{{self.correction!r}}}(dmgmodel=CriticalStretch())"


class CMaterial(AbstractMaterial):
    """Correspondence formulation (correspondence.jl:111-128) with ZEMSilling or ZEMWan."""
    material_id = L.MAT_CMAT

    def __init__(self, kernel=linear_kernel, model=None, zem=None, dmgmodel=None, maxdmg=0.85):
        self.kernel = kernel
        self.model = model if model is not None else SaintVenantKirchhoff()
        self.zem = zem if zem is not None else ZEMSilling()
        if not isinstance(self.zem, (ZEMSilling, ZEMWan)):
            raise ValueError("zem must be ZEMSilling(Cs) or ZEMWan()")
        self.dmgmodel = dmgmodel or CriticalStretch()
        self.maxdmg = float(maxdmg)

    def __repr__(self):
        return (f"CMaterial(model={type(self.model).__name__}, zem={self.zem!r}, "
                f"maxdmg={self.maxdmg})")


# ----------------------------------------------------------------------------------------
# material parameters
# ----------------------------------------------------------------------------------------
@dataclass
class PointParameters:
    """StandardPointParameters (src/core/parameters.jl:107-125)."""
    delta: float
    rho: float
    E: float
    nu: float
    G: float
    K: float
    lambda_: float
    mu: float
    Gc: float
    epsilon_c: float
    bc: float

    def to_c(self):
        return L.PointParams(self.delta, self.rho, self.E, self.nu, self.G, self.K, self.lambda_,
                             self.mu, self.Gc, self.epsilon_c, self.bc)

    @property
    def has_fracture(self):
        # has_fracture (fracture.jl:169-175)
        eps = 2.220446049250313e-16
        return not (abs(self.Gc) <= eps or abs(self.epsilon_c) <= eps)


_NAN = float("nan")
ALLOWED_KWARGS = {"horizon", "rho", "E", "nu", "G", "K", "lambda", "mu", "Gc", "epsilon_c"}


def _isapprox(a, b):
    return abs(a - b) <= 1.4901161193847656e-8 * max(abs(a), abs(b))


def _fin(x):
    return x is not None and math.isfinite(x)


def _given(kw, key):
    return float(kw[key]) if key in kw else _NAN


def elastic_parameters(kw):
    """get_given_elastic_params, check_elastic_params and get_E_and_nu
    (material_parameters.jl:118-231)."""
    E, nu, G, K = (_given(kw, k) for k in ("E", "nu", "G", "K"))
    lam, mu = _given(kw, "lambda"), _given(kw, "mu")
    if _fin(E) and E <= 0:
        raise ValueError("`E` should be larger than zero!")
    if _fin(nu) and nu <= 0:
        raise ValueError("`nu` should be larger than zero!")
    if _fin(nu) and nu >= 1:
        raise ValueError("too high value of `nu`! Condition: 0 < `nu` ≤ 1")
    if _fin(G) and G <= 0:
        raise ValueError("`G` should be larger than zero!")
    if _fin(K) and K <= 0:
        raise ValueError("`K` should be larger than zero!")
    if _fin(mu) and mu <= 0:
        raise ValueError("`μ` should be larger than zero!")
    nfin = sum(_fin(x) for x in (E, nu, G, K, lam, mu))
    if _fin(G) and _fin(mu):
        raise ValueError("`G` and `μ` are defined! Please define either `G` or `μ`!")
    if nfin < 2:
        raise ValueError("Not enough material parameters defined!")
    if nfin > 2:
        raise ValueError("Too many material parameters defined!")
    if _fin(E) and _fin(nu):
        pass
    elif _fin(E) and _fin(G):
        nu = E / (2 * G) - 1
    elif _fin(E) and _fin(K):
        nu = (3 * K - E) / (6 * K)
    elif _fin(E) and _fin(lam):
        nu = (-(E + lam) + math.sqrt((E + lam) ** 2 + 8 * lam ** 2)) / (4 * lam)
    elif _fin(E) and _fin(mu):
        nu = E / (2 * mu) - 1
    elif _fin(nu) and _fin(G):
        E = 2 * G * (1 + nu)
    elif _fin(nu) and _fin(K):
        E = 3 * K * (1 - 2 * nu)
    elif _fin(nu) and _fin(lam):
        E = (lam * (1 + nu) * (1 - 2 * nu)) / nu
    elif _fin(nu) and _fin(mu):
        E = 2 * mu * (1 + nu)
    elif _fin(G) and _fin(K):
        E = 9 * K * G / (3 * K + G)
        nu = (3 * K - 2 * G) / (2 * (3 * K + G))
    elif _fin(G) and _fin(lam):
        E = G * (3 * lam + 2 * G) / (lam + G)
        nu = lam / (2 * (lam + G))
    elif _fin(K) and _fin(lam):
        E = 9 * K * (K - lam) / (3 * K - lam)
        nu = lam / (3 * K - lam)
    elif _fin(K) and _fin(mu):
        E = 9 * K * mu / (3 * K + mu)
        nu = (3 * K - 2 * mu) / (2 * (3 * K + mu))
    elif _fin(lam) and _fin(mu):
        E = mu * (3 * lam + 2 * mu) / (lam + mu)
        nu = lam / (2 * (lam + mu))
    Gm = E / (2 * (1 + nu))
    Km = E / (3 * (1 - 2 * nu))
    lm = E * nu / ((1 + nu) * (1 - 2 * nu))
    return E, nu, Gm, Km, lm, Gm


def point_parameters(mat, **kw):
    """get_point_params of the material (bond_based.jl:86-113, correspondence.jl:163-169)."""
    unknown = set(kw) - ALLOWED_KWARGS
    if unknown:
        raise ValueError(f"keyword(s) {sorted(unknown)} not allowed for {type(mat).__name__}")
    if "horizon" not in kw:
        raise TypeError("UndefKeywordError: keyword argument `horizon` not assigned")
    if "rho" not in kw:
        raise TypeError("UndefKeywordError: keyword argument `rho` not assigned")
    delta = float(kw["horizon"])
    if delta <= 0:
        raise ValueError("`horizon` should be larger than zero!")
    rho = float(kw["rho"])
    if rho <= 0:
        raise ValueError("`rho` should be larger than zero!")
    kw = dict(kw)
    if isinstance(mat, BBMaterial):
        nu = _given(kw, "nu")
        nfin = sum(_fin(_given(kw, k)) for k in ("E", "nu", "G", "K", "lambda", "mu"))
        if _fin(nu) and not _isapprox(nu, 0.25):
            raise ValueError("Bond-based peridynamics has a limitation on the Poisson's ratio!\n"
                             "With BBMaterial, no other values than nu=0.25 are allowed!")
        if not _fin(nu) and nfin == 1:
            kw["nu"] = 0.25
    E, nu, G, K, lam, mu = elastic_parameters(kw)
    if isinstance(mat, BBMaterial) and not _isapprox(nu, 0.25):
        raise ValueError("Bond-based peridynamics has a limitation on the Poisson's ratio!\n"
                         "The submitted parameter combination results in an illegal value for nu!")
    # get_frac_params (fracture.jl:110-130)
    has_gc, has_ec = "Gc" in kw, "epsilon_c" in kw
    if has_gc and not has_ec:
        Gc = float(kw["Gc"])
        epsc = math.sqrt(5.0 * Gc / (9.0 * K * delta))
    elif has_ec and not has_gc:
        epsc = float(kw["epsilon_c"])
        Gc = 9.0 / 5.0 * K * delta * epsc ** 2
    elif has_gc and has_ec:
        raise ValueError("insufficient keywords for calculation of fracture parameters!\n"
                         "Define either Gc or epsilon_c, not both!")
    else:
        Gc, epsc = 0.0, 0.0
    d2 = delta * delta
    bc = 18 * K / (math.pi * (d2 * d2))
    return PointParameters(delta, rho, E, nu, G, K, lam, mu, Gc, epsc, bc)
