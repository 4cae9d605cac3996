"""pdcuda -- B200 (sm_100a) engine for Peridynamics.jl's explicit-dynamics hot path.

The user surface mirrors the reference's (``Body``, ``material!``, ``velocity_bc!``,
``VelocityVerlet``, ``Job``, ``submit``; Julia's trailing ``!`` dropped) and drives the C ABI
of ``libpdcuda.so`` (include/pdcuda.h). The bond loops, failure, damage and the Velocity
Verlet update run as CUDA kernels; there is no CPU fallback.
"""
from ._lib import NaNError, PDCudaError, lib, LIB_PATH, EXPORTS
from .materials import (BBMaterial, OSBMaterial, CMaterial, SaintVenantKirchhoff, NeoHooke,
                        NeoHookePenalty, ZEMSilling, ZEMWan, CriticalStretch, NoCorrection,
                        EnergySurfaceCorrection,
                        const_one_kernel, linear_kernel, cubic_b_spline_kernel,
                        point_parameters, PointParameters)
from .body import (Body, point_set, material, failure_permit, no_failure, velocity_bc,
                   forcedensity_bc, displacement_bc, velocity_databc, forcedensity_databc,
                   velocity_ic, precrack, uniform_box, get_dim)
from .solver import VelocityVerlet, Job, DeviceBody, submit
from .ensemble import Ensemble
from .newton_krylov import NewtonKrylov
from .dynamic_relaxation import DynamicRelaxation
from . import mpnn
from ._lib import NotConvergedError

__version__ = "0.1.0"
