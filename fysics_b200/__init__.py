"""fysics_b200 -- B200-native (sm_100a) drop-in for fysics' per-cube restoration path.

The product is the C-ABI library libfysics_b200.so (include/fysics_b200.h), which exports
the reference's fysics.h entry points for this path. This package is its host-side
mirror: `lib` is the ctypes handle with the exact C signatures, and the numpy wrappers
below call those entry points with the reference's argument meaning and error behaviour
(nonzero status -> FysicsError).
"""
from ._lib import (FY_OK, FY_EINVAL, FY_ENOMEM, FY_ECUDA, FY_ENODEV, FY_EUNSUPPORTED,
                   FY_ETIMEDOUT, FY_EBUSY, FY_EDEGENERATE, FY_EIO, AnisoResult, BatchCube, Dering, FysicsError, HistState,
                   NoiseModel,
                   Physics, PipelineCfg, RadialEps, Request, RequestResult, RestoreCfg, ServerCfg, ServerStats, SIGNATURES,
                   Zarr, check, check_void, load)
from .api import (deconvolve, deconvolve_matched, u8_to_phys, phys_to_u8, u8_to_float,
                  float_to_u8, kernel_halo, physics)

__all__ = [
    "Physics", "BatchCube", "NoiseModel", "Dering", "HistState", "PipelineCfg", "AnisoResult", "RadialEps", "RestoreCfg", "ServerCfg", "Request",
    "RequestResult", "ServerStats", "Zarr", "FysicsError", "SIGNATURES", "load", "check",
    "check_void", "deconvolve", "deconvolve_matched", "u8_to_phys", "phys_to_u8",
    "u8_to_float", "float_to_u8", "kernel_halo", "physics",
]
