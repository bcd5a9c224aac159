"""numpy wrappers over the C-ABI (host buffers, synchronous), mirroring fysics.h.

Each wrapper allocates the output, calls the matching fy_* entry point of
libfysics_b200.so and raises FysicsError on a nonzero status -- the same contract as the
reference's int returns. Arrays are C-contiguous (nz, ny, nx), x fastest.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import Physics, check, check_void, load


def _ptr(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


def _c(a: np.ndarray, dtype) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=dtype)


def physics(delta_beta=1000.0, energy_kev=78.0, distance_mm=220.0, pixel_um=2.4,
            unsharp_sigma=1.2, unsharp_coeff=4.0, psf_sigma_vox=0.0,
            psf_sigma_z_vox=0.0) -> Physics:
    """fy_physics with the reference tests' default physics (test_fysics.c:229)."""
    return Physics(delta_beta, energy_kev, distance_mm, pixel_um, unsharp_sigma, unsharp_coeff,
                   psf_sigma_vox, psf_sigma_z_vox)


def u8_to_phys(u8: np.ndarray, f32_min: float, f32_max: float) -> np.ndarray:
    a = _c(u8, np.uint8)
    out = np.empty(a.shape, np.float32)
    load().fy_u8_to_phys(_ptr(a), _ptr(out), a.size, f32_min, f32_max)
    check_void("fy_u8_to_phys")
    return out


def phys_to_u8(v: np.ndarray, f32_min: float, f32_max: float) -> np.ndarray:
    a = _c(v, np.float32)
    out = np.empty(a.shape, np.uint8)
    load().fy_phys_to_u8(_ptr(a), _ptr(out), a.size, f32_min, f32_max)
    check_void("fy_phys_to_u8")
    return out


def u8_to_float(u8: np.ndarray) -> np.ndarray:
    a = _c(u8, np.uint8)
    out = np.empty(a.shape, np.float32)
    load().fy_u8_to_float(_ptr(a), _ptr(out), a.size)
    check_void("fy_u8_to_float")
    return out


def float_to_u8(v: np.ndarray) -> np.ndarray:
    a = _c(v, np.float32)
    out = np.empty(a.shape, np.uint8)
    load().fy_float_to_u8(_ptr(a), _ptr(out), a.size)
    check_void("fy_float_to_u8")
    return out


def deconvolve(vol: np.ndarray, p: Physics, reg: float = 0.0) -> np.ndarray:
    a = _c(vol, np.float32)
    out = np.empty_like(a)
    nz, ny, nx = a.shape
    check(load().fy_deconvolve(_ptr(a), _ptr(out), nz, ny, nx, C.byref(p), reg), "fy_deconvolve")
    return out


def deconvolve_matched(vol: np.ndarray, p: Physics, tikhonov: float = 0.0) -> np.ndarray:
    a = _c(vol, np.float32)
    out = np.empty_like(a)
    nz, ny, nx = a.shape
    check(load().fy_deconvolve_matched(_ptr(a), _ptr(out), nz, ny, nx, C.byref(p), tikhonov),
          "fy_deconvolve_matched")
    return out


def kernel_halo(p: Physics) -> int:
    return int(load().fy_kernel_halo(C.byref(p)))
