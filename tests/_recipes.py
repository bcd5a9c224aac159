"""Seeded input recipes of the reference's own tests (tests/test_fysics.c), in numpy.

The reference synthesises every test input in-test from 32-bit LCGs; these functions
produce the same volumes so that the reference's tolerances and known answers can be
applied to the oracle and to the GPU path. The LCG stream x_{k+1} = a*x_k + c (mod 2^32)
is generated in closed form: x_k = a^k x_0 + c*(1 + a + ... + a^(k-1)), with the powers
and their prefix sums taken modulo 2^64 by numpy's wrapping uint64 arithmetic (2^32
divides 2^64, so the low 32 bits are exact).
"""
from __future__ import annotations

import numpy as np

M32 = np.uint64(0xFFFFFFFF)


def lcg(seed: int, a: int, c: int, n: int) -> np.ndarray:
    """x_1..x_n of x_{k+1} = a*x_k + c mod 2^32 (as uint64 in [0, 2^32))."""
    with np.errstate(over="ignore"):
        pw = np.cumprod(np.full(n, a, dtype=np.uint64))                   # a^k, k = 1..n
        s = np.cumsum(np.concatenate([[np.uint64(1)], pw[:-1]]))           # 1 + ... + a^(k-1)
        x = pw * np.uint64(seed) + np.uint64(c) * s
    return x & M32


def numrec(seed: int, n: int) -> np.ndarray:
    """rng = rng*1664525u + 1013904223u (test_fysics.c:99 and others)."""
    return lcg(seed, 1664525, 1013904223, n)


def deconv_equivalence_input():
    """test_deconv_rfft_equivalence (test_fysics.c:218-228): 22x27x30, rng 99."""
    nz, ny, nx = 22, 27, 30
    r = numrec(99, nz * ny * nx)
    return (((r >> np.uint64(8)) & np.uint64(0xFFFF)).astype(np.float32) / np.float32(65535.0)).reshape(nz, ny, nx)


def guided_step_input():
    """test_guided_fast (test_fysics.c:92-103): 32^3 step edge + 0.05 LCG noise."""
    nz = ny = nx = 32
    r = numrec(12345, nz * ny * nx).reshape(nz, ny, nx)
    noise = ((r >> np.uint64(8)) & np.uint64(0xFFFF)).astype(np.float32) / np.float32(65535.0) - np.float32(0.5)
    sig = np.where(np.arange(nx) < nx // 2, np.float32(0.3), np.float32(0.7)).astype(np.float32)
    return (sig[None, None, :] + np.float32(0.05) * noise).astype(np.float32)


def noise_input(sigma: float, seed: int):
    """test_estimate_noise (test_fysics.c:381-397): 48^3 smooth signal + LCG Box-Muller noise."""
    nz = ny = nx = 48
    r = numrec(seed, 2 * nz * ny * nx).reshape(nz, ny, nx, 2)
    u1 = ((r[..., 0] >> np.uint64(8)) & np.uint64(0xFFFFFF)).astype(np.float64) / float(0x1000000)
    u2 = ((r[..., 1] >> np.uint64(8)) & np.uint64(0xFFFFFF)).astype(np.float64) / float(0x1000000)
    u1 = np.maximum(u1, 1e-9)
    g0 = np.sqrt(-2 * np.log(u1)) * np.cos(6.283185307 * u2)
    x = np.arange(nx)[None, None, :]
    y = np.arange(ny)[None, :, None]
    s = 0.5 + 0.3 * np.sin(x * 0.10) * np.cos(y * 0.09)
    return (s + sigma * g0).astype(np.float32)


def dering_input():
    """test_dering (test_fysics.c:121-142): 32x256x256 u8 spiral + rings at r=60 (+10)
    and r=110 (-8) + LCG noise; returns (vol_u8, cy, cx)."""
    nz, ny, nx = 32, 256, 256
    cy = cx = 127.5
    y = np.arange(ny, dtype=np.float64)[:, None] - cy
    x = np.arange(nx, dtype=np.float64)[None, :] - cx
    r = np.sqrt(y * y + x * x)
    th = np.arctan2(y, x)
    v = 128 + 30 * np.cos(2 * np.pi * (r - 192 * th / (2 * np.pi)) / 24)
    v = v + 10 * np.exp(-(r - 60) ** 2 / (2 * 0.8 * 0.8)) - 8 * np.exp(-(r - 110) ** 2 / (2 * 0.8 * 0.8))
    rng = numrec(777, nz * ny * nx).reshape(nz, ny, nx)
    v = v[None] + ((rng >> np.uint64(8)) & np.uint64(0xFF)).astype(np.float64) / 25.5 - 5.0
    v = np.clip(v, 1, 255)
    return v.astype(np.uint8), cy, cx


def fourier_shift(f: np.ndarray, s) -> np.ndarray:
    """Exact band-limited circular shift (test_fysics.c:580-605), in FP64."""
    nz, ny, nx = f.shape
    F = np.fft.fftn(f.astype(np.float64))
    kz = np.fft.fftfreq(nz) * nz
    ky = np.fft.fftfreq(ny) * ny
    kx = np.fft.fftfreq(nx) * nx
    # the reference's fftfreq keeps k = n/2 positive: (z <= n/2) ? z : z - n
    kz[nz // 2] = nz // 2; ky[ny // 2] = ny // 2; kx[nx // 2] = nx // 2
    ph = -2 * np.pi * (kz[:, None, None] * s[0] / nz + ky[None, :, None] * s[1] / ny + kx[None, None, :] * s[2] / nx)
    return np.real(np.fft.ifftn(F * np.exp(1j * ph))).astype(np.float32)


def phasecorr_texture():
    """test_phase_correlate_subvoxel (test_fysics.c:895-905): 32^3 LCG texture, 1-2-1 in x."""
    n = 32
    seed = lcg(12345, 1103515245, 12345, n ** 3)
    f = (((seed >> np.uint64(9)) & np.uint64(8191)).astype(np.float32) / np.float32(8191.0)).reshape(n, n, n)
    return ((np.roll(f, 1, axis=2) + 2 * f + np.roll(f, -1, axis=2)) / 4).astype(np.float32)


PHASECORR_CASES = [(0.5, -0.25, 0.0), (0.33, 0.66, -0.4), (-0.7, 0.2, 0.85)]   # test_fysics.c:907
