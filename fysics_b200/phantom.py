"""Seeded synthetic scroll phantoms for the benchmark and parity workloads.

Recipe (the benchmark configurations' phantom; no real data is involved):
  * attenuation mu = 0.15 + 0.6 * sum_k exp(-d_k^2 / (2*1.5^2)) over 10 warped sheets
    z = z_k + A*sin(2*pi*x/Lx + phi)*cos(2*pi*y/Ly), z_k evenly spaced, A ~ U[2,8] px,
    Lx, Ly ~ U[40,160] px, phi ~ U[0, 2*pi); d_k is the vertical distance to sheet k;
  * 20 spherical voids of radius U[2,6] px with mu = 0.02;
  * forward blur by H(f) = T_paganin(f) * U_unsharp(f) (FP64, the same transfer the
    deconvolution inverts), optionally with the z frequency scaled by sigma_z/sigma_xy;
  * Poisson-Gaussian noise, var = g*I + b;
  * window [lo, hi] -> u8 = clip(round(255*(v - lo)/(hi - lo)));
  * optional ring artefacts: concentric 1-px annuli about an axis, +-amp u8.
Everything is generated with torch (CUDA when available) from a master seed; sub-seeds
for batches come from SplitMix64.
"""
from __future__ import annotations

import math

import numpy as np
import torch

MASK64 = (1 << 64) - 1


def splitmix64(x: int) -> int:
    x = (x + 0x9E3779B97F4A7C15) & MASK64
    z = x
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
    return z ^ (z >> 31)


def sub_seed(master: int, i: int) -> int:
    return splitmix64(master * 0x100000001B3 + i) & 0x7FFFFFFF


def transfer(fz2, fy2, fx2, delta_beta, energy_kev, distance_mm, pixel_um, unsharp_sigma, unsharp_coeff,
             fz2_scale=1.0):
    """H = max(T*U, 1e-4) on a frequency grid (cycles/voxel squared per axis)."""
    f2 = fz2 * fz2_scale + fy2 + fx2
    lam = 1.23984199e-3 / energy_kev
    dist = distance_mm * 1000.0
    px = pixel_um * 1000.0 if 0.0 < pixel_um < 0.1 else pixel_um
    T = 1.0 / (1.0 + delta_beta * lam * dist * math.pi * f2 / (px * px))
    U = 1.0 + unsharp_coeff * (1.0 - torch.exp(-2.0 * math.pi ** 2 * unsharp_sigma ** 2 * f2))
    return torch.clamp(T * U, min=1e-4)


def phantom(shape, seed=0, delta_beta=500.0, energy_kev=110.0, distance_mm=1200.0, pixel_um=7.91,
            unsharp_sigma=0.8, unsharp_coeff=0.5, fz2_scale=1.0, g=0.002, b=1e-4, window=(0.0, 1.0),
            rings=0, ring_axis=None, ring_amp=3.0, device=None, return_float=False):
    """u8 phantom volume (numpy uint8 on CPU, or a torch uint8 tensor on `device`)."""
    nz, ny, nx = shape
    dev = torch.device(device or ("cuda" if torch.cuda.is_available() else "cpu"))
    rng = np.random.default_rng(seed)
    gen = torch.Generator(device=dev).manual_seed(int(seed))
    z = torch.arange(nz, device=dev, dtype=torch.float64)[:, None, None]
    y = torch.arange(ny, device=dev, dtype=torch.float64)[None, :, None]
    x = torch.arange(nx, device=dev, dtype=torch.float64)[None, None, :]
    mu = torch.full(shape, 0.15, dtype=torch.float64, device=dev)
    zk = np.linspace(0, nz, 12)[1:-1]
    for k in range(10):
        A = rng.uniform(2, 8)
        Lx, Ly = rng.uniform(40, 160, 2)
        phi = rng.uniform(0, 2 * math.pi)
        surf = zk[k] + A * torch.sin(2 * math.pi * x / Lx + phi) * torch.cos(2 * math.pi * y / Ly)
        mu += 0.6 * torch.exp(-(z - surf) ** 2 / (2 * 1.5 ** 2))
    for _ in range(20):
        c = rng.uniform([0, 0, 0], [nz, ny, nx])
        r = rng.uniform(2, 6)
        inside = (z - c[0]) ** 2 + (y - c[1]) ** 2 + (x - c[2]) ** 2 < r * r
        mu = torch.where(inside, torch.full_like(mu, 0.02), mu)
    # forward blur by the reconstruction transfer
    fz = torch.fft.fftfreq(nz, device=dev, dtype=torch.float64)[:, None, None]
    fy = torch.fft.fftfreq(ny, device=dev, dtype=torch.float64)[None, :, None]
    fx = torch.fft.rfftfreq(nx, device=dev, dtype=torch.float64)[None, None, :]
    H = transfer(fz * fz, fy * fy, fx * fx, delta_beta, energy_kev, distance_mm, pixel_um, unsharp_sigma,
                 unsharp_coeff, fz2_scale)
    spec = torch.fft.rfftn(mu) * H
    del H
    I = torch.fft.irfftn(spec, s=shape)
    del spec
    noise = torch.randn(shape, generator=gen, device=dev, dtype=torch.float64)
    I = I + noise * torch.sqrt(torch.clamp(g * I + b, min=0.0))
    del noise
    lo, hi = window
    v = (I - lo) / (hi - lo) * 255.0
    if rings:
        cy, cx = ring_axis if ring_axis is not None else ((ny - 1) / 2.0, (nx - 1) / 2.0)
        rr = torch.sqrt((y - cy) ** 2 + (x - cx) ** 2)
        for _ in range(rings):
            R = rng.uniform(20, 250)
            amp = ring_amp if rng.uniform() < 0.5 else -ring_amp
            v = v + amp * (torch.abs(rr - R) < 0.5).to(torch.float64)
    if return_float:
        return I.float()
    u8 = torch.clamp(torch.round(v), 0, 255).to(torch.uint8)
    if device is None and dev.type == "cpu":
        return u8.numpy()
    return u8


# The workloads of the benchmark configurations (physics and sizes).
CONFIG1 = dict(shape=(128, 128, 128), delta_beta=500.0, energy_kev=110.0, distance_mm=1200.0, pixel_um=7.91,
               unsharp_sigma=0.8, unsharp_coeff=0.5, g=0.002, b=1e-4)
CONFIG2 = dict(shape=(512, 512, 512), delta_beta=500.0, energy_kev=110.0, distance_mm=1200.0, pixel_um=2.4,
               unsharp_sigma=0.8, unsharp_coeff=0.5, g=0.002, b=1e-4, sigma_ratio=1.17, rings=40)


def scroll_volume(shape, seed=0, specks_per_mvox=400, masked=True):
    """u8 volume for the per-tile export chain: noisy air (u8 ~ 22) around a cylindrical
    body of spiral papyrus wraps (sheets ~ 150, gaps ~ 70, thickness ~3 voxels), small
    bright specks in the air (1-27 voxels; the islands the despeckle removes) and an
    exactly-zero masked slab (the first tenth of y), so that the air-cut histogram has two
    modes and a valley. Generated plane by plane (numpy, seeded)."""
    nz, ny, nx = shape
    rng = np.random.default_rng(seed)
    cy, cx = (ny - 1) / 2 + rng.uniform(-3, 3), (nx - 1) / 2 + rng.uniform(-3, 3)
    y, x = np.mgrid[0:ny, 0:nx]
    r = np.hypot(y - cy, x - cx)
    turn = r / 4.5 + np.arctan2(y - cy, x - cx) / (2 * np.pi)
    body = r < 0.42 * min(ny, nx)
    out = np.empty(shape, np.uint8)
    for z in range(nz):
        sheet = np.cos(2 * np.pi * (turn + 0.15 * np.sin(z / 11.0))) > 0.2
        air = rng.normal(22, 6, (ny, nx))
        mat = np.where(sheet, rng.normal(150, 12, (ny, nx)), rng.normal(70, 10, (ny, nx)))
        out[z] = np.clip(np.rint(np.where(body, mat, air)), 0, 255).astype(np.uint8)
    for _ in range(int(specks_per_mvox * nz * ny * nx / 1e6)):
        c = rng.integers([0, 0, 0], [nz, ny, nx])
        if body[c[1], c[2]]:
            continue
        e = rng.integers(0, 3, 3)
        out[c[0]:c[0] + e[0] + 1, c[1]:c[1] + e[1] + 1, c[2]:c[2] + e[2] + 1] = np.uint8(
            np.clip(np.rint(rng.normal(150, 10)), 0, 255))
    if masked:
        out[:, : max(1, ny // 10), :] = 0
    return out
