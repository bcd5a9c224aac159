"""Radial eps model (pipeline.c:851-891) pinned to the reference's own calibration.

The reference fits fn(r) = a + b*r inside fy_calibrate (fysics.h:499), over (radius, flat
noise floor) samples of pass 1: the central 128^3 sub-block of every sampled 256^3 tile
with >= 60% nonzero voxels, the floor fy_flat_noise(u8/255, blk 8) and the radius of the
sub-block centre from the rotation axis (pipeline.c:704-770). Here the reference runs
fy_calibrate on a local zarr volume whose noise grows with the radius, and the same samples
are rebuilt from the public fy_flat_noise on the same sub-blocks; then
  - the FP64 oracle's fit (o64_fit_radial_eps, o64_median_floor) must give the reference's
    have_eps_r, eps_fn_a, eps_fn_b, eps_fn_med and guided_eps (CPU);
  - the product library's floors (fy_flat_noise on the GPU) and fit (fy_fit_radial_eps,
    one FP64 CTA) must give them too (GPU).
The reference sums its samples in the order its OpenMP workers finish, so a and b are held
to 1e-9 relative; the median is an order statistic of identical floors and must be equal.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from oracle import o64, p
from tests._zarr import write_zarr

needs_ref = pytest.mark.skipif(not oracle.have_ref(), reason="reference library not built")

SHAPE = (128, 512, 1024)             # 2 x 4 tiles of 256^2 in (y, x): 8 samples, the fit's minimum


def volume(kind, seed=5):
    nz, ny, nx = SHAPE
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:ny, 0:nx]
    r = np.hypot(yy - (ny - 1) / 2, xx - (nx - 1) / 2)
    sd = 2.0 + 0.012 * r if kind == "rising" else np.full(r.shape, 3.0)
    vol = np.empty(SHAPE, np.uint8)
    for z in range(nz):
        vol[z] = np.clip(np.rint(120 + sd * rng.standard_normal((ny, nx))), 1, 255)
    return vol


def samples(vol, flat_noise):
    """(radii, floors) of the sampled sub-blocks, in tile order (pipeline.c:704-770)."""
    nz, ny, nx = vol.shape
    ecy, ecx = (ny - 1) / 2.0, (nx - 1) / 2.0
    rads, floors = [], []
    for z0 in range(0, nz, 256):
        for y0 in range(0, ny, 256):
            for x0 in range(0, nx, 256):
                dz, dy, dx = min(256, nz - z0), min(256, ny - y0), min(256, nx - x0)
                sdz, sdy, sdx = min(128, dz), min(128, dy), min(128, dx)
                oz, oy, ox = (dz - sdz) // 2, (dy - sdy) // 2, (dx - sdx) // 2
                sub = vol[z0 + oz:z0 + oz + sdz, y0 + oy:y0 + oy + sdy, x0 + ox:x0 + ox + sdx]
                if np.count_nonzero(sub) / sub.size < 0.6:
                    continue
                sf = np.ascontiguousarray(sub.astype(np.float32) * np.float32(1.0 / 255.0))
                fn = flat_noise(sf)
                if fn > 0:
                    ry, rx = y0 + oy + sdy / 2.0 - ecy, x0 + ox + sdx / 2.0 - ecx
                    rads.append(np.sqrt(ry * ry + rx * rx))
                    floors.append(fn)
    return np.array(rads), np.array(floors)


def reference_calibration(tmp_path, vol):
    root = write_zarr(tmp_path / "v.zarr", vol, (128, 128, 128))
    cfg = oracle.ref_pipeline_cfg(oracle.pipeline_defaults())
    assert oracle.ref().fy_calibrate(str(root).encode(), C.byref(cfg), 128, 0) == 0
    return cfg


def close(x, y, rel=1e-9):
    return abs(x - y) <= rel * max(abs(y), 1e-300)


@needs_ref
@pytest.mark.parametrize("kind", ["rising", "flat"])
def test_oracle_fit_equals_reference_calibration(tmp_path, kind):
    vol = volume(kind)
    cfg = reference_calibration(tmp_path, vol)
    L = oracle.ref()
    rads, floors = samples(vol, lambda sf: L.fy_flat_noise(p(sf), *sf.shape, 8))
    assert rads.size == 8
    a, b, cc = C.c_double(), C.c_double(), C.c_double()
    have = o64().o64_fit_radial_eps(p(rads), p(floors), rads.size, C.byref(a), C.byref(b), C.byref(cc))
    assert have == cfg.have_eps_r == (1 if kind == "rising" else 0)
    if have:
        assert close(a.value, cfg.eps_fn_a) and close(b.value, cfg.eps_fn_b)
    med = o64().o64_median_floor(p(floors.copy()), floors.size)
    assert med == cfg.eps_fn_med
    assert close((4.2 * med) ** 2, cfg.guided_eps, 1e-15)


@needs_ref
@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["rising", "flat"])
def test_gpu_floors_and_fit_equal_reference_calibration(gpu, tmp_path, kind):
    vol = volume(kind)
    cfg = reference_calibration(tmp_path, vol)
    lib = gpu.load()
    rads, floors = samples(vol, lambda sf: lib.fy_flat_noise(p(sf), *sf.shape, 8))
    assert rads.size == 8
    fit = gpu.RadialEps()
    assert lib.fy_fit_radial_eps(p(rads), p(floors), rads.size, 0.0, C.byref(fit)) == 0, lib.fy_gpu_last_error()
    assert fit.have == cfg.have_eps_r
    if fit.have:
        assert close(fit.a, cfg.eps_fn_a) and close(fit.b, cfg.eps_fn_b)
    assert close(fit.median, cfg.eps_fn_med)
    assert close(fit.guided_eps, cfg.guided_eps)
