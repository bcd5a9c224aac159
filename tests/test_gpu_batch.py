"""fy_gpu_restore_u8_batch: a batch of uneven device-resident cubes through the chain in one
call (deconvolutions on several streams, the two box passes as work-queue launches over all
cubes' tiles, the noise selection as one launch per step over all cubes).

Bar: every cube's output equals fy_gpu_restore_u8 on that cube alone, bit for bit (the same
tiles, chunks, kernels and exact order statistics; fy_gpu_restore_u8 itself is held to the
reference's chain in test_gpu_chain_parity.py). Configurations outside the batched form, and
cubes whose x extent is not a multiple of 4, run one by one and must match as well.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPES = [(40, 52, 64), (96, 96, 96), (33, 70, 48), (64, 128, 100), (20, 24, 28), (128, 64, 96), (48, 48, 48)]


def _cfg(fb):
    cfg = fb.RestoreCfg()
    fb.load().fy_restore_cfg_default(C.byref(cfg))
    cfg.deconv_kind, cfg.deconv_param = 1, 0.05
    cfg.noise_win, cfg.noise_flat_pct, cfg.noise_ref_intensity = 5, 10.0, 0.4
    cfg.guided_radius, cfg.guided_s = 2, 1
    return cfg


def _cubes(fb, shapes, seed=0):
    import torch
    import fysics_b200.phantom as ph
    rng = np.random.default_rng(seed)
    items, outs = [], []
    for i, shp in enumerate(shapes):
        db = float(rng.uniform(200, 1000))
        u = ph.phantom(shp, seed=seed + i, delta_beta=db, pixel_um=2.4, fz2_scale=1.17 ** 2, device="cuda")
        out = torch.full(shp, -1.0, dtype=torch.float32, device="cuda")
        q = fb.BatchCube()
        q.u8, q.out = u.data_ptr(), out.data_ptr()
        q.nz, q.ny, q.nx = shp
        q.f32_min, q.f32_max = 0.0, float(rng.uniform(0.9, 1.1))
        q.phys = fb.physics(delta_beta=db, energy_kev=110.0, distance_mm=1200.0, pixel_um=2.4, unsharp_sigma=0.8,
                            unsharp_coeff=0.5, psf_sigma_vox=1.0, psf_sigma_z_vox=1.17)
        items.append(q)
        outs.append((u, out))
    return items, outs


def _alone(fb, q, cfg):
    import torch
    lib = fb.load()
    out = torch.empty((q.nz, q.ny, q.nx), dtype=torch.float32, device="cuda")
    rc = lib.fy_gpu_restore_u8(C.c_void_p(q.u8), C.c_void_p(out.data_ptr()), q.nz, q.ny, q.nx, q.f32_min, q.f32_max,
                               C.byref(q.phys), C.byref(cfg), None)
    assert rc == 0, lib.fy_gpu_last_error()
    torch.cuda.synchronize()
    return out.cpu().numpy()


def _batch(fb, items, cfg):
    import torch
    lib = fb.load()
    arr = (fb.BatchCube * len(items))(*items)
    rc = lib.fy_gpu_restore_u8_batch(arr, len(items), C.byref(cfg), None)
    assert rc == 0, lib.fy_gpu_last_error()
    torch.cuda.synchronize()


def test_batch_equals_each_cube_alone(gpu):
    cfg = _cfg(gpu)
    items, outs = _cubes(gpu, SHAPES, seed=11)
    lib = gpu.load()
    t0 = lib.fy_gpu_kernel_timeouts()
    for rep in range(2):                                  # the second call reuses the batch buffers
        _batch(gpu, items, cfg)
        for q, (_, out) in zip(items, outs):
            got = out.cpu().numpy()
            want = _alone(gpu, q, cfg)
            assert np.isfinite(got).all()
            assert np.array_equal(got, want), ((q.nz, q.ny, q.nx), rep, np.abs(got - want).max())
    assert lib.fy_gpu_kernel_timeouts() == t0


def test_batch_of_one_and_ragged_x(gpu):
    """A single cube, and a batch holding a cube whose x extent is not a multiple of 4 (the
    whole batch then runs one cube at a time)."""
    cfg = _cfg(gpu)
    for shapes in ([(72, 80, 88)], [(40, 40, 40), (30, 34, 37), (52, 44, 60)]):
        items, outs = _cubes(gpu, shapes, seed=5)
        _batch(gpu, items, cfg)
        for q, (_, out) in zip(items, outs):
            assert np.array_equal(out.cpu().numpy(), _alone(gpu, q, cfg)), (q.nz, q.ny, q.nx)


@pytest.mark.parametrize("change", ["fixed_eps", "other_window"])
def test_batch_other_configs_match(gpu, change):
    cfg = _cfg(gpu)
    if change == "fixed_eps":
        cfg.guided_eps = 8e-4
    else:
        cfg.noise_win = 3
    items, outs = _cubes(gpu, SHAPES[:3], seed=7)
    _batch(gpu, items, cfg)
    for q, (_, out) in zip(items, outs):
        assert np.array_equal(out.cpu().numpy(), _alone(gpu, q, cfg)), (change, q.nz, q.ny, q.nx)


def test_batch_rejects_bad_arguments(gpu):
    lib = gpu.load()
    cfg = _cfg(gpu)
    q = gpu.BatchCube()
    arr = (gpu.BatchCube * 1)(q)                         # null pointers
    assert lib.fy_gpu_restore_u8_batch(arr, 1, C.byref(cfg), None) == gpu.FY_EINVAL
    assert lib.fy_gpu_restore_u8_batch(arr, -1, C.byref(cfg), None) == gpu.FY_EINVAL
    assert lib.fy_gpu_restore_u8_batch(arr, 0, C.byref(cfg), None) == 0
