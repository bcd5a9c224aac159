"""Guided filter and box mean on the GPU vs the reference and the FP64 oracle.

Tolerance: max abs error <= 1e-4 x window range (inputs span ~1). The reference's own
FP32 error against FP64 on these inputs is ~1.3e-5 (E[I^2]-E[I]^2 cancellation).
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from oracle import o64, p
from tests import _recipes as R
from tests.test_oracle_pins import golden

pytestmark = pytest.mark.gpu
TOL = 1e-4


def gpu_guided(fy, vol, r, eps, s=1):
    a = np.ascontiguousarray(vol, np.float32)
    out = np.empty_like(a)
    ws = np.empty(4 * a.size, np.float32)
    lib = fy.load()
    if s <= 1:
        rc = lib.fy_guided_denoise_ws(p(a), p(out), *a.shape, r, eps, p(ws))
    else:
        rc = lib.fy_guided_denoise_fast_ws(p(a), p(out), *a.shape, r, eps, s, p(ws))
    assert rc == 0, lib.fy_gpu_last_error()
    return out


def o64_guided(vol, r, eps, s=1):
    a = np.ascontiguousarray(vol, np.float64)
    out = np.empty_like(a)
    if s <= 1:
        assert o64().o64_guided(p(a), p(out), *a.shape, r, eps) == 0
    else:
        assert o64().o64_guided_fast(p(a), p(out), *a.shape, r, eps, s) == 0
    return out


def ref_guided(vol, r, eps, s=1):
    a = np.ascontiguousarray(vol, np.float32)
    out = np.empty_like(a)
    ws = np.empty(4 * a.size, np.float32)
    if s <= 1:
        assert oracle.ref().fy_guided_denoise_ws(p(a), p(out), *a.shape, r, eps, p(ws)) == 0
    else:
        assert oracle.ref().fy_guided_denoise_fast_ws(p(a), p(out), *a.shape, r, eps, s, p(ws)) == 0
    return out


def test_step_edge_recipe(gpu):
    vol = R.guided_step_input()
    got = gpu_guided(gpu, vol, 2, 0.0004)
    ref = ref_guided(vol, 2, 0.0004) if oracle.have_ref() else golden()["guided_exact"]
    assert np.abs(got - o64_guided(vol, 2, 0.0004)).max() < 2e-5      # closer to FP64 than the reference
    assert np.abs(got - ref).max() < TOL


@pytest.mark.parametrize("shape,r", [((32, 32, 32), 1), ((33, 17, 45), 2), ((5, 70, 3), 2), ((1, 1, 1), 2),
                                     ((2, 9, 40), 3), ((40, 40, 40), 4), ((20, 30, 25), 5), ((12, 12, 12), 7)])
def test_shapes_and_radii(gpu, shape, r):
    rng = np.random.default_rng(sum(shape) + r)
    base = np.linspace(0.2, 0.8, shape[2], dtype=np.float32)[None, None, :]
    vol = (base + 0.05 * rng.standard_normal(shape)).astype(np.float32)
    eps = 0.003
    got = gpu_guided(gpu, vol, r, eps)
    assert np.abs(got - o64_guided(vol, r, eps)).max() < TOL
    if oracle.have_ref():
        assert np.abs(got - ref_guided(vol, r, eps)).max() < TOL


def test_radius_default(gpu):
    vol = np.random.default_rng(0).uniform(0, 1, (16, 16, 16)).astype(np.float32)
    assert np.array_equal(gpu_guided(gpu, vol, 0, 0.01), gpu_guided(gpu, vol, 2, 0.01))   # guided.c:115


def test_fast_variant(gpu):
    vol = R.guided_step_input()
    fast = gpu_guided(gpu, vol, 2, 0.0004, s=2)
    exact = gpu_guided(gpu, vol, 2, 0.0004)
    ref = ref_guided(vol, 2, 0.0004, 2) if oracle.have_ref() else golden()["guided_fast"]
    assert np.abs(fast - ref).max() < TOL
    assert np.abs(fast - o64_guided(vol, 2, 0.0004, 2)).max() < TOL
    # test_guided_fast (test_fysics.c:107-117)
    assert np.abs(fast - exact).mean() < 0.01
    nz, ny, nx = vol.shape
    ee = (exact[:, :, nx // 2 + 4] - exact[:, :, nx // 2 - 4]).mean()
    ef = (fast[:, :, nx // 2 + 4] - fast[:, :, nx // 2 - 4]).mean()
    assert ef > 0.8 * ee


@pytest.mark.parametrize("shape,s", [((31, 40, 57), 2), ((64, 64, 64), 3), ((3, 64, 64), 2)])
def test_fast_shapes(gpu, shape, s):
    rng = np.random.default_rng(7)
    vol = (0.5 + 0.1 * rng.standard_normal(shape)).astype(np.float32)
    got = gpu_guided(gpu, vol, 2, 0.002, s)
    assert np.abs(got - o64_guided(vol, 2, 0.002, s)).max() < TOL
    if oracle.have_ref():
        assert np.abs(got - ref_guided(vol, 2, 0.002, s)).max() < TOL


@pytest.mark.parametrize("r", [1, 2, 5])
def test_box_smooth(gpu, r):
    vol = np.random.default_rng(r).uniform(0, 1, (21, 34, 47)).astype(np.float32)
    out = np.empty_like(vol)
    tmp = np.empty_like(vol)
    gpu.load().fy_box_smooth(p(vol), p(out), p(tmp), *vol.shape, r)
    gpu.check_void("fy_box_smooth")
    want = np.empty(vol.shape, np.float64)
    v64 = vol.astype(np.float64)
    o64().o64_box_mean(p(v64), p(want), *vol.shape, r)
    assert np.abs(out - want).max() < 1e-6


def test_device_inplace(gpu):
    import torch
    vol = np.random.default_rng(3).uniform(0, 1, (48, 40, 56)).astype(np.float32)
    want = gpu_guided(gpu, vol, 2, 0.002)
    d = torch.from_numpy(vol).cuda()
    torch.cuda.synchronize()
    rc = gpu.load().fy_gpu_guided(C.c_void_p(d.data_ptr()), C.c_void_p(d.data_ptr()), 48, 40, 56, 2, 0.002, 1, None)
    assert rc == 0
    torch.cuda.synchronize()
    assert np.array_equal(d.cpu().numpy(), want)


def test_box_pass_waits_never_expired(gpu):
    """The box passes' bounded waits on tensor-copy completion never gave up during the
    GPU tests run so far (their expiry would leave the output unfinished)."""
    vol = np.random.default_rng(2).uniform(0, 1, (40, 64, 64)).astype(np.float32)
    out = np.empty_like(vol)
    assert gpu.load().fy_guided_denoise(p(vol), p(out), *vol.shape, 2, 1e-3) == 0
    assert gpu.load().fy_gpu_kernel_timeouts() == 0
