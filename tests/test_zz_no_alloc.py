"""fy_gpu_estimate_noise_noalloc (static library scratch, no allocation) against
fy_gpu_estimate_noise (caller scratch) on the same device volumes, and against the
reference's own fy_estimate_noise (noise.c:75-192; the FP64 oracle where the reference
library is not built).

The two GPU entry points run the same kernels, so their models must agree within the noise
tests' stated tolerance (noise_ref 1e-3 relative, bin count exact); in practice they are
identical. The reference computes its box sums and percentiles in FP64, so against it the
same tolerance is the bar of the noise tests.
Consecutive calls share the static scratch, so each case runs twice in a row on different
volumes and shapes: a result must not depend on what the previous call left behind.
The file is collected last so the calls also run after every other GPU test.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from oracle import o64, p
from tests import _recipes as R

pytestmark = pytest.mark.gpu

MAX_VOXELS = 2097152          # FY_NOISE_NOALLOC_MAX_VOXELS (128^3)


def close(a, b, rel=1e-3):
    return abs(a - b) <= rel * max(abs(b), 1e-12)


def model_with_scratch(fy, d, shape, win, pct, ref):
    import torch
    lib = fy.load()
    scratch = torch.empty(lib.fy_gpu_noise_scratch_bytes(*shape), dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    assert lib.fy_gpu_estimate_noise(C.c_void_p(d.data_ptr()), *shape, win, pct, ref,
                                     C.c_void_p(scratch.data_ptr()), None) == 0, lib.fy_gpu_last_error()
    nm = fy.NoiseModel()
    assert lib.fy_gpu_noise_model(C.c_void_p(scratch.data_ptr()), *shape, C.byref(nm), None) == 0
    return nm


def model_noalloc(fy, d, shape, win, pct, ref, with_eps=True):
    import torch
    lib = fy.load()
    out = torch.full((C.sizeof(fy.NoiseModel),), 0xAB, dtype=torch.uint8, device="cuda")
    eps = torch.full((1,), -1.0, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    rc = lib.fy_gpu_estimate_noise_noalloc(C.c_void_p(d.data_ptr()), *shape, win, pct, ref,
                                           C.c_void_p(out.data_ptr()),
                                           C.c_void_p(eps.data_ptr()) if with_eps else None, None)
    assert rc == 0, lib.fy_gpu_last_error()
    torch.cuda.synchronize()
    nm = fy.NoiseModel.from_buffer_copy(out.cpu().numpy().tobytes())
    return nm, float(eps.cpu().numpy()[0])


def model_reference(vol, win, pct, ref):
    """The reference's fy_estimate_noise on the host (the FP64 oracle without the library)."""
    nm = oracle.RefNoise()
    a = np.ascontiguousarray(vol, np.float32)
    fn = oracle.ref().fy_estimate_noise if oracle.have_ref() else o64().o64_estimate_noise
    assert fn(p(a), *a.shape, win, pct, ref, C.byref(nm)) == 0
    return nm


def check_same(fy, vol, win=5, pct=10.0, ref=0.5, with_eps=True):
    import torch
    d = torch.from_numpy(np.ascontiguousarray(vol, np.float32)).cuda()
    want = model_with_scratch(fy, d, vol.shape, win, pct, ref)
    got, eps = model_noalloc(fy, d, vol.shape, win, pct, ref, with_eps)
    assert got.n_bins_used == want.n_bins_used
    assert close(got.noise_ref, want.noise_ref)
    scale = max(abs(want.g), abs(want.b), 1e-12)
    assert abs(got.g - want.g) <= 1e-3 * scale and abs(got.b - want.b) <= 1e-3 * scale
    assert got.ref_intensity == want.ref_intensity
    if with_eps:
        assert eps == np.float32(fy.load().fy_guided_eps_for_noise(got.noise_ref))
    else:
        assert eps == -1.0                                            # d_eps NULL: untouched
    r = model_reference(vol, win, pct, ref)
    assert got.n_bins_used == r.n_bins_used
    assert close(got.noise_ref, r.noise_ref)
    return got


def test_noalloc_matches_scratch_entry_point(gpu):
    v1 = R.noise_input(0.05, 12345)                                   # recipe volume
    v2 = np.random.default_rng(7).normal(0.4, 0.08, (33, 70, 41)).astype(np.float32)
    a = check_same(gpu, v1)
    b = check_same(gpu, v2, win=3, pct=20.0, ref=0.3)                 # second call in a row
    a2 = check_same(gpu, v1, with_eps=False)                          # and back, no eps output
    assert a2.noise_ref == a.noise_ref and a2.n_bins_used == a.n_bins_used
    assert b.noise_ref != a.noise_ref


def test_noalloc_largest_volume(gpu):
    vol = np.random.default_rng(3).normal(0.5, 0.05, (128, 128, 128)).astype(np.float32)
    assert vol.size == MAX_VOXELS
    check_same(gpu, vol)
    check_same(gpu, vol[:, :64, :], win=7)


def test_noalloc_rejects_oversize(gpu):
    import torch
    lib = gpu.load()
    d = torch.zeros(8, dtype=torch.float32, device="cuda")
    out = torch.zeros(C.sizeof(gpu.NoiseModel), dtype=torch.uint8, device="cuda")
    rc = lib.fy_gpu_estimate_noise_noalloc(C.c_void_p(d.data_ptr()), 129, 128, 128, 5, 10.0, 0.5,
                                           C.c_void_p(out.data_ptr()), None, None)
    assert rc == 5                                                    # FY_EUNSUPPORTED
    assert b"static scratch limit" in lib.fy_gpu_last_error()


def test_noalloc_rejects_misaligned_model(gpu):
    import torch
    lib = gpu.load()
    d = torch.zeros(8 * 8 * 8, dtype=torch.float32, device="cuda")
    out = torch.zeros(C.sizeof(gpu.NoiseModel) + 16, dtype=torch.uint8, device="cuda")
    rc = lib.fy_gpu_estimate_noise_noalloc(C.c_void_p(d.data_ptr()), 8, 8, 8, 5, 10.0, 0.5,
                                           C.c_void_p(out.data_ptr() + 4), None, None)
    assert rc == 1                                                    # FY_EINVAL, nothing enqueued
    assert b"aligned" in lib.fy_gpu_last_error()
    rc = lib.fy_gpu_estimate_noise_noalloc(C.c_void_p(d.data_ptr()), 8, 8, 8, 5, 10.0, 0.5,
                                           C.c_void_p(out.data_ptr()), C.c_void_p(out.data_ptr() + 2), None)
    assert rc == 1
