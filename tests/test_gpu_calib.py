"""Calibration statistics on the GPU vs the reference and the FP64 oracle.

Bars: histogram counts exact (integer work); the flat-region noise floor and the
anisotropy ratios within 1e-9 relative (FP64 sums whose order differs from the reference's
-Ofast order by a few ulp), return codes exact.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from oracle import o64, p
from tests.test_calib_oracle import calib_volume

pytestmark = pytest.mark.gpu
REL = 1e-9


def rel_close(a, b):
    return abs(a - b) <= REL * max(abs(b), 1e-300)


@pytest.mark.parametrize("n", [0, 1, 15, 31, 4096, 1_000_003])
def test_hist_accumulate_exact(gpu, n):
    lib = gpu.load()
    rng = np.random.default_rng(n)
    u = rng.integers(0, 256, n).astype(np.uint8)
    if n > 100:
        u[: n // 3] = 0                                       # a masked run: many equal bytes
    h = gpu.HistState()
    lib.fy_hist_init(C.byref(h))
    lib.fy_hist_accumulate_u8(C.byref(h), p(u), n)
    lib.fy_hist_accumulate_u8(C.byref(h), p(u), n)            # accumulates
    want = np.zeros(256, np.int64)
    o64().o64_hist_u8(p(u), n, p(want))
    assert np.array_equal(np.array(h.hist[:]), 2 * want) and h.total == 2 * n
    if oracle.have_ref():
        r = oracle.RefHist()
        oracle.ref().fy_hist_init(C.byref(r))
        oracle.ref().fy_hist_accumulate_u8(C.byref(r), p(u), n)
        oracle.ref().fy_hist_accumulate_u8(C.byref(r), p(u), n)     # the same two chunks
        assert np.array_equal(np.array(r.hist[:]), np.array(h.hist[:])) and r.total == h.total
        for pct in (0.5, 10.0, 50.0, 99.5):
            assert lib.fy_hist_percentile_u8(C.byref(h), pct) == oracle.ref().fy_hist_percentile_u8(C.byref(r), pct)
            assert (lib.fy_hist_percentile_u8_inner(C.byref(h), pct)
                    == oracle.ref().fy_hist_percentile_u8_inner(C.byref(r), pct))


def test_hist_unaligned_device_chunk(gpu):
    import torch
    lib = gpu.load()
    u = np.random.default_rng(3).integers(0, 256, 70001).astype(np.uint8)
    d = torch.from_numpy(u).cuda()
    dh = torch.zeros(256, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    for off in (0, 1, 7, 13):                                   # chunk starts off 16-byte alignment
        dh.zero_()
        assert lib.fy_gpu_hist_accumulate_u8(C.c_void_p(d.data_ptr() + off), u.size - off,
                                             C.c_void_p(dh.data_ptr()), None) == 0
        torch.cuda.synchronize()
        want = np.zeros(256, np.int64)
        o64().o64_hist_u8(p(u[off:]), u.size - off, p(want))
        assert np.array_equal(dh.cpu().numpy(), want)


@pytest.mark.parametrize("shape,blk", [((48, 40, 56), 8), ((64, 64, 64), 4), ((33, 47, 29), 6),
                                       ((96, 96, 96), 8), ((7, 7, 7), 8), ((40, 40, 40), 0)])
def test_flat_noise(gpu, shape, blk):
    v = calib_volume(shape, sum(shape))
    got = gpu.load().fy_flat_noise(p(v), *shape, blk)
    assert rel_close(got, o64().o64_flat_noise(p(v), *shape, blk))
    if oracle.have_ref():
        assert rel_close(got, oracle.ref().fy_flat_noise(p(v), *shape, blk))


def test_flat_noise_dark_volume(gpu):
    v = np.full((32, 32, 32), 0.05, np.float32)                # no block brighter than 0.1
    assert gpu.load().fy_flat_noise(p(v), 32, 32, 32, 8) == 0.0


@pytest.mark.parametrize("shape", [(48, 40, 56), (64, 64, 64), (40, 40, 40), (96, 80, 72), (16, 16, 16)])
def test_noise_aniso(gpu, shape):
    v = calib_volume(shape, 7 + sum(shape))
    rz, rx, oz, ox = C.c_double(), C.c_double(), C.c_double(), C.c_double()
    rc = gpu.load().fy_noise_aniso(p(v), *shape, C.byref(rz), C.byref(rx))
    assert rc == o64().o64_noise_aniso(p(v), *shape, C.byref(oz), C.byref(ox))
    if rc == 0:
        assert rel_close(rz.value, oz.value) and rel_close(rx.value, ox.value)
    if oracle.have_ref():
        qz, qx = C.c_double(), C.c_double()
        assert rc == oracle.ref().fy_noise_aniso(p(v), *shape, C.byref(qz), C.byref(qx))
        if rc == 0:
            assert rel_close(rz.value, qz.value) and rel_close(rx.value, qx.value)


def test_noise_aniso_all_masked(gpu):
    v = np.zeros((64, 64, 64), np.float32)                     # every block has a voxel <= 0
    rz, rx = C.c_double(-5), C.c_double(-5)
    assert gpu.load().fy_noise_aniso(p(v), 64, 64, 64, C.byref(rz), C.byref(rx)) == 1
    assert rz.value == -5 and rx.value == -5                   # untouched on failure


def test_device_forms(gpu):
    import torch
    lib = gpu.load()
    shape = (64, 64, 64)
    v = calib_volume(shape, 11)
    d = torch.from_numpy(v).cuda()
    scratch = torch.empty(lib.fy_gpu_calib_scratch_bytes(*shape, 8), dtype=torch.uint8, device="cuda")
    out = torch.zeros(4, dtype=torch.float64, device="cuda")
    res = torch.zeros(3, dtype=torch.float64, device="cuda")   # fy_aniso_result: 24 bytes
    torch.cuda.synchronize()
    assert lib.fy_gpu_flat_noise(C.c_void_p(d.data_ptr()), *shape, 8, C.c_void_p(out.data_ptr()),
                                 C.c_void_p(scratch.data_ptr()), None) == 0
    assert lib.fy_gpu_noise_aniso(C.c_void_p(d.data_ptr()), *shape, C.c_void_p(res.data_ptr()),
                                  C.c_void_p(scratch.data_ptr()), None) == 0
    torch.cuda.synchronize()
    assert rel_close(out[0].item(), o64().o64_flat_noise(p(v), *shape, 8))
    r = gpu.AnisoResult.from_buffer_copy(res.cpu().numpy().tobytes())
    oz, ox = C.c_double(), C.c_double()
    assert r.status == o64().o64_noise_aniso(p(v), *shape, C.byref(oz), C.byref(ox)) == 0
    assert rel_close(r.rho_z, oz.value) and rel_close(r.rho_xy, ox.value)


@pytest.mark.parametrize("case", range(9))
def test_psf_sigma_gpu(gpu, case):
    """The GPU PSF edge fit equals the oracle bit for bit (same draws, same accepted edges,
    same FP64 operations in the same order) and the reference within 1e-12."""
    from tests._tiles import PSF_CASES, psf_volume
    shape, sigma, orient, noise = PSF_CASES[case]
    v = psf_volume(shape, sigma, orient, noise, 7)
    lib = gpu.load()
    n = C.c_int(-1)
    got = lib.fy_measure_psf_sigma(v.ctypes.data, *shape, C.byref(n))
    on = C.c_int(-1)
    want = o64().ot_measure_psf_sigma(p(v), *shape, C.byref(on))
    assert n.value == on.value and got == want, (got, want, n.value, on.value)
    if oracle.ref_psf() is not None:
        ref = oracle.ref_psf().ref_measure_tile_psf_sigma(p(v), *shape)
        assert abs(got - ref) <= 1e-12 * max(abs(ref), 1.0)


def test_psf_sigma_device_form(gpu):
    import torch
    from tests._tiles import psf_volume
    v = psf_volume((32, 64, 64), 1.2, "xy", 1.0, 3)
    lib = gpu.load()
    d = torch.from_numpy(v).cuda()
    out = torch.zeros(2, dtype=torch.float64, device="cuda")       # { double sigma; int nprof; }
    torch.cuda.synchronize()
    assert lib.fy_gpu_measure_psf_sigma(C.c_void_p(d.data_ptr()), *v.shape, C.c_void_p(out.data_ptr()), None) == 0
    torch.cuda.synchronize()
    h = out.cpu().numpy()
    sigma, nprof = h[0], int(h[1:].view(np.int32)[0])
    n = C.c_int()
    assert sigma == lib.fy_measure_psf_sigma(v.ctypes.data, *v.shape, C.byref(n)) and nprof == n.value
    assert np.isnan(lib.fy_measure_psf_sigma(v.ctypes.data, 0, 64, 64, None))      # bad dims: NaN + status
    assert lib.fy_gpu_last_status() == gpu.FY_EINVAL
