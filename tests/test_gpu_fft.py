"""fy_fft1d / fy_fft3d / fy_fft3d_normalize on the GPU vs numpy FP64, plus the
reference's FFT known-answer tests and fy_kernel_halo."""
import ctypes as C

import numpy as np
import pytest

import oracle
from oracle import p

pytestmark = pytest.mark.gpu

SIZES = [1, 2, 3, 4, 6, 8, 12, 16, 24, 32, 48, 64, 96, 128, 192, 256, 384, 512, 768, 1024, 1536, 2048, 3072, 4096]


def fft1(fy, x, sign):
    re = np.ascontiguousarray(x.real, np.float32)
    im = np.ascontiguousarray(x.imag, np.float32)
    fy.load().fy_fft1d(p(re), p(im), x.size, sign)
    fy.check_void("fy_fft1d")
    return re.astype(np.float64) + 1j * im


@pytest.mark.parametrize("n", SIZES)
def test_fft1d_vs_numpy(gpu, n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    x = x.astype(np.complex64).astype(np.complex128)
    scale = np.sqrt(n) * np.log2(max(n, 2))
    assert np.abs(fft1(gpu, x, -1) - np.fft.fft(x)).max() < 2e-6 * scale
    assert np.abs(fft1(gpu, x, +1) - np.fft.ifft(x) * n).max() < 2e-6 * scale


def test_fft_vs_dft_kat(gpu):
    """test_fft_vs_dft (test_fysics.c:26-40) and the radix-3 n=48 case (:56-72)."""
    i = np.arange(16)
    x = (np.sin(i * np.float32(0.7)).astype(np.float32) + np.float32(0.3) * i).astype(np.complex128)
    assert np.abs(fft1(gpu, x, -1) - np.fft.fft(x)).max() < 1e-3
    i = np.arange(48)
    x = (np.sin(i * np.float32(0.7)) + np.float32(0.3) * np.cos(i * np.float32(1.3))).astype(np.float32) \
        + 1j * (np.float32(0.2) * np.sin(i * np.float32(0.31))).astype(np.float32)
    got = fft1(gpu, x, -1)
    assert (np.abs(got.real - np.fft.fft(x).real) + np.abs(got.imag - np.fft.fft(x).imag)).max() < 1e-3


@pytest.mark.parametrize("shape", [(8, 8, 8), (12, 8, 24), (1, 16, 48), (32, 3, 64), (96, 128, 24)])
def test_fft3d_roundtrip_and_numpy(gpu, shape):
    n = int(np.prod(shape))
    rng = np.random.default_rng(n)
    re = rng.uniform(0, 1, shape).astype(np.float32)
    im = np.zeros(shape, np.float32)
    orig = re.copy()
    lib = gpu.load()
    lib.fy_fft3d(p(re), p(im), *shape, -1)
    gpu.check_void("fy_fft3d")
    want = np.fft.fftn(orig.astype(np.float64))
    # FP32 rounding relative to the spectrum's peak (the DC bin is ~n/2)
    assert np.abs((re + 1j * im) - want).max() < 2e-7 * np.log2(n) * np.abs(want).max()
    lib.fy_fft3d(p(re), p(im), *shape, +1)
    lib.fy_fft3d_normalize(p(re), p(im), *shape)
    gpu.check_void("fy_fft3d_normalize")
    assert np.abs(re - orig).max() < 1e-4 and np.abs(im).max() < 1e-4      # test_fysics.c:42-54, 74-84


def test_unsupported_size_recorded(gpu):
    re = np.zeros(10, np.float32)
    im = np.zeros(10, np.float32)
    gpu.load().fy_fft1d(p(re), p(im), 10, -1)
    assert gpu.load().fy_gpu_last_status() == gpu.FY_EUNSUPPORTED


def test_kernel_halo(gpu):
    ph = gpu.physics()
    h = gpu.kernel_halo(ph)
    assert 8 <= h <= 96                                          # test_fysics.c:352-357
    if oracle.have_ref():
        for kw in ({}, dict(delta_beta=500, pixel_um=7.91, energy_kev=110, distance_mm=1200, unsharp_sigma=0.8,
                            unsharp_coeff=0.5), dict(delta_beta=100, pixel_um=9.4)):
            a = gpu.physics(**kw)
            r = oracle.ref_physics(**kw)
            assert gpu.kernel_halo(a) == oracle.ref().fy_kernel_halo(C.byref(r))
