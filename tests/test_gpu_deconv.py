"""Wiener deconvolution on the GPU vs the reference CPU path and the FP64 oracle.

Tolerance (stated bar): max abs error <= 1e-4 x window range; inputs here live in a
window of range 1, so 1e-4 absolute. Measured errors are ~1e-6 (FP32 FFT rounding).
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from tests import _recipes as R
from tests.test_oracle_pins import golden

pytestmark = pytest.mark.gpu
TOL = 1e-4


def rphys(ph):
    return oracle.RefPhysics(*[getattr(ph, n) for n, _ in ph._fields_])


def test_rfft_equivalence_recipe(gpu):
    """test_deconv_rfft_equivalence input (22x27x30, pads to 24x32x32)."""
    vol = R.deconv_equivalence_input()
    ph = gpu.physics()
    got = gpu.deconvolve(vol, ph, 0.015)
    ref = oracle.ref_deconvolve(vol, rphys(ph), 0.015) if oracle.have_ref() else golden()["deconv_equiv"]
    o64 = oracle.o64_deconvolve(vol, rphys(ph), 0.015, kind=0)
    assert np.abs(got - ref).max() < 1e-5
    assert np.abs(got - o64).max() < 1e-5


SHAPES = [(1, 1, 1), (1, 1, 8), (2, 3, 5), (3, 1, 7), (8, 8, 8), (17, 9, 33), (12, 8, 24),
          (48, 48, 48), (64, 96, 80), (13, 200, 7), (96, 96, 96), (40, 33, 130)]


@pytest.mark.parametrize("shape", SHAPES)
def test_deconv_shapes_vs_reference_and_fp64(gpu, shape):
    rng = np.random.default_rng(sum(shape))
    vol = rng.uniform(0, 1, shape).astype(np.float32)
    ph = gpu.physics()
    got = gpu.deconvolve(vol, ph, 0.015)
    o64 = oracle.o64_deconvolve(vol, rphys(ph), 0.015, kind=0)
    assert np.abs(got - o64).max() < TOL
    # The reference reads its LUT at index (int)NaN for a 1x1x1 volume (us = 4096/0,
    # paganin.c:225-239) and crashes; that shape is checked against the FP64 oracle only.
    if oracle.have_ref() and shape != (1, 1, 1):
        ref = oracle.ref_deconvolve(vol, rphys(ph), 0.015)
        assert np.abs(got - ref).max() < TOL


@pytest.mark.parametrize("shape", [(22, 27, 30), (48, 48, 48), (33, 64, 20)])
def test_matched_aniso_vs_reference(gpu, shape):
    rng = np.random.default_rng(5)
    vol = rng.uniform(0, 1, shape).astype(np.float32)
    ph = gpu.physics(psf_sigma_vox=1.0, psf_sigma_z_vox=1.17)
    got = gpu.deconvolve_matched(vol, ph, 0.05)
    o64 = oracle.o64_deconvolve(vol, rphys(ph), 0.05, kind=1)
    assert np.abs(got - o64).max() < TOL
    if oracle.have_ref():
        assert np.abs(got - oracle.ref_deconvolve(vol, rphys(ph), 0.05, matched=True)).max() < TOL
    elif shape == (22, 27, 30):
        pass


def test_default_regs(gpu):
    """reg <= 0 -> 0.015 (paganin.c:305); tikhonov <= 0 -> 0.05 (paganin.c:333)."""
    vol = np.random.default_rng(9).uniform(0, 1, (16, 16, 16)).astype(np.float32)
    ph = gpu.physics(psf_sigma_vox=0.0)
    assert np.array_equal(gpu.deconvolve(vol, ph, 0.0), gpu.deconvolve(vol, ph, 0.015))
    assert np.array_equal(gpu.deconvolve_matched(vol, ph, -1.0), gpu.deconvolve_matched(vol, ph, 0.05))


def test_inplace_alias(gpu):
    vol = np.random.default_rng(2).uniform(0, 1, (20, 24, 28)).astype(np.float32)
    ph = gpu.physics()
    want = gpu.deconvolve(vol, ph, 0.015)
    buf = vol.copy()
    lib = gpu.load()
    assert lib.fy_deconvolve(buf.ctypes.data, buf.ctypes.data, 20, 24, 28, C.byref(ph), 0.015) == 0
    assert np.array_equal(buf, want)


def test_constant_volume_dc_gain(gpu):
    """A constant volume has only DC: out = c * w(0) = c / (1 + reg) for H(0) = 1."""
    vol = np.full((24, 40, 36), 0.37, np.float32)
    got = gpu.deconvolve(vol, gpu.physics(), 0.015)
    assert np.abs(got - 0.37 / 1.015).max() < 2e-6


def test_linearity_full_size(gpu):
    """Size-independent property at a production size: deconv is linear."""
    rng = np.random.default_rng(11)
    a = rng.uniform(0, 1, (128, 128, 128)).astype(np.float32)
    b = rng.uniform(0, 1, (128, 128, 128)).astype(np.float32)
    ph = gpu.physics()
    da, db = gpu.deconvolve(a, ph, 0.015), gpu.deconvolve(b, ph, 0.015)
    dab = gpu.deconvolve((0.25 * a + 0.5 * b).astype(np.float32), ph, 0.015)
    assert np.abs(dab - (0.25 * da + 0.5 * db)).max() < 2e-5


def test_u8_source_fused_dewindow(gpu):
    """fy_gpu_deconvolve_ex with a u8 source == fy_u8_to_phys then fy_deconvolve."""
    import torch
    rng = np.random.default_rng(4)
    u8 = rng.integers(0, 256, (40, 48, 56), dtype=np.uint8)
    lo, hi = -0.03, 0.21
    ph = gpu.physics()
    want = gpu.deconvolve(gpu.u8_to_phys(u8, lo, hi), ph, 0.015)
    d_in = torch.from_numpy(u8).cuda()
    d_out = torch.empty(u8.shape, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    rc = gpu.load().fy_gpu_deconvolve_ex(C.c_void_p(d_in.data_ptr()), 1, lo, hi,
                                         C.c_void_p(d_out.data_ptr()), 40, 48, 56, C.byref(ph),
                                         0.015, 0, 1.0, None)
    assert rc == 0, gpu.load().fy_gpu_last_error()
    torch.cuda.synchronize()
    assert np.array_equal(d_out.cpu().numpy(), want)


def test_aniso_paganin_kind2_vs_fp64(gpu):
    import torch
    rng = np.random.default_rng(6)
    vol = rng.uniform(0, 1, (32, 48, 40)).astype(np.float32)
    ph = gpu.physics()
    d_in = torch.from_numpy(vol).cuda()
    d_out = torch.empty_like(d_in)
    torch.cuda.synchronize()
    rc = gpu.load().fy_gpu_deconvolve_ex(C.c_void_p(d_in.data_ptr()), 0, 0.0, 0.0,
                                         C.c_void_p(d_out.data_ptr()), 32, 48, 40, C.byref(ph),
                                         0.015, 2, 1.17 ** 2, None)
    assert rc == 0
    torch.cuda.synchronize()
    o64 = oracle.o64_deconvolve(vol, rphys(ph), 0.015, kind=2, fz2_scale=1.17 ** 2)
    assert np.abs(d_out.cpu().numpy() - o64).max() < TOL


def test_oversize_axis_rejected(gpu):
    """Axes whose padded size exceeds 4096 are refused with FY_EUNSUPPORTED (no crash)."""
    lib = gpu.load()
    dummy = np.zeros(8, np.float32)
    rc = lib.fy_deconvolve(dummy.ctypes.data, dummy.ctypes.data, 1, 1, 5000, C.byref(gpu.physics()), 0.015)
    assert rc == gpu.FY_EUNSUPPORTED


def test_viewer_slab(gpu):
    """The viewer path (README.md:109-118, :190): fy_kernel_halo, then fy_deconvolve on an
    8x512x512 slab -- a thin z axis (pz = 8) under full 512^2 planes."""
    ph = gpu.physics(delta_beta=1000.0, energy_kev=78.0, distance_mm=220.0, pixel_um=2.4,
                     unsharp_sigma=1.2, unsharp_coeff=4.0)
    r = rphys(ph)
    halo = gpu.kernel_halo(ph)
    if oracle.have_ref():
        assert halo == oracle.ref().fy_kernel_halo(C.byref(r))
    rng = np.random.default_rng(190)
    slab = rng.uniform(0, 1, (8, 512, 512)).astype(np.float32)
    got = gpu.deconvolve(slab, ph, -1.0)
    o64 = oracle.o64_deconvolve(slab, r, -1.0, kind=0)
    assert np.abs(got - o64).max() < TOL
    if oracle.have_ref():
        ref = oracle.ref_deconvolve(slab, r, -1.0)
        assert np.abs(got - ref).max() < TOL


@pytest.mark.parametrize("shape,matched", [((16, 40, 320), False), ((320, 24, 20), True),
                                           ((96, 200, 320), False), ((96, 200, 320), True)])
def test_deconv_384_pad_vs_reference(gpu, shape, matched):
    """An axis of 320 pads to 384 = 3*2^7 (fy_next_fft_size, fft.c:34-38; paganin.c:155):
    the reflect padding, the radix-3 plans and the LUT range at that size against the
    reference and the FP64 oracle. (96, 200, 320) is one of the uneven-cube shapes of the
    batched configuration (pads 96 / 256 / 384)."""
    assert gpu.load().fy_next_fft_size(320) == 384
    rng = np.random.default_rng(sum(shape) + matched)
    vol = rng.uniform(0, 1, shape).astype(np.float32)
    if matched:
        ph = gpu.physics(psf_sigma_vox=1.0, psf_sigma_z_vox=1.17)
        got = gpu.deconvolve_matched(vol, ph, 0.05)
    else:
        ph = gpu.physics()
        got = gpu.deconvolve(vol, ph, 0.015)
    o64 = oracle.o64_deconvolve(vol, rphys(ph), 0.05 if matched else 0.015, kind=1 if matched else 0)
    assert np.abs(got - o64).max() < TOL
    if oracle.have_ref():
        ref = oracle.ref_deconvolve(vol, rphys(ph), 0.05 if matched else 0.015, matched=matched)
        assert np.abs(got - ref).max() < TOL
