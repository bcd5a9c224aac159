"""Phase correlation on the GPU: integer peaks bit-exact against the reference and the
FP64 oracle; sub-voxel shift within 0.01 vox of the reference (FP32 side lobes) and
within the reference test's 0.15 L1 of the ground truth."""
import ctypes as C

import numpy as np
import pytest

import oracle
from oracle import o64, p
from tests import _recipes as R
from tests.test_oracle_pins import golden

pytestmark = pytest.mark.gpu


def gpu_pc(fy, f, m, window):
    sh = (C.c_double * 3)()
    pk = C.c_double()
    rc = fy.load().fy_phase_correlate(p(f), p(m), *f.shape, sh, C.byref(pk), window)
    return rc, np.array(sh[:]), pk.value


def o64_pc(f, m, window):
    sh = (C.c_double * 3)()
    pk = C.c_double()
    idx = C.c_long()
    f64, m64 = f.astype(np.float64), m.astype(np.float64)
    rc = o64().o64_phase_correlate(p(f64), p(m64), *f.shape, sh, C.byref(pk), window, C.byref(idx))
    return rc, np.array(sh[:]), pk.value, idx.value


def ref_pc(f, m, window):
    sh = (C.c_double * 3)()
    pk = C.c_double()
    rc = oracle.ref().fy_phase_correlate(p(f), p(m), *f.shape, sh, C.byref(pk), window)
    return rc, np.array(sh[:]), pk.value


def integer_part(s):
    return np.round(s - np.clip(s - np.round(s), -0.5, 0.5)).astype(int)


@pytest.mark.parametrize("case", range(3))
def test_subvoxel_recipe(gpu, case):
    f = R.phasecorr_texture()
    truth = np.array(R.PHASECORR_CASES[case])
    m = R.fourier_shift(f, truth)
    rc, s, pk = gpu_pc(gpu, f, m, 0)
    assert rc == 0
    assert np.abs(s - truth).sum() < 0.15                        # test_fysics.c:923
    ref = ref_pc(f, m, 0)[1] if oracle.have_ref() else golden()[f"phasecorr_{case}"][:3]
    assert np.array_equal(integer_part(s), integer_part(ref))
    assert np.abs(s - ref).max() < 1e-2
    o = o64_pc(f, m, 0)
    assert np.array_equal(integer_part(s), integer_part(o[1]))


def test_contrast_invariance(gpu):
    f = R.phasecorr_texture()
    m = (0.3 * R.fourier_shift(f, (0.4, -0.6, 0.5)) + 0.4).astype(np.float32)
    rc, s, _ = gpu_pc(gpu, f, m, 0)
    assert rc == 0 and np.abs(s - np.array([0.4, -0.6, 0.5])).sum() < 0.15


@pytest.mark.parametrize("shape,shift,window", [((40, 48, 56), (5, -7, 3), 1), ((20, 24, 30), (2, 3, -4), 1),
                                                ((64, 64, 64), (-11, 9, 20), 0), ((33, 17, 70), (1, -2, 6), 1)])
def test_integer_shifts_windowed(gpu, shape, shift, window):
    rng = np.random.default_rng(sum(shape))
    big = rng.uniform(0, 1, tuple(s + 2 * abs(t) + 2 for s, t in zip(shape, shift))).astype(np.float32)
    o = [abs(t) + 1 for t in shift]
    f = np.ascontiguousarray(big[o[0]:o[0] + shape[0], o[1]:o[1] + shape[1], o[2]:o[2] + shape[2]])
    m = np.ascontiguousarray(big[o[0] - shift[0]:o[0] - shift[0] + shape[0], o[1] - shift[1]:o[1] - shift[1] + shape[1],
                                 o[2] - shift[2]:o[2] - shift[2] + shape[2]])
    rc, s, pk = gpu_pc(gpu, f, m, window)
    assert rc == 0
    ro = o64_pc(f, m, window)
    assert np.array_equal(integer_part(s), integer_part(ro[1]))
    assert np.array_equal(integer_part(s), np.array(shift))
    if oracle.have_ref():
        rr = ref_pc(f, m, window)
        assert np.array_equal(integer_part(s), integer_part(rr[1]))
        assert np.abs(s - rr[1]).max() < 1e-2 and abs(pk - rr[2]) < 1e-3


def test_degenerate_and_bad_args(gpu):
    f = np.full((16, 16, 16), 0.5, np.float32)
    m = np.random.default_rng(0).uniform(0, 1, f.shape).astype(np.float32)
    rc, s, pk = gpu_pc(gpu, f, m, 1)
    assert rc == 1 and not s.any() and pk == 0.0                  # phasecorr.c:111-114
    small = np.zeros((1, 8, 8), np.float32)
    assert gpu_pc(gpu, small, small, 0)[0] == 1                  # phasecorr.c:47


def test_batch_device_api(gpu):
    import torch
    f = R.phasecorr_texture()
    pairs = [R.fourier_shift(f, c) for c in R.PHASECORR_CASES] + [np.roll(f, (3, -5, 7), axis=(0, 1, 2))]
    lib = gpu.load()
    df = torch.from_numpy(np.stack([f] * len(pairs))).cuda()
    dm = torch.from_numpy(np.stack(pairs).astype(np.float32)).cuda()
    scratch = torch.empty(lib.fy_gpu_phase_correlate_scratch_bytes(32, 32, 32), dtype=torch.uint8, device="cuda")
    n = len(pairs)
    sh = (C.c_double * (3 * n))()
    pk = (C.c_double * n)()
    idx = (C.c_longlong * n)()
    st = (C.c_int * n)()
    torch.cuda.synchronize()
    rc = lib.fy_gpu_phase_correlate_batch(C.c_void_p(df.data_ptr()), C.c_void_p(dm.data_ptr()), n, 32, 32, 32, 0,
                                          C.c_void_p(scratch.data_ptr()), sh, pk, idx, st, None)
    assert rc == 0
    for i, m in enumerate(pairs):
        rc1, s1, p1 = gpu_pc(gpu, f, m, 0)
        assert st[i] == 0 and np.array_equal(np.array(sh[3 * i:3 * i + 3]), s1) and pk[i] == p1
        assert idx[i] == o64_pc(f, m, 0)[3]                      # bit-exact integer peak
    assert np.array_equal(integer_part(np.array(sh[9:12])), [3, -5, 7])


@pytest.mark.skipif(not oracle.have_ref(), reason="reference library not built")
@pytest.mark.parametrize("window,seed", [(0, 41), (1, 42)])
def test_config4_pair_256_vs_reference(gpu, window, seed):
    """A registration pair at the batched-registration configuration's size: 256^3 phantom
    (u8/255), the moving volume an FP64 Fourier shift by an integer U[-40,40] plus a
    subvoxel U[-0.5,0.5] per axis, independent noise var = 0.002*I + 1e-4 on each. The
    integer peak must equal the reference's fy_phase_correlate (phasecorr.c:121-131) and
    the subvoxel shift be within 0.01 vox of it; without the window the shift is also held
    to the reference test's 0.15 L1 of the truth."""
    import torch
    import fysics_b200.phantom as ph
    n = 256
    rng = np.random.default_rng(seed)
    u = ph.phantom((n, n, n), seed=seed, delta_beta=175.0, pixel_um=2.4, device="cuda")
    f = u.to(torch.float64) / 255.0
    k = torch.fft.fftfreq(n, device="cuda", dtype=torch.float64) * n
    k[n // 2] = n // 2
    s = rng.integers(-40, 41, 3) + rng.uniform(-0.5, 0.5, 3)
    phase = -2 * np.pi * (k[:, None, None] * s[0] + k[None, :, None] * s[1] + k[None, None, :] * s[2]) / n
    m = torch.fft.ifftn(torch.fft.fftn(f) * torch.exp(1j * phase)).real
    g = torch.Generator(device="cuda").manual_seed(seed)

    def noisy(v):
        return (v + torch.sqrt(0.002 * v.clamp(min=0) + 1e-4) *
                torch.randn(v.shape, generator=g, device="cuda", dtype=torch.float64)).float().cpu().numpy()

    fixed, moving = noisy(f), noisy(m)
    del f, m, phase
    rc, got, pk = gpu_pc(gpu, fixed, moving, window)
    assert rc == 0
    rr = ref_pc(fixed, moving, window)
    assert rr[0] == 0
    assert np.array_equal(integer_part(got), integer_part(rr[1]))
    assert np.abs(got - rr[1]).max() < 1e-2
    if window == 0:
        assert np.abs(got - s).sum() < 0.15
