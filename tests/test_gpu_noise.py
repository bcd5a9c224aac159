"""fy_estimate_noise on the GPU vs the reference and the FP64 oracle.

Stated tolerance: noise_ref within 1e-3 relative (order statistics of local variances
whose FP32 values differ from the reference's FP64 ones in the last bits); bin count
exact; g, b within 1e-3 relative of max(|g|,|b|)-scale.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from oracle import o64, p
from tests import _recipes as R
from tests.test_oracle_pins import golden

pytestmark = pytest.mark.gpu


def gpu_noise(fy, vol, win=5, pct=10.0, ref=0.5):
    nm = fy.NoiseModel()
    a = np.ascontiguousarray(vol, np.float32)
    rc = fy.load().fy_estimate_noise(p(a), *a.shape, win, pct, ref, C.byref(nm))
    assert rc == 0, fy.load().fy_gpu_last_error()
    return nm


def o64_noise(vol, win=5, pct=10.0, ref=0.5):
    nm = oracle.RefNoise()
    a = np.ascontiguousarray(vol, np.float32)
    assert o64().o64_estimate_noise(p(a), *a.shape, win, pct, ref, C.byref(nm)) == 0
    return nm


def ref_noise(vol, win=5, pct=10.0, ref=0.5):
    nm = oracle.RefNoise()
    a = np.ascontiguousarray(vol, np.float32)
    assert oracle.ref().fy_estimate_noise(p(a), *a.shape, win, pct, ref, C.byref(nm)) == 0
    return nm


def close(a, b, rel=1e-3):
    return abs(a - b) <= rel * max(abs(b), 1e-12)


def test_noise_recipe(gpu):
    v1 = R.noise_input(0.05, 12345)
    v2 = R.noise_input(0.10, 999)
    g1, g2 = gpu_noise(gpu, v1), gpu_noise(gpu, v2)
    # test_fysics.c:402-420
    assert 0.5 * 0.05 < g1.noise_ref < 1.7 * 0.05
    assert g2.noise_ref > g1.noise_ref
    gold = ref_noise(v1) if oracle.have_ref() else None
    want = np.array([gold.g, gold.b, gold.noise_ref, gold.n_bins_used]) if gold else golden()["noise_model"]
    assert g1.n_bins_used == int(want[3])
    assert close(g1.noise_ref, want[2])
    o = o64_noise(v1)
    assert g1.n_bins_used == o.n_bins_used and close(g1.noise_ref, o.noise_ref)


@pytest.mark.parametrize("shape,win,pct", [((40, 50, 60), 5, 10.0), ((64, 64, 64), 3, 10.0),
                                           ((33, 47, 29), 7, 25.0), ((96, 96, 96), 5, 10.0),
                                           ((30, 30, 30), 9, 5.0), ((25, 25, 25), 2, 0.0)])
def test_noise_shapes(gpu, shape, win, pct):
    rng = np.random.default_rng(sum(shape) + win)
    z, y, x = np.meshgrid(*[np.linspace(0, 1, n) for n in shape], indexing="ij")
    sig = 0.3 + 0.5 * x * (0.5 + 0.5 * np.sin(3 * y + 2 * z))
    vol = (sig + rng.standard_normal(shape) * np.sqrt(0.002 * sig + 1e-4)).astype(np.float32)
    g = gpu_noise(gpu, vol, win, pct, 0.4)
    o = o64_noise(vol, win, pct, 0.4)
    assert g.n_bins_used == o.n_bins_used
    assert close(g.noise_ref, o.noise_ref)
    if oracle.have_ref():
        r = ref_noise(vol, win, pct, 0.4)
        assert g.n_bins_used == r.n_bins_used
        assert close(g.noise_ref, r.noise_ref)
        assert abs(g.g - r.g) <= 1e-3 * max(abs(r.g), abs(r.b) / 0.4, 1e-9)


def test_noise_fallbacks(gpu):
    """Few voxels per bin: 0 bins (whole-volume percentile) and 1-2 bins (flat model)."""
    rng = np.random.default_rng(1)
    tiny = (0.5 + 0.05 * rng.standard_normal((6, 6, 6))).astype(np.float32)      # 216 voxels: no bin >= 200
    g, o = gpu_noise(gpu, tiny), o64_noise(tiny)
    assert g.n_bins_used == o.n_bins_used == 0
    assert close(g.noise_ref, o.noise_ref) and g.g == 0.0
    two = np.concatenate([np.full((10, 10, 10), 0.2), np.full((10, 10, 10), 0.8)]).astype(np.float32)
    two += (0.01 * rng.standard_normal(two.shape)).astype(np.float32)
    g, o = gpu_noise(gpu, two), o64_noise(two)
    assert g.n_bins_used == o.n_bins_used
    assert close(g.noise_ref, o.noise_ref, 2e-3)


def test_noise_constant_volume(gpu):
    vol = np.full((20, 20, 20), 0.25, np.float32)
    g, o = gpu_noise(gpu, vol), o64_noise(vol)
    assert g.n_bins_used == o.n_bins_used
    assert abs(g.noise_ref - o.noise_ref) < 1e-4


def test_device_eps_chain(gpu):
    """fy_gpu_estimate_noise keeps the model on the device; eps = (3*noise_ref)^2."""
    import torch
    vol = R.noise_input(0.05, 12345)
    lib = gpu.load()
    d = torch.from_numpy(vol).cuda()
    scratch = torch.empty(lib.fy_gpu_noise_scratch_bytes(*vol.shape), dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    assert lib.fy_gpu_estimate_noise(C.c_void_p(d.data_ptr()), *vol.shape, 5, 10.0, 0.5,
                                     C.c_void_p(scratch.data_ptr()), None) == 0
    nm = gpu.NoiseModel()
    assert lib.fy_gpu_noise_model(C.c_void_p(scratch.data_ptr()), *vol.shape, C.byref(nm), None) == 0
    host = gpu_noise(gpu, vol)
    assert nm.noise_ref == host.noise_ref
    eps_ptr = lib.fy_gpu_noise_eps(C.c_void_p(scratch.data_ptr()), *vol.shape)
    off = eps_ptr - scratch.data_ptr()
    eps = scratch[off:off + 4].cpu().numpy().view(np.float32)[0]
    assert eps == np.float32(lib.fy_guided_eps_for_noise(host.noise_ref))


def test_noise_window_overflow_falls_back(gpu):
    """The mean percentiles come from a sample-guided window and a candidate list of n/8 +
    4096 entries. A volume whose low 60% is one constant ties the 1st percentile across far
    more voxels than that, so the window's candidate list overflows and the exact radix
    passes over the whole field run instead: the model must still equal the oracle's."""
    rng = np.random.default_rng(7)
    shape = (64, 64, 64)
    vol = np.full(shape, 0.1, np.float32)
    z, y, x = np.meshgrid(*[np.linspace(0, 1, s) for s in shape], indexing="ij")
    upper = z > 0.6
    sig = (0.3 + 0.5 * x * y)[upper]
    vol[upper] = (sig + rng.standard_normal(sig.shape) * np.sqrt(0.002 * sig + 1e-4)).astype(np.float32)
    g, o = gpu_noise(gpu, vol, 5, 10.0, 0.4), o64_noise(vol, 5, 10.0, 0.4)
    assert g.n_bins_used == o.n_bins_used
    assert close(g.noise_ref, o.noise_ref)
    if oracle.have_ref():
        r = ref_noise(vol, 5, 10.0, 0.4)
        assert g.n_bins_used == r.n_bins_used
        assert close(g.noise_ref, r.noise_ref)


def _paths_volume(shape, seed):
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid(*[np.linspace(0, 1, n) for n in shape], indexing="ij")
    sig = 0.3 + 0.5 * x * (0.5 + 0.5 * np.sin(3 * y + 2 * z))
    return (sig + rng.standard_normal(shape) * np.sqrt(0.002 * sig + 1e-4)).astype(np.float32)


@pytest.mark.parametrize("shape,win,pct", [((96, 96, 96), 5, 10.0), ((64, 80, 72), 3, 25.0),
                                           ((128, 128, 128), 5, 10.0), ((40, 50, 60), 7, 5.0)])
def test_noise_windows_equal_radix_paths(gpu, shape, win, pct):
    """Both order-statistic paths are exact, so the model must be bit-identical whether the
    sample-guided windows (one pass over the means, one over mean and variance) or the radix
    passes over the whole field find the 1st/99th mean percentiles and the per-bin variance
    percentiles; and on such volumes the windows are the path that normally runs."""
    _windows_vs_radix(gpu, _paths_volume(shape, sum(shape) + win), win, pct)


def test_noise_window_across_zero(gpu):
    """Means whose 1st percentile lies at 0: that window holds keys of both signs, a range of
    ~2^31 keys, so its candidates take all four offset digit passes (a narrow window takes
    two). The windows must still hold and equal the radix paths bit for bit."""
    rng = np.random.default_rng(23)
    vol = (1.0 + 0.1 * rng.standard_normal((96, 96, 96))).astype(np.float32)
    # a zero-mean slab: the means of its two middle planes (2.1% of the voxels, all of their
    # windows inside it) are the lowest, so the 1st percentile is about their median, 0
    vol[40:46] = rng.standard_normal((6, 96, 96)).astype(np.float32)
    _windows_vs_radix(gpu, vol, 5, 10.0)


def _windows_vs_radix(gpu, vol, win, pct):
    lib = gpu.load()
    used = C.c_int(-1)
    try:
        assert lib.fy_gpu_test_noise_paths(0, C.byref(used)) == 0
        base = gpu_noise(gpu, vol, win, pct, 0.4)
        assert lib.fy_gpu_test_noise_paths(0, C.byref(used)) == 0
        assert used.value == 3, used.value                    # both windows held their targets
        for force in (1, 2, 3):
            assert lib.fy_gpu_test_noise_paths(force, None) == 0
            got = gpu_noise(gpu, vol, win, pct, 0.4)
            assert lib.fy_gpu_test_noise_paths(0, C.byref(used)) == 0
            assert used.value == 3 & ~force, (force, used.value)
            assert (got.g, got.b, got.noise_ref, got.n_bins_used) == (base.g, base.b, base.noise_ref,
                                                                        base.n_bins_used), force
    finally:
        lib.fy_gpu_test_noise_paths(0, None)
    o = o64_noise(vol, win, pct, 0.4)
    assert base.n_bins_used == o.n_bins_used and close(base.noise_ref, o.noise_ref)
