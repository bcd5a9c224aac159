"""The FP64 oracle's calibration statistics against the compiled reference (CPU only).

fy_hist_accumulate_u8 counts must match exactly. fy_flat_noise and fy_noise_aniso sum in
FP64; the -Ofast reference may reorder those sums, so they agree to 1e-12 relative, and the
return codes exactly.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from oracle import o64, p

pytestmark = pytest.mark.skipif(not oracle.have_ref(), reason="needs the compiled reference")


def calib_volume(shape, seed, zero_slab=True):
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid(*[np.linspace(0, 1, n) for n in shape], indexing="ij")
    sig = 0.05 + 0.6 * (x > 0.3) * (0.5 + 0.5 * np.sin(4 * y + 3 * z))
    v = sig + rng.standard_normal(shape) * np.sqrt(0.002 * sig + 1e-4)
    if zero_slab:
        v[:, :, : shape[2] // 6] = 0.0                      # a masked region: blocks skipped
    return v.astype(np.float32)


def test_hist_matches_reference():
    rng = np.random.default_rng(1)
    for n in (0, 1, 15, 17, 100003):
        u = rng.integers(0, 256, n).astype(np.uint8)
        h = oracle.RefHist()
        oracle.ref().fy_hist_init(C.byref(h))
        oracle.ref().fy_hist_accumulate_u8(C.byref(h), p(u), n)
        mine = np.zeros(256, np.int64)
        o64().o64_hist_u8(p(u), n, p(mine))
        assert np.array_equal(np.array(h.hist[:]), mine) and h.total == n


@pytest.mark.parametrize("shape,blk", [((48, 40, 56), 8), ((64, 64, 64), 4), ((33, 47, 29), 6), ((7, 7, 7), 8)])
def test_flat_noise_matches_reference(shape, blk):
    v = calib_volume(shape, sum(shape))
    a = oracle.ref().fy_flat_noise(p(v), *shape, blk)
    b = o64().o64_flat_noise(p(v), *shape, blk)
    assert abs(a - b) <= 1e-12 * max(abs(a), 1e-300)


@pytest.mark.parametrize("shape", [(48, 40, 56), (64, 64, 64), (40, 40, 40), (16, 16, 16)])
def test_noise_aniso_matches_reference(shape):
    v = calib_volume(shape, 7 + sum(shape))
    rz, rx, oz, ox = C.c_double(), C.c_double(), C.c_double(), C.c_double()
    ra = oracle.ref().fy_noise_aniso(p(v), *shape, C.byref(rz), C.byref(rx))
    rb = o64().o64_noise_aniso(p(v), *shape, C.byref(oz), C.byref(ox))
    assert ra == rb
    if ra == 0:
        assert abs(rz.value - oz.value) <= 1e-12 * abs(rz.value)
        assert abs(rx.value - ox.value) <= 1e-12 * abs(rx.value)


def test_hist_host_bookkeeping_matches_reference(fy):
    """fy_hist_init / merge / percentile* are host O(256) work: same answers as the reference."""
    lib = fy.load()
    rng = np.random.default_rng(2)
    for n in (1, 15, 4096, 50000):
        u = rng.integers(0, 256, n).astype(np.uint8)
        u[: n // 4] = 0
        r = oracle.RefHist()
        oracle.ref().fy_hist_init(C.byref(r))
        for _ in range(2):
            oracle.ref().fy_hist_accumulate_u8(C.byref(r), p(u), n)
        h = fy.HistState()
        lib.fy_hist_init(C.byref(h))
        h.hist[:] = r.hist[:]
        h.total = r.total
        m = fy.HistState()
        lib.fy_hist_init(C.byref(m))
        lib.fy_hist_merge(C.byref(m), C.byref(h))
        assert np.array_equal(np.array(m.hist[:]), np.array(h.hist[:])) and m.total == h.total
        for pct in (0.0, 0.5, 10.0, 50.0, 99.5, 100.0):
            assert lib.fy_hist_percentile_u8(C.byref(h), pct) == oracle.ref().fy_hist_percentile_u8(C.byref(r), pct)
            assert (lib.fy_hist_percentile_u8_inner(C.byref(h), pct)
                    == oracle.ref().fy_hist_percentile_u8_inner(C.byref(r), pct))


@pytest.mark.parametrize("case", range(9))
def test_psf_sigma_oracle_vs_reference(case):
    """measure_tile_psf_sigma (pipeline.c:107-196), static in the reference, through the shim:
    the profile count exactly, sigma within 1e-12 relative (the reference build vectorises
    the final sums). Covers y-only, x-only and mixed edges, and tiles too thin for one axis
    (12 voxels) or both."""
    from tests._tiles import PSF_CASES, psf_volume
    shape, sigma, orient, noise = PSF_CASES[case]
    R = oracle.ref_psf()
    if R is None:
        pytest.skip("needs the compiled reference")
    v = psf_volume(shape, sigma, orient, noise, 7)
    n = C.c_int(-1)
    got = oracle.o64().ot_measure_psf_sigma(oracle.p(v), *shape, C.byref(n))
    want = R.ref_measure_tile_psf_sigma(oracle.p(v), *shape)
    assert abs(got - want) <= 1e-12 * max(abs(want), 1.0), (got, want, n.value)
    if shape[1] > 14 or shape[2] > 14:
        assert n.value > 0
    else:
        assert n.value == 0 and got == -1.0
