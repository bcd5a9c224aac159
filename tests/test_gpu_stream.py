"""u8 dewindow / requantisation on the GPU: bit-exact against the reference CPU path."""
import numpy as np
import pytest

import oracle
from tests.test_oracle_pins import golden

pytestmark = pytest.mark.gpu

WINDOWS = [(-0.03, 0.21), (0.0, 1.0), (-1.5, 2.25), (0.1, 0.1000001), (1e-3, 7.0)]


def ref_dewindow(u8, lo, hi):
    if oracle.have_ref():
        return oracle.ref_u8_to_phys(u8, lo, hi)
    g = golden()
    i = [tuple(w) for w in g["dewindow_windows"]].index((lo, hi))
    return g["dewindow"][i][u8]


def ref_requant(v, lo, hi):
    if oracle.have_ref():
        return oracle.ref_phys_to_u8(v, lo, hi)
    g = golden()
    assert np.array_equal(v, g["requant_in"])
    i = [tuple(w) for w in g["dewindow_windows"]].index((lo, hi))
    return g["requant"][i]


@pytest.mark.parametrize("win", WINDOWS)
def test_dewindow_all_levels_bit_exact(gpu, win):
    u8 = np.arange(256, dtype=np.uint8)
    got = gpu.u8_to_phys(u8, *win)
    assert np.array_equal(got.view(np.uint32), ref_dewindow(u8, *win).view(np.uint32))


def test_dewindow_random_windows_and_sizes(gpu):
    if not oracle.have_ref():
        pytest.skip("random windows need the reference library")
    rng = np.random.default_rng(3)
    for n in (1, 15, 16, 17, 1000, 1 << 20):
        u8 = rng.integers(0, 256, n, dtype=np.uint8)
        lo, hi = sorted(rng.uniform(-2, 2, 2))
        got = gpu.u8_to_phys(u8, lo, hi)
        assert np.array_equal(got.view(np.uint32), oracle.ref_u8_to_phys(u8, lo, hi).view(np.uint32))


@pytest.mark.parametrize("win", WINDOWS)
def test_requant_bit_exact(gpu, win):
    v = np.random.default_rng(7).uniform(-0.5, 1.5, 4096).astype(np.float32)
    assert np.array_equal(gpu.phys_to_u8(v, *win), ref_requant(v, *win))


def test_dewindow_roundtrip_kat(gpu):
    """test_fysics.c:439-453: u8 -> phys -> u8 exact for all levels, endpoints 1e-6."""
    f0, f1 = -0.03, 0.21
    u8 = np.arange(256, dtype=np.uint8)
    phys = gpu.u8_to_phys(u8, f0, f1)
    assert np.array_equal(gpu.phys_to_u8(phys, f0, f1), u8)
    assert abs(phys[0] - f0) < 1e-6 and abs(phys[255] - f1) < 1e-6


def test_unit_conversions_bit_exact(gpu):
    if not oracle.have_ref():
        pytest.skip("needs the reference library")
    import ctypes as C
    u8 = np.arange(256, dtype=np.uint8)
    r = np.empty(256, np.float32)
    oracle.ref().fy_u8_to_float(oracle.p(u8), oracle.p(r), 256)
    assert np.array_equal(gpu.u8_to_float(u8).view(np.uint32), r.view(np.uint32))
    v = np.random.default_rng(1).uniform(-0.2, 1.2, 100003).astype(np.float32)
    ru = np.empty(v.size, np.uint8)
    oracle.ref().fy_float_to_u8(oracle.p(v), oracle.p(ru), v.size)
    assert np.array_equal(gpu.float_to_u8(v), ru)
    del C
