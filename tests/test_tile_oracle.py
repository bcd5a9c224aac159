"""The per-tile chain's oracle (oracle/fy_oracle_tile.c) against the reference's own
fy_process_buffer (pipeline.c:252-510, compiled from its sources), on CPU.

Bars:
  * every stage that is integer or float-decision work (u8/255, rings, z drift, the
    decimated scratch smooth, histogram, valley, air cut, texture split, connected
    components, recenter, dithered quantiser) -- the u8 output equals the reference's
    bit for bit whenever the deconvolution and guided filter are off;
  * with those float stages on (FP64 in the oracle, float in the reference), at most
    MISMATCH_FRAC of the output voxels differ, each by at most one level;
  * the oracle's scratch smooth differs from the reference's only through the reference
    build's approximate reciprocals (< 4e-6 absolute), and its connected components equal
    scipy's.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from oracle import p
from tests._tiles import fill_dering, halo_box, ring_table, scroll_volume

pytestmark = pytest.mark.skipif(not oracle.have_ref(), reason="needs the compiled reference")

MISMATCH_FRAC = 2e-4
VOL = (80, 96, 96)
HALO = 8


@pytest.fixture(scope="module")
def vol():
    return scroll_volume(VOL, seed=11)


def tile_of(vol, tile0=(HALO, 24, 24), tsize=(64, 48, 48)):
    org, inner, sl = halo_box(vol.shape, tile0, tsize, HALO)
    return np.ascontiguousarray(vol[sl]), org, inner


INTEGER_CASES = {
    "air": dict(),
    "air_cc": dict(air_min_component=40),
    "air_cc_norm": dict(air_min_component=40, have_norm=1, norm_lo=50, norm_hi=190),
    "global_cut_aggr_lo": dict(air_cut_u8=60, air_cut_band=10, air_cut_aggr=0.4),
    "global_cut_aggr_hi": dict(air_cut_u8=60, air_cut_band=10, air_cut_aggr=1.6, air_thresh=0.12),
    "no_air_no_dither": dict(do_air_zero=0, no_dither=1),
    "scratch_passes_2": dict(scratch_passes=2, air_min_component=10),
    "norm_only": dict(do_air_zero=0, have_norm=1, norm_lo=30, norm_hi=220),
}


@pytest.mark.parametrize("name", sorted(INTEGER_CASES))
def test_integer_stages_bit_exact(vol, name):
    d = oracle.pipeline_defaults(**INTEGER_CASES[name])
    buf, org, inner = tile_of(vol)
    r, ra = oracle.ref_process_buffer(d, buf, org, inner, VOL[1:])
    o, oa = oracle.ot_process_buffer(d, buf, org, inner, VOL[1:])
    assert ra == oa == 0
    assert np.array_equal(r, o), np.count_nonzero(r != o)


@pytest.mark.parametrize("corner", ["origin", "far_edge", "tiny_full_res"])
def test_clamped_and_tiny_buffers_bit_exact(vol, corner):
    """Haloes clamped at the volume faces (asymmetric buffers) and a buffer too thin for the
    decimated scratch (the full-resolution branch, pipeline.c:324-328)."""
    d = oracle.pipeline_defaults(air_min_component=20)
    if corner == "origin":
        buf, org, inner = tile_of(vol, (0, 0, 0), (40, 40, 40))
    elif corner == "far_edge":
        buf, org, inner = tile_of(vol, (VOL[0] - 30, VOL[1] - 37, VOL[2] - 41), (30, 37, 41))
    else:
        buf, org, inner = vol[40:43, 30:70, 30:70].copy(), (40, 30, 30), (40, 30, 30, 3, 40, 40)
    r, _ = oracle.ref_process_buffer(d, buf, org, inner, VOL[1:])
    o, _ = oracle.ot_process_buffer(d, buf, org, inner, VOL[1:])
    assert np.array_equal(r, o), np.count_nonzero(r != o)


def test_rings_and_zdrift_bit_exact(vol):
    """Ring subtraction (dering.c:200-248 at scale 1/255) and z drift before the copy."""
    ring = ring_table(3, 70, seed=4)
    rd = fill_dering(oracle.RefDering(), ring, 32, 47.5, 47.5, VOL)
    zd = (1.0 + 0.04 * np.sin(np.arange(VOL[0]) / 7.0)).astype(np.float32)
    d = oracle.pipeline_defaults(have_dering=1, have_zdrift=1, air_min_component=25)
    buf, org, inner = tile_of(vol, (20, 16, 8), (50, 60, 70))
    r, _ = oracle.ref_process_buffer(d, buf, org, inner, VOL[1:], dering=rd, zdrift=zd)
    o, _ = oracle.ot_process_buffer(d, buf, org, inner, VOL[1:], ring=ring, ring_geo=(3, 70, 32, 47.5, 47.5),
                                    zdrift=zd)
    plain, _ = oracle.ot_process_buffer(oracle.pipeline_defaults(air_min_component=25), buf, org, inner, VOL[1:])
    assert not np.array_equal(o, plain)                 # the rings and drift changed the tile
    assert np.array_equal(r, o), np.count_nonzero(r != o)


def test_all_air_buffer():
    d = oracle.pipeline_defaults()
    buf = np.zeros((24, 24, 24), np.uint8)
    inner = (4, 4, 4, 16, 16, 16)
    r, ra = oracle.ref_process_buffer(d, buf, (0, 0, 0), inner, (24, 24))
    o, oa = oracle.ot_process_buffer(d, buf, (0, 0, 0), inner, (24, 24))
    assert ra == oa == 1 and not r.any() and not o.any()


FLOAT_CASES = {
    "guided_s2": dict(guided_eps=8e-4),
    "guided_exact": dict(guided_eps=8e-4, guided_subsample=1),
    "deconv_plain_guided": dict(do_deconv=1, use_matched_deconv=0, guided_eps=8e-4, window_lo=-0.02,
                                window_hi=0.3),
    "deconv_matched_guided_cc": dict(do_deconv=1, guided_eps=8e-4, window_lo=-0.02, window_hi=0.3,
                                     air_min_component=30, psf_z_ratio=1.17),
    "deconv_dec_range_norm": dict(do_deconv=1, guided_eps=8e-4, have_dec_range=1, dec_lo=0.05, dec_hi=0.9,
                                  have_norm=1, norm_lo=40, norm_hi=200),
    "radial_eps": dict(guided_eps=8e-4, have_eps_r=1, eps_fn_a=0.01, eps_fn_b=2e-4, eps_fn_med=0.012),
}


@pytest.mark.parametrize("name", sorted(FLOAT_CASES))
def test_float_stages_within_one_level(vol, name):
    d = oracle.pipeline_defaults(**FLOAT_CASES[name])
    buf, org, inner = tile_of(vol)
    r, _ = oracle.ref_process_buffer(d, buf, org, inner, VOL[1:])
    o, _ = oracle.ot_process_buffer(d, buf, org, inner, VOL[1:])
    diff = np.abs(r.astype(int) - o.astype(int))
    frac = np.count_nonzero(diff) / diff.size
    print(f"TILE {name}: {np.count_nonzero(diff)} of {diff.size} voxels differ, max {diff.max()}")
    assert frac <= MISMATCH_FRAC and diff.max() <= 1


def test_valley_depth_matches_reference():
    rng = np.random.default_rng(3)
    R, O = oracle.ref(), oracle.o64()
    x = np.arange(256)
    hists = [np.zeros(256, np.int64), np.full(256, 7, np.int64)]
    for k in range(60):
        h = 1e4 * np.exp(-0.5 * ((x - rng.uniform(10, 80)) / rng.uniform(3, 15)) ** 2)
        if k % 4:
            h += rng.uniform(0.1, 2) * 1e4 * np.exp(-0.5 * ((x - rng.uniform(90, 240)) / rng.uniform(3, 25)) ** 2)
        h += rng.poisson(20, 256) * (k % 3)
        hists.append(np.rint(h).astype(np.int64))
    for h in hists:
        outs = []
        for fn in (R.fy_valley_depth, O.ot_valley_depth):
            a, b, v = C.c_int(-9), C.c_int(-9), C.c_int(-9)
            dd = fn(p(h), C.byref(a), C.byref(b), C.byref(v))
            outs.append((dd, a.value, b.value, v.value))
        assert outs[0] == outs[1]


def test_box_smooth_close_to_reference():
    """The reference build vectorises box_recip (guided.c:22-28): vector lanes take an
    approximate reciprocal (one ulp low on the machines measured, and host-CPU dependent),
    the scalar tail an IEEE one; the oracle takes IEEE 1/count everywhere. The sliding sums
    are the same, so the two agree to a few 1e-7 and both sit on the FP64 box mean."""
    rng = np.random.default_rng(5)
    for shape, r in [((20, 33, 47), 1), ((40, 36, 36), 3), ((9, 50, 51), 5)]:
        a = (rng.integers(0, 256, shape).astype(np.float32) * np.float32(1 / 255))
        ref, tmp, o = np.empty_like(a), np.empty_like(a), np.empty_like(a)
        oracle.ref().fy_box_smooth(p(a), p(ref), p(tmp), *shape, r)
        oracle.o64().ot_box_smooth(p(a), p(o), *shape, r)
        assert np.abs(o - ref).max() < 4e-6
        exact = np.empty(shape, np.float64)
        a64 = a.astype(np.float64)
        oracle.o64().o64_box_mean(p(a64), p(exact), *shape, r)
        assert np.abs(o - exact).max() < 2e-6


def test_cc_despeckle_matches_scipy():
    """Zeroed voxels = 6-connected components of f > 0 that touch no face and have fewer
    than min_size voxels (pipeline.c:223-250)."""
    ndimage = pytest.importorskip("scipy.ndimage")
    rng = np.random.default_rng(9)
    for shape, density, min_size in [((30, 31, 32), 0.3, 5), ((16, 40, 24), 0.45, 40), ((8, 8, 8), 0.2, 3)]:
        f = (rng.random(shape) < density).astype(np.float32) * rng.uniform(0.1, 1, shape).astype(np.float32)
        got = f.copy()
        n = oracle.o64().ot_cc_despeckle(p(got), *shape, min_size)
        lab, k = ndimage.label(f > 0)
        sizes = np.bincount(lab.ravel(), minlength=k + 1)
        edge = np.zeros(k + 1, bool)
        for face in (lab[0], lab[-1], lab[:, 0], lab[:, -1], lab[:, :, 0], lab[:, :, -1]):
            edge[np.unique(face)] = True
        drop = (~edge) & (sizes < min_size)
        drop[0] = False
        want = np.where(drop[lab], 0, f).astype(np.float32)
        assert np.array_equal(got, want) and n == int(drop[lab].sum())


def test_product_valley_depth_is_host_math(fy):
    """fy_valley_depth is O(256) host arithmetic in the product library too (no device)."""
    lib = fy.load()
    x = np.arange(256)
    h = np.rint(5e3 * np.exp(-0.5 * ((x - 30) / 6) ** 2) + 3e3 * np.exp(-0.5 * ((x - 150) / 20) ** 2)).astype(np.int64)
    outs = []
    for fn in (lib.fy_valley_depth, oracle.ref().fy_valley_depth):
        a, b, v = C.c_int(), C.c_int(), C.c_int()
        outs.append((fn(p(h), C.byref(a), C.byref(b), C.byref(v)), a.value, b.value, v.value))
    assert outs[0] == outs[1] and outs[0][1] < outs[0][3] < outs[0][2]
