"""The per-tile chain on the GPU (fy_process_buffer / fy_gpu_process_buffer) against the
oracle restatement and the reference's own fy_process_buffer (pipeline.c:252-510).

Bars: with the deconvolution and guided filter off, the u8 tile and the air-cut state
(histogram, cuts) equal the oracle's bit for bit, and the reference's tile too; with
them on, at most MISMATCH_FRAC of the voxels differ by one level from either.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from tests._tiles import fill_dering, gpu_cfg, gpu_process_buffer, halo_box, ring_table, scroll_volume
from tests.test_tile_oracle import FLOAT_CASES, HALO, INTEGER_CASES, MISMATCH_FRAC, VOL, tile_of

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def vol():
    return scroll_volume(VOL, seed=11)


def air_state(lib):
    hist = np.zeros(256, np.int64)
    cuts = np.zeros(3, np.int32)
    rc = lib.fy_process_buffer_air_state(hist.ctypes.data, cuts.ctypes.data)
    return rc, hist, cuts


@pytest.mark.parametrize("name", sorted(INTEGER_CASES))
def test_integer_stages_bit_exact(gpu, vol, name):
    d = oracle.pipeline_defaults(**INTEGER_CASES[name])
    buf, org, inner = tile_of(vol)
    rc, g, ga = gpu_process_buffer(gpu, d, buf, org, inner, VOL[1:])
    assert rc == 0, gpu.load().fy_gpu_last_error()
    o, oa, hist, cuts = oracle.ot_process_buffer(d, buf, org, inner, VOL[1:], state=True)
    assert ga == oa == 0
    assert np.array_equal(g, o), np.count_nonzero(g != o)
    if d["do_air_zero"]:
        src, gh, gc = air_state(gpu.load())
        assert src == 0 and np.array_equal(gh, hist) and np.array_equal(gc, cuts)
    if oracle.have_ref():
        r, _ = oracle.ref_process_buffer(d, buf, org, inner, VOL[1:])
        assert np.array_equal(g, r), np.count_nonzero(g != r)


@pytest.mark.parametrize("corner", ["origin", "far_edge", "tiny_full_res", "odd"])
def test_clamped_and_tiny_buffers(gpu, vol, corner):
    d = oracle.pipeline_defaults(air_min_component=20)
    if corner == "origin":
        buf, org, inner = tile_of(vol, (0, 0, 0), (40, 40, 40))
    elif corner == "far_edge":
        buf, org, inner = tile_of(vol, (VOL[0] - 30, VOL[1] - 37, VOL[2] - 41), (30, 37, 41))
    elif corner == "odd":
        buf, org, inner = tile_of(vol, (17, 29, 31), (33, 19, 45))
    else:
        buf, org, inner = vol[40:43, 30:70, 30:70].copy(), (40, 30, 30), (40, 30, 30, 3, 40, 40)
    rc, g, _ = gpu_process_buffer(gpu, d, buf, org, inner, VOL[1:])
    assert rc == 0, gpu.load().fy_gpu_last_error()
    o, _ = oracle.ot_process_buffer(d, buf, org, inner, VOL[1:])
    assert np.array_equal(g, o), np.count_nonzero(g != o)


def test_rings_and_zdrift_bit_exact(gpu, vol):
    ring = ring_table(3, 70, seed=4)
    gd = fill_dering(gpu.Dering(), ring, 32, 47.5, 47.5, VOL)
    zd = (1.0 + 0.04 * np.sin(np.arange(VOL[0]) / 7.0)).astype(np.float32)
    d = oracle.pipeline_defaults(have_dering=1, have_zdrift=1, air_min_component=25)
    buf, org, inner = tile_of(vol, (20, 16, 8), (50, 60, 70))
    rc, g, _ = gpu_process_buffer(gpu, d, buf, org, inner, VOL[1:], dering=gd, zdrift=zd)
    assert rc == 0, gpu.load().fy_gpu_last_error()
    o, _ = oracle.ot_process_buffer(d, buf, org, inner, VOL[1:], ring=ring, ring_geo=(3, 70, 32, 47.5, 47.5),
                                    zdrift=zd)
    assert np.array_equal(g, o), np.count_nonzero(g != o)


@pytest.mark.parametrize("name", sorted(FLOAT_CASES))
def test_float_stages_within_one_level(gpu, vol, name):
    d = oracle.pipeline_defaults(**FLOAT_CASES[name])
    buf, org, inner = tile_of(vol)
    rc, g, _ = gpu_process_buffer(gpu, d, buf, org, inner, VOL[1:])
    assert rc == 0, gpu.load().fy_gpu_last_error()
    refs = {"oracle": oracle.ot_process_buffer(d, buf, org, inner, VOL[1:])[0]}
    if oracle.have_ref():
        refs["reference"] = oracle.ref_process_buffer(d, buf, org, inner, VOL[1:])[0]
    for who, r in refs.items():
        diff = np.abs(g.astype(int) - r.astype(int))
        print(f"TILE {name} vs {who}: {np.count_nonzero(diff)} of {diff.size} differ, max {diff.max()}")
        assert np.count_nonzero(diff) / diff.size <= MISMATCH_FRAC and diff.max() <= 1


def test_all_air_and_errors(gpu):
    lib = gpu.load()
    d = oracle.pipeline_defaults(do_musica=1)
    buf = np.zeros((24, 24, 24), np.uint8)
    rc, g, air = gpu_process_buffer(gpu, d, buf, (0, 0, 0), (4, 4, 4, 16, 16, 16), (24, 24))
    assert rc == 0 and air == 1 and not g.any()          # empty: zeros before anything else
    assert air_state(lib)[0] == 1
    buf[3, 5, 7] = 9
    rc, _, _ = gpu_process_buffer(gpu, d, buf, (0, 0, 0), (4, 4, 4, 16, 16, 16), (24, 24))
    assert rc == gpu.FY_EUNSUPPORTED                     # MUSICA is not on this path
    d = oracle.pipeline_defaults()
    rc, _, _ = gpu_process_buffer(gpu, d, buf, (0, 0, 0), (4, 4, 4, 16, 16, 21), (24, 24))
    assert rc == gpu.FY_EINVAL                           # inner tile leaves the buffer
    rc, _, _ = gpu_process_buffer(gpu, d, buf, (10, 0, 0), (4, 4, 4, 16, 16, 16), (24, 24))
    assert rc == gpu.FY_EINVAL


def test_device_form_equals_host_form(gpu, vol):
    import torch
    lib = gpu.load()
    d = oracle.pipeline_defaults(guided_eps=8e-4, air_min_component=30, have_norm=1, norm_lo=40, norm_hi=200)
    buf, org, inner = tile_of(vol)
    rc, host, _ = gpu_process_buffer(gpu, d, buf, org, inner, VOL[1:])
    assert rc == 0
    tz, ty, tx = inner[3:]
    db = torch.from_numpy(buf).cuda()
    dout = torch.zeros((tz, ty, tx), dtype=torch.uint8, device="cuda")
    st = torch.cuda.Stream()
    torch.cuda.synchronize()
    cfg = gpu_cfg(gpu, d)
    air = C.c_int(-1)
    rc = lib.fy_gpu_process_buffer(C.byref(cfg), C.c_void_p(db.data_ptr()), *org, *buf.shape, *inner, *VOL[1:],
                                   C.c_void_p(dout.data_ptr()), C.byref(air), C.c_void_p(st.cuda_stream))
    assert rc == 0 and air.value == 0
    assert np.array_equal(dout.cpu().numpy(), host)


def test_export_tile_size(gpu):
    """The export tool's shape: a 128^3 inner tile with an 8-voxel halo (144^3 buffer)."""
    v = scroll_volume((144, 160, 160), seed=21)
    org, inner, sl = halo_box(v.shape, (8, 16, 16), (128, 128, 128), HALO)
    buf = np.ascontiguousarray(v[sl])
    d = oracle.pipeline_defaults(air_min_component=50, have_norm=1, norm_lo=40, norm_hi=200)
    rc, g, _ = gpu_process_buffer(gpu, d, buf, org, inner, (160, 160))
    assert rc == 0, gpu.load().fy_gpu_last_error()
    o, _ = oracle.ot_process_buffer(d, buf, org, inner, (160, 160))
    assert np.array_equal(g, o), np.count_nonzero(g != o)


def test_wide_thin_buffer(gpu):
    """A thin buffer with wide planes: rows of 212 voxels end in a partial warp."""
    v = scroll_volume((24, 210, 212), seed=33)
    d = oracle.pipeline_defaults(air_min_component=40, have_norm=1, norm_lo=40, norm_hi=200)
    inner = (4, 4, 4, 16, 202, 204)
    rc, g, _ = gpu_process_buffer(gpu, d, v, (0, 0, 0), inner, (210, 212))
    assert rc == 0, gpu.load().fy_gpu_last_error()
    o, _ = oracle.ot_process_buffer(d, v, (0, 0, 0), inner, (210, 212))
    assert np.array_equal(g, o), np.count_nonzero(g != o)


def test_rows_over_one_cta(gpu):
    """Rows longer than 1024 voxels span several CTAs: run heads are per row segment and the
    union joins runs across the segment boundaries."""
    v = scroll_volume((8, 24, 1100), seed=44, specks_per_mvox=4000)
    d = oracle.pipeline_defaults(air_min_component=30, have_norm=1, norm_lo=40, norm_hi=200)
    inner = (2, 2, 2, 4, 20, 1096)
    rc, g, _ = gpu_process_buffer(gpu, d, v, (0, 0, 0), inner, (24, 1100))
    assert rc == 0, gpu.load().fy_gpu_last_error()
    o, _ = oracle.ot_process_buffer(d, v, (0, 0, 0), inner, (24, 1100))
    assert np.array_equal(g, o), np.count_nonzero(g != o)
