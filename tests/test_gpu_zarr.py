"""Local zarr v2 input staged into the GPU (fy_zarr_read, fy_gpu_zarr_read, fy_process_chunk)
against the reference's fy_zarr_read (zarr_io.c:237-331) and fy_process_chunk
(pipeline.c:512-537).

Bars: region assembly is bit-exact (byte work): every region of every tree equals the
reference's, including missing chunks, short files, a nonzero fill value, regions reaching
past the volume (whose outside voxels keep the destination's contents) and regions of more
chunks than one gather launch takes. fy_process_chunk equals fy_process_buffer on the region
the reference reads (the same GPU chain), and the reference's fy_process_chunk within the
per-tile chain's bar (bit-exact with the deconvolution and guided filter off; otherwise at
most MISMATCH_FRAC of the voxels differ, by one level).
"""
import ctypes as C
import os
import threading

import numpy as np
import pytest

import oracle
from tests._tiles import gpu_cfg, scroll_volume
from tests._zarr import write_zarr
from tests.test_tile_oracle import MISMATCH_FRAC

pytestmark = pytest.mark.gpu
needs_ref = pytest.mark.skipif(not oracle.have_ref(), reason="reference library not built")

SHAPE = (37, 50, 45)
CHUNK = (16, 16, 16)
DROP = {(0, 1, 1), (2, 3, 2)}
TRUNC = {(1, 0, 0): 16 * 16 * 16 - 100, (0, 0, 2): 1000, (2, 2, 1): 0}
REGIONS = [(0, 0, 0, 37, 50, 45), (5, 7, 9, 20, 30, 25), (30, 40, 40, 16, 16, 16), (0, 0, 0, 1, 1, 1),
           (15, 15, 15, 3, 3, 3), (36, 49, 44, 4, 5, 6), (40, 0, 0, 3, 3, 3), (10, 10, 44, 5, 5, 20),
           (1, 2, 3, 36, 48, 42)]


def opened(fy, root):
    z = fy.Zarr()
    assert fy.load().fy_zarr_open(C.byref(z), str(root).encode()) == 0
    return z


def ref_read(root, region):
    z = oracle.RefZarr()
    assert oracle.ref().fy_zarr_open(C.byref(z), str(root).encode()) == 0
    out = np.full(region[3:], 0xCD, np.uint8)
    assert oracle.ref().fy_zarr_read(C.byref(z), *region, oracle.p(out)) == 0
    return out


def gpu_read(fy, z, region, pinned=False):
    import torch
    if pinned:
        t = torch.full(region[3:], 0xCD, dtype=torch.uint8, pin_memory=True)
        rc = fy.load().fy_zarr_read(C.byref(z), *region, t.data_ptr())
        return rc, t.numpy().copy()
    out = np.full(region[3:], 0xCD, np.uint8)
    rc = fy.load().fy_zarr_read(C.byref(z), *region, out.ctypes.data)
    return rc, out


@needs_ref
@pytest.mark.parametrize("fill,chunk", [(0, CHUNK), (7, CHUNK), (0, (8, 8, 8)), (3, (5, 16, 40))])
def test_read_bit_exact_vs_reference(gpu, tmp_path, fill, chunk):
    vol = np.random.default_rng(3).integers(0, 256, SHAPE, dtype=np.uint8)
    drop = DROP if chunk == CHUNK else {(1, 1, 1)}
    trunc = TRUNC if chunk == CHUNK else {(0, 0, 0): 17}
    root = write_zarr(tmp_path / "v.zarr", vol, chunk, fill=fill, drop=drop, truncate=trunc)
    z = opened(gpu, root)
    for i, reg in enumerate(REGIONS):
        rc, got = gpu_read(gpu, z, reg, pinned=bool(i & 1))
        assert rc == 0, gpu.load().fy_gpu_last_error()
        assert np.array_equal(got, ref_read(root, reg)), reg


@needs_ref
def test_device_read_keeps_outside_voxels(gpu, tmp_path):
    import torch
    vol = np.random.default_rng(5).integers(1, 256, SHAPE, dtype=np.uint8)
    root = write_zarr(tmp_path / "v.zarr", vol, (8, 8, 8), drop={(0, 0, 0)})
    z = opened(gpu, root)
    for reg in [(30, 40, 30, 10, 15, 20), (0, 0, 0, 37, 50, 45), (2, 3, 4, 9, 9, 9)]:
        d = torch.full(reg[3:], 0xCD, dtype=torch.uint8, device="cuda")     # 9x12x9 chunks: split launches
        torch.cuda.synchronize()
        assert gpu.load().fy_gpu_zarr_read(C.byref(z), *reg, C.c_void_p(d.data_ptr()), None) == 0
        torch.cuda.synchronize()
        assert np.array_equal(d.cpu().numpy(), ref_read(root, reg)), reg


def test_cache_sees_rewritten_chunk_and_counts(gpu, tmp_path):
    vol = np.random.default_rng(9).integers(0, 256, (32, 32, 32), dtype=np.uint8)
    root = write_zarr(tmp_path / "v.zarr", vol, (16, 16, 16))
    z = opened(gpu, root)
    lib = gpu.load()
    stats = [C.c_ulonglong() for _ in range(3)]
    lib.fy_gpu_zarr_cache_stats(*[C.byref(s) for s in stats])
    h0, l0 = stats[0].value, stats[1].value
    rc, a = gpu_read(gpu, z, (0, 0, 0, 32, 32, 32))
    assert rc == 0 and np.array_equal(a, vol)
    rc, b = gpu_read(gpu, z, (8, 8, 8, 16, 16, 16))              # all 8 chunks again: cache hits
    assert rc == 0 and np.array_equal(b, vol[8:24, 8:24, 8:24])
    lib.fy_gpu_zarr_cache_stats(*[C.byref(s) for s in stats])
    assert stats[1].value - l0 == 8 and stats[0].value - h0 == 8
    vol2 = vol.copy()
    vol2[16:, 16:, 16:] ^= 0x5A                                  # rewrite one chunk file
    path = tmp_path / "v.zarr" / "0" / "1" / "1" / "1"
    st = os.stat(path)
    path.write_bytes(np.ascontiguousarray(vol2[16:, 16:, 16:]).tobytes())
    os.utime(path, ns=(st.st_atime_ns, st.st_mtime_ns + 1_000_000))
    rc, c = gpu_read(gpu, z, (0, 0, 0, 32, 32, 32))
    assert rc == 0 and np.array_equal(c, vol2)
    path.unlink()                                                # and remove it: fill
    rc, d = gpu_read(gpu, z, (0, 0, 0, 32, 32, 32))
    vol3 = vol.copy()
    vol3[16:, 16:, 16:] = 0
    assert rc == 0 and np.array_equal(d, vol3)


def test_concurrent_readers_and_small_cache(gpu, tmp_path):
    """Eight host threads read overlapping regions through a cache smaller than the volume's
    chunks (16 MiB against 48 chunks of 512 KiB), so loads, waits for other threads' loads,
    evictions and reads that pin more chunks than the cache holds all interleave."""
    vol = np.random.default_rng(13).integers(0, 256, (256, 256, 384), dtype=np.uint8)
    root = write_zarr(tmp_path / "v.zarr", vol, (64, 64, 128))
    z = opened(gpu, root)
    lib = gpu.load()
    assert lib.fy_gpu_zarr_cache_limit(16 << 20) == 0
    errors = []
    rng = np.random.default_rng(1)
    regions = [(int(rng.integers(0, 200)), int(rng.integers(0, 170)), int(rng.integers(0, 270)), 60, 90, 120)
               for _ in range(64)]

    def worker(k):
        try:
            for reg in regions[k::8]:
                rc, got = gpu_read(gpu, z, reg)
                z0, y0, x0, dz, dy, dx = reg
                want = np.full((dz, dy, dx), 0xCD, np.uint8)
                sub = vol[z0:z0 + dz, y0:y0 + dy, x0:x0 + dx]
                want[:sub.shape[0], :sub.shape[1], :sub.shape[2]] = sub
                if rc != 0 or not np.array_equal(got, want):
                    errors.append((reg, rc))
        except Exception as exc:                                  # reported by the assertion below
            errors.append(repr(exc))

    try:
        th = [threading.Thread(target=worker, args=(k,)) for k in range(8)]
        for t in th:
            t.start()
        for t in th:
            t.join()
    finally:
        lib.fy_gpu_zarr_cache_limit(4 << 30)
    assert not errors, errors[:3]


@pytest.fixture(scope="module")
def band(tmp_path_factory):
    vol = scroll_volume((80, 160, 160), seed=21)
    root = write_zarr(tmp_path_factory.mktemp("band") / "band.zarr", vol, (64, 64, 64))
    return vol, root


CASES = {"integer": dict(air_min_component=30), "float": dict(guided_eps=8e-4, air_min_component=30),
         "deconv": dict(do_deconv=1, use_matched_deconv=0, guided_eps=8e-4, window_lo=-0.02, window_hi=1.05)}


@needs_ref
@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("tile0", [(0, 0, 0), (64, 64, 96)])
def test_process_chunk_vs_reference(gpu, band, name, tile0):
    vol, root = band
    lib = gpu.load()
    d = oracle.pipeline_defaults(halo=8, **CASES[name])
    tile = 64
    z = opened(gpu, root)
    cfg = gpu_cfg(gpu, d)
    out = np.full((tile,) * 3, 0xCD, np.uint8)
    tz, ty, tx, air = C.c_int(), C.c_int(), C.c_int(), C.c_int(-1)
    rc = lib.fy_process_chunk(C.byref(z), C.byref(cfg), *tile0, tile, out.ctypes.data, C.byref(tz), C.byref(ty),
                              C.byref(tx), C.byref(air))
    assert rc == 0, lib.fy_gpu_last_error()
    shp = (tz.value, ty.value, tx.value)
    got = out.ravel()[:int(np.prod(shp))].reshape(shp)
    # the same region through fy_process_buffer: identical (the same GPU chain)
    halo = 8
    org = tuple(max(0, t - halo) for t in tile0)
    end = tuple(min(n, t + s + halo) for n, t, s in zip(vol.shape, tile0, shp))
    buf = np.ascontiguousarray(vol[org[0]:end[0], org[1]:end[1], org[2]:end[2]])
    pb = np.full(shp, 0xCD, np.uint8)
    air2 = C.c_int(-1)
    assert lib.fy_process_buffer(C.byref(cfg), buf.ctypes.data, *org, *buf.shape, *tile0, *shp, *vol.shape[1:],
                                 pb.ctypes.data, C.byref(air2)) == 0
    assert np.array_equal(got, pb) and air.value == air2.value
    # against the reference's own fy_process_chunk on the same zarr
    rz = oracle.RefZarr()
    assert oracle.ref().fy_zarr_open(C.byref(rz), str(root).encode()) == 0
    rcfg = oracle.ref_pipeline_cfg(d)
    rout = np.full((tile,) * 3, 0xCD, np.uint8)
    rt = [C.c_int() for _ in range(3)]
    rair = C.c_int(-1)
    assert oracle.ref().fy_process_chunk(C.byref(rz), C.byref(rcfg), *tile0, tile, oracle.p(rout),
                                         *[C.byref(v) for v in rt], C.byref(rair)) == 0
    assert (rt[0].value, rt[1].value, rt[2].value) == shp and rair.value == air.value
    want = rout.ravel()[:int(np.prod(shp))].reshape(shp)
    diff = np.abs(got.astype(int) - want.astype(int))
    if name == "integer":
        assert np.array_equal(got, want), np.count_nonzero(diff)
    else:
        assert diff.max() <= 1 and np.count_nonzero(diff) <= MISMATCH_FRAC * diff.size
