"""Ring removal on the GPU: bin sums/counts, ring-vote results and detected radii
bit-exact against the reference; apply within FP32 rounding of the reference."""
import ctypes as C

import numpy as np
import pytest

import oracle
from oracle import o64, p
from tests import _recipes as R
from tests.test_oracle_pins import golden

pytestmark = pytest.mark.gpu


def run_gpu(fy, vol, cy=-1.0, cx=-1.0, slab_z=64, ns=8, ss=1, fin=(15, 50, 2.0, 15.0), tiles=None):
    lib = fy.load()
    nz, ny, nx = vol.shape
    d, t = fy.Dering(), fy.Dering()
    assert lib.fy_dering_init(C.byref(d), nz, ny, nx, cy, cx, slab_z, ns) == 0
    assert lib.fy_dering_tile_init(C.byref(t), C.byref(d)) == 0
    for (z0, y0, x0, dz, dy, dx) in (tiles or [(0, 0, 0, nz, ny, nx)]):
        sub = np.ascontiguousarray(vol[z0:z0 + dz, y0:y0 + dy, x0:x0 + dx])
        lib.fy_dering_accumulate_u8(C.byref(t), p(sub), y0, x0, dz, dy, dx, ss)
        fy.check_void("fy_dering_accumulate_u8")
    lib.fy_dering_merge_tile(C.byref(d), 0, C.byref(t))
    det = lib.fy_dering_finalize(C.byref(d), *fin)
    return lib, d, t, det


def arrays(d):
    nb = d.nslab * d.ns * d.nr
    return (np.ctypeslib.as_array(d.sum, shape=(nb,)).copy(), np.ctypeslib.as_array(d.cnt, shape=(nb,)).copy(),
            np.ctypeslib.as_array(d.ring, shape=(d.nslab * d.nr,)).copy())


def run_ref(vol, cy=-1.0, cx=-1.0, slab_z=64, ns=8, ss=1, fin=(15, 50, 2.0, 15.0), tiles=None):
    L = oracle.ref()
    nz, ny, nx = vol.shape
    d, t = oracle.RefDering(), oracle.RefDering()
    assert L.fy_dering_init(C.byref(d), nz, ny, nx, cy, cx, slab_z, ns) == 0
    assert L.fy_dering_tile_init(C.byref(t), C.byref(d)) == 0
    for (z0, y0, x0, dz, dy, dx) in (tiles or [(0, 0, 0, nz, ny, nx)]):
        sub = np.ascontiguousarray(vol[z0:z0 + dz, y0:y0 + dy, x0:x0 + dx])
        L.fy_dering_accumulate_u8(C.byref(t), p(sub), y0, x0, dz, dy, dx, ss)
    L.fy_dering_merge_tile(C.byref(d), 0, C.byref(t))
    det = L.fy_dering_finalize(C.byref(d), *fin)
    return L, d, t, det


def test_dering_recipe(gpu):
    vol, cy, cx = R.dering_input()
    lib, d, t, det = run_gpu(gpu, vol)
    s, c, ring = arrays(d)
    if oracle.have_ref():
        L, rd, rt, rdet = run_ref(vol)
        rs, rc, rring = arrays(rd)
        assert det == rdet
    else:
        g = golden()["dering"]
        nr = d.nr
        rring, rc, rs = g[:nr], g[nr:nr + 8 * nr], g[nr + 8 * nr:]
    assert np.array_equal(c, rc) and np.array_equal(s, rs)            # bit-exact sums/counts
    assert np.array_equal(np.nonzero(ring)[0], np.nonzero(rring)[0])   # detected radii
    # Vote values: the -Ofast reference divides sum/cnt with a vectorised reciprocal +
    # Newton step (<= 2 ulp), so values agree to ~1e-5 u8, not bit for bit.
    assert np.abs(ring - rring).max() < 1e-4
    # reference test bars (test_fysics.c:150-161)
    assert d.have_rings and max(ring[59:62], key=abs) > 4.0 and max(ring[109:112], key=abs) < -3.0
    # apply: removes > 60% of the ring amplitude, matches the reference's float result
    f = (vol * np.float32(1.0 / 255.0)).astype(np.float32)
    lib.fy_dering_apply(C.byref(d), p(f), 0, 0, 0, *vol.shape, 1.0 / 255.0)
    gpu.check_void("fy_dering_apply")
    if oracle.have_ref():
        fr = (vol * np.float32(1.0 / 255.0)).astype(np.float32)
        L.fy_dering_apply(C.byref(rd), p(fr), 0, 0, 0, *vol.shape, 1.0 / 255.0)
        assert np.abs(f - fr).max() <= 1e-7
        L.fy_dering_free(C.byref(rt)); L.fy_dering_free(C.byref(rd))
    else:
        assert np.abs(f[0] - golden()["dering_apply_slice0"]).max() <= 1e-7
    lib.fy_dering_free(C.byref(t)); lib.fy_dering_free(C.byref(d))


@pytest.mark.parametrize("cy,cx,ss", [(-1.0, -1.0, 2), (120.3, 131.7, 1), (100.0, 90.5, 3)])
def test_dering_tiles_centers_subsample(gpu, cy, cx, ss):
    if not oracle.have_ref():
        pytest.skip("needs the reference library")
    vol, _, _ = R.dering_input()
    tiles = [(0, 0, 0, 32, 128, 256), (0, 128, 0, 32, 128, 130), (0, 128, 130, 32, 128, 126)]
    lib, d, t, det = run_gpu(gpu, vol, cy, cx, ss=ss, tiles=tiles, fin=(15, 20, 1.0, 15.0))
    L, rd, rt, rdet = run_ref(vol, cy, cx, ss=ss, tiles=tiles, fin=(15, 20, 1.0, 15.0))
    s, c, ring = arrays(d)
    rs, rc, rring = arrays(rd)
    assert np.array_equal(c, rc) and np.array_equal(s, rs)
    assert det == rdet and np.array_equal(np.nonzero(ring)[0], np.nonzero(rring)[0])
    assert np.abs(ring - rring).max() < 1e-4
    for h, lb in ((t, lib), (d, lib)):
        lb.fy_dering_free(C.byref(h))
    L.fy_dering_free(C.byref(rt)); L.fy_dering_free(C.byref(rd))


def test_dering_finalize_defaults_and_slabs(gpu):
    if not oracle.have_ref():
        pytest.skip("needs the reference library")
    vol, _, _ = R.dering_input()
    lib, L = gpu.load(), oracle.ref()
    nz, ny, nx = vol.shape
    d, rd = gpu.Dering(), oracle.RefDering()
    lib.fy_dering_init(C.byref(d), nz, ny, nx, -1, -1, 16, 6)
    L.fy_dering_init(C.byref(rd), nz, ny, nx, -1, -1, 16, 6)
    for slab in range(2):
        t, rt = gpu.Dering(), oracle.RefDering()
        lib.fy_dering_tile_init(C.byref(t), C.byref(d)); L.fy_dering_tile_init(C.byref(rt), C.byref(rd))
        sub = np.ascontiguousarray(vol[16 * slab:16 * slab + 16])
        lib.fy_dering_accumulate_u8(C.byref(t), p(sub), 0, 0, 16, ny, nx, 2)
        L.fy_dering_accumulate_u8(C.byref(rt), p(sub), 0, 0, 16, ny, nx, 2)
        lib.fy_dering_merge_tile(C.byref(d), slab, C.byref(t)); L.fy_dering_merge_tile(C.byref(rd), slab, C.byref(rt))
        lib.fy_dering_free(C.byref(t)); L.fy_dering_free(C.byref(rt))
    assert lib.fy_dering_finalize(C.byref(d), 0, 10, 0.0, 0.0) == L.fy_dering_finalize(C.byref(rd), 0, 10, 0.0, 0.0)
    ring, rring = arrays(d)[2], arrays(rd)[2]
    assert np.array_equal(np.nonzero(ring)[0], np.nonzero(rring)[0]) and d.have_rings == rd.have_rings
    assert np.abs(ring - rring).max() < 1e-4
    f = (vol * np.float32(1 / 255.0)).astype(np.float32)
    fr = f.copy()
    lib.fy_dering_apply(C.byref(d), p(f), 0, 0, 0, nz, ny, nx, 1 / 255.0)
    L.fy_dering_apply(C.byref(rd), p(fr), 0, 0, 0, nz, ny, nx, 1 / 255.0)
    assert np.abs(f - fr).max() <= 1e-7
    lib.fy_dering_free(C.byref(d)); L.fy_dering_free(C.byref(rd))


def test_device_handle_matches_host_path(gpu):
    import torch
    vol, _, _ = R.dering_input()
    nz, ny, nx = vol.shape
    lib = gpu.load()
    h = C.c_void_p()
    assert lib.fy_gpu_dering_create(C.byref(h), nz, ny, nx, -1, -1, 64, 8) == 0
    dv = torch.from_numpy(vol).cuda()
    torch.cuda.synchronize()
    assert lib.fy_gpu_dering_accumulate_u8(h, C.c_void_p(dv.data_ptr()), 0, 0, 0, nz, ny, nx, 1, None) == 0
    assert lib.fy_gpu_dering_finalize(h, 15, 50, 2.0, 15.0, None) == 0
    d = gpu.Dering()
    lib.fy_dering_init(C.byref(d), nz, ny, nx, -1, -1, 64, 8)
    det = C.c_long()
    assert lib.fy_gpu_dering_download(h, C.byref(d), C.byref(det), None) == 0
    _, hd, ht, hdet = run_gpu(gpu, vol)
    assert det.value == hdet and d.have_rings == hd.have_rings
    for a, b in zip(arrays(d), arrays(hd)):
        assert np.array_equal(a, b)
    f = torch.from_numpy((vol * np.float32(1 / 255.0)).astype(np.float32)).cuda()
    torch.cuda.synchronize()
    assert lib.fy_gpu_dering_apply(h, C.c_void_p(f.data_ptr()), 0, 0, 0, nz, ny, nx, 1 / 255.0, None) == 0
    fh = (vol * np.float32(1 / 255.0)).astype(np.float32)
    lib.fy_dering_apply(C.byref(hd), p(fh), 0, 0, 0, nz, ny, nx, 1 / 255.0)
    torch.cuda.synchronize()
    assert np.array_equal(f.cpu().numpy(), fh)
    lib.fy_gpu_dering_destroy(h)
    for x in (d, hd, ht):
        lib.fy_dering_free(C.byref(x))
