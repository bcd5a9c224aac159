"""Local zarr v2 input (zarr_io.c:133-331) on the CPU: the region-assembly rule restated in
numpy (tests/_zarr.py) is pinned against the reference's own fy_zarr_read on trees with edge
chunks of their true extent, missing chunks, short files, a nonzero fill value and regions
that reach past the volume; the product library's fy_zarr_open parses every header the way
the reference's does (same grammar, first key occurrence, first integer after it); and with
no GPU the product's fy_zarr_read refuses instead of assembling on the host."""
import ctypes as C

import numpy as np
import pytest

import oracle
from tests._zarr import expected_region, write_zarr, zarray_text
from tests.conftest import has_cuda

needs_ref = pytest.mark.skipif(not oracle.have_ref(), reason="reference library not built")

SHAPE = (37, 50, 45)
CHUNK = (16, 16, 16)
DROP = {(0, 1, 1), (2, 3, 2)}
TRUNC = {(1, 0, 0): 16 * 16 * 16 - 100, (0, 0, 2): 1000, (2, 2, 1): 0}
REGIONS = [(0, 0, 0, 37, 50, 45), (5, 7, 9, 20, 30, 25), (30, 40, 40, 16, 16, 16), (0, 0, 0, 1, 1, 1),
           (15, 15, 15, 3, 3, 3), (36, 49, 44, 4, 5, 6), (40, 0, 0, 3, 3, 3), (10, 10, 44, 5, 5, 20)]


def volume(seed=3):
    return np.random.default_rng(seed).integers(0, 256, SHAPE, dtype=np.uint8)


def ref_read(root, region):
    z = oracle.RefZarr()
    assert oracle.ref().fy_zarr_open(C.byref(z), str(root).encode()) == 0
    out = np.full(region[3:], 0xCD, np.uint8)
    assert oracle.ref().fy_zarr_read(C.byref(z), *region, oracle.p(out)) == 0
    return out


@needs_ref
@pytest.mark.parametrize("fill", [0, 7])
def test_reference_read_matches_restatement(tmp_path, fill):
    vol = volume()
    root = write_zarr(tmp_path / "v.zarr", vol, CHUNK, fill=fill, drop=DROP, truncate=TRUNC)
    for reg in REGIONS:
        want = expected_region(vol, CHUNK, reg, np.full(reg[3:], 0xCD, np.uint8), fill, DROP, TRUNC)
        assert np.array_equal(ref_read(root, reg), want), reg


HEADERS = {
    "standard": zarray_text((37, 50, 45), (16, 16, 16), 0),
    "fill": zarray_text((37, 50, 45), (16, 8, 32), 9),
    "pretty": '{\n  "chunks": [\n    16,\n    16,\n    16\n  ],\n  "compressor": null,\n  "dtype": "|u1",\n'
              '  "fill_value": 3,\n  "order": "C",\n  "shape": [\n    37,\n    50,\n    45\n  ],\n'
              '  "zarr_format": 2\n}',
    # null fill: the grammar takes the next integer in the text (here the shape's first)
    "fill_null": '{"fill_value":null,"order":"C","shape":[200,100,90],"chunks":[64,64,64],"zarr_format":2}',
    "negative": '{"shape":[-5,10,10],"chunks":[8,8,8],"fill_value":0}',
    "no_chunks": '{"shape":[10,10,10],"fill_value":0}',
}


@needs_ref
@pytest.mark.parametrize("name", sorted(HEADERS))
def test_open_header_grammar_matches_reference(fy, tmp_path, name):
    root = tmp_path / f"{name}.zarr"
    (root / "0").mkdir(parents=True)
    (root / "0" / ".zarray").write_text(HEADERS[name])
    g, r = fy.Zarr(), oracle.RefZarr()
    rc_g = fy.load().fy_zarr_open(C.byref(g), str(root).encode())
    rc_r = oracle.ref().fy_zarr_open(C.byref(r), str(root).encode())
    assert (rc_g == 0) == (rc_r == 0)
    if rc_r == 0:
        assert list(g.shape) == list(r.shape) and list(g.chunk) == list(r.chunk) and g.fill == r.fill
        assert g.root == r.root


def test_open_missing_and_s3(fy, tmp_path):
    z = fy.Zarr()
    assert fy.load().fy_zarr_open(C.byref(z), str(tmp_path / "absent.zarr").encode()) == 1
    assert fy.load().fy_zarr_open(C.byref(z), b"s3://bucket/volume.zarr") == 1
    assert b"S3" in fy.load().fy_gpu_last_error()


@pytest.mark.skipif(has_cuda(), reason="checks the behaviour without a GPU")
def test_read_refuses_without_gpu(fy, tmp_path):
    vol = volume()
    root = write_zarr(tmp_path / "v.zarr", vol, CHUNK)
    z = fy.Zarr()
    assert fy.load().fy_zarr_open(C.byref(z), str(root).encode()) == 0
    out = np.full((4, 4, 4), 0xCD, np.uint8)
    assert fy.load().fy_zarr_read(C.byref(z), 0, 0, 0, 4, 4, 4, out.ctypes.data) == fy.FY_ENODEV
    assert (out == 0xCD).all()
