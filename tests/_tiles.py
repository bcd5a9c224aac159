"""Seeded haloed tiles and settings for the per-tile chain (fy_process_buffer).

The volumes are fysics_b200.phantom.scroll_volume: noisy air around a cylindrical body of
papyrus wraps, bright specks in the air (the islands the connected-component despeckle
removes) and an exactly-zero masked slab, so the air-cut histogram has two modes and a
valley, as on the volumes the export tool processes.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from fysics_b200.phantom import scroll_volume  # noqa: F401  (re-exported for the tests)


def halo_box(vol_shape, tile0, tsize, halo):
    """(org, inner, slices) of the haloed buffer around the inner tile, clamped to the volume
    as the export tool does (mca_export.c:643-648)."""
    org, sl = [], []
    for d in range(3):
        a = max(0, tile0[d] - halo)
        b = min(vol_shape[d], tile0[d] + tsize[d] + halo)
        org.append(a)
        sl.append(slice(a, b))
    return tuple(org), (*tile0, *tsize), tuple(sl)


def ring_table(nslab, nr, seed=0):
    """A detected-ring profile [nslab][nr] in u8 units: a few rings of +-1..4 levels."""
    rng = np.random.default_rng(seed)
    t = np.zeros((nslab, nr), np.float32)
    for _ in range(max(2, nr // 12)):
        ri = rng.integers(2, nr)
        t[:, ri] = rng.uniform(1, 4) * rng.choice([-1, 1])
    return t


def fill_dering(dstruct, ring, slab_z, cy, cx, shape):
    """Point a fy_dering-layout ctypes struct at `ring` (kept alive by the caller)."""
    dstruct.Z, dstruct.Y, dstruct.X = shape
    dstruct.cy, dstruct.cx = cy, cx
    dstruct.slab_z, dstruct.nslab, dstruct.ns, dstruct.nr = slab_z, ring.shape[0], 16, ring.shape[1]
    dstruct.ring = ring.ctypes.data_as(C.POINTER(C.c_float))
    dstruct.have_rings = 1
    return dstruct


def gpu_cfg(fb, d: dict, dering=None, zdrift=None):
    """fy_pipeline_cfg of the product library from a cfg dict (oracle.pipeline_defaults)."""
    c = fb.PipelineCfg()
    for n, _ in fb.PipelineCfg._fields_:
        if n in ("zdrift_factor", "dering", "occ"):
            continue
        setattr(c, n, d.get(n, 0))
    if zdrift is not None:
        c.zdrift_factor = zdrift.ctypes.data_as(C.POINTER(C.c_float))
    if dering is not None:
        c.dering = C.cast(C.pointer(dering), C.c_void_p).value
    return c


def gpu_process_buffer(fb, d: dict, u8, org, inner, vol_yx, dering=None, zdrift=None):
    """fy_process_buffer of the product library; returns (rc, out, all_air)."""
    lib = fb.load()
    u8 = np.ascontiguousarray(u8, np.uint8)
    z0, y0, x0, tz, ty, tx = inner
    out = np.full((tz, ty, tx), 0xCD, np.uint8)
    air = C.c_int(-1)
    cfg = gpu_cfg(fb, d, dering, zdrift)
    rc = lib.fy_process_buffer(C.byref(cfg), u8.ctypes.data, *org, *u8.shape, z0, y0, x0, tz, ty, tx, *vol_yx,
                               out.ctypes.data, C.byref(air))
    return rc, out, air.value
