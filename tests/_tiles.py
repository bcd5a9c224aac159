"""Seeded haloed tiles and settings for the per-tile chain (fy_process_buffer).

A synthetic scroll volume: noisy air (u8 ~ 22) around a cylindrical body of papyrus sheets
(u8 ~ 90-170), small bright specks in the air (the islands the connected-component
despeckle removes) and an exactly-zero masked slab, so the air-cut histogram has two
modes and a valley, as on the volumes the export tool processes.
"""
from __future__ import annotations

import ctypes as C

import numpy as np


def scroll_volume(shape, seed=0, specks=300, masked=True):
    nz, ny, nx = shape
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    cy, cx = (ny - 1) / 2 + rng.uniform(-3, 3), (nx - 1) / 2 + rng.uniform(-3, 3)
    r = np.hypot(y - cy, x - cx)
    body = r < 0.42 * min(ny, nx)
    # sheets: a spiral-like wrap, thickness ~3 voxels
    phase = r / 4.5 + np.arctan2(y - cy, x - cx) / (2 * np.pi) + 0.15 * np.sin(z / 11.0)
    sheet = np.cos(2 * np.pi * phase) > 0.2
    v = rng.normal(22, 6, shape)
    v = np.where(body, np.where(sheet, rng.normal(150, 12, shape), rng.normal(70, 10, shape)), v)
    for _ in range(specks):                          # islands of 1..~30 voxels in the air
        c = rng.integers([0, 0, 0], [nz, ny, nx])
        if body[tuple(c)]:
            continue
        e = rng.integers(0, 3, 3)
        v[c[0]:c[0] + e[0] + 1, c[1]:c[1] + e[1] + 1, c[2]:c[2] + e[2] + 1] = rng.normal(150, 10)
    u8 = np.clip(np.rint(v), 0, 255).astype(np.uint8)
    if masked:
        u8[:, : max(1, ny // 10), :] = 0                # a masked slab (exact zeros)
    return u8


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
