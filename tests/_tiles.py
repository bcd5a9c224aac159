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


def psf_volume(shape, sigma, orient, noise, seed):
    """u8 tile of blurred two-level steps (35 / 185) for the PSF edge fit: the steps vary
    along y ("y"), x ("x") or both ("xy"), blurred by a Gaussian of `sigma` voxels, plus
    Gaussian noise of `noise` levels."""
    from scipy.ndimage import gaussian_filter
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid(*[np.arange(s) for s in shape], indexing="ij")
    if orient == "y":
        f = np.sin(y / 6.0 + 0.3 * np.sin(x / 17.0))
    elif orient == "x":
        f = np.sin(x / 6.0 + 0.3 * np.sin(z / 13.0))
    else:
        f = np.sin(x / 5.0) + np.cos(y / 7.0)
    step = (f > 0).astype(float) * 150 + 35
    v = gaussian_filter(step, sigma) + rng.normal(0, noise, shape)
    return np.clip(np.rint(v), 0, 255).astype(np.uint8)


PSF_CASES = [((32, 64, 64), 0.7, "y", 0.5), ((32, 64, 64), 2.0, "xy", 2.0), ((40, 96, 80), 1.2, "x", 2.0),
             ((40, 96, 80), 3.0, "xy", 0.5), ((16, 30, 200), 2.0, "x", 0.5), ((16, 30, 200), 0.7, "y", 2.0),
             ((24, 12, 90), 1.2, "x", 0.5), ((24, 90, 12), 1.2, "y", 0.5), ((8, 10, 10), 1.0, "xy", 0.5)]
