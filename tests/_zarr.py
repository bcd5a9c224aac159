"""Local zarr v2 raw-u8 trees in the reference's layout (zarr_io.c:1-9, 170-185, 328-340):
<root>/0/.zarray and <root>/0/cz/cy/cx chunk files of the chunk's TRUE extent (edge chunks
are smaller). Test and benchmark input only."""
from __future__ import annotations

import os
from pathlib import Path

import numpy as np


def zarray_text(shape, chunk, fill=0) -> str:
    return ('{"chunks":[%d,%d,%d],"compressor":null,"dtype":"|u1","fill_value":%s,"order":"C",'
            '"shape":[%d,%d,%d],"zarr_format":2,"dimension_separator":"/"}'
            % (*chunk, fill, *shape))


def write_zarr(root, vol: np.ndarray, chunk, fill=0, drop=(), truncate=None, header=None) -> Path:
    """Write `vol` as a chunked tree. `drop`: chunk coordinates left without a file (read as
    fill); `truncate`: {chunk coord: bytes kept} (a short file, its tail reads as fill);
    `header`: the .zarray text to write instead of the standard one."""
    root = Path(root)
    (root / "0").mkdir(parents=True, exist_ok=True)
    (root / "0" / ".zarray").write_text(header if header is not None else zarray_text(vol.shape, chunk, fill))
    truncate = truncate or {}
    nz, ny, nx = vol.shape
    cz, cy, cx = chunk
    for iz in range(-(-nz // cz)):
        for iy in range(-(-ny // cy)):
            for ix in range(-(-nx // cx)):
                if (iz, iy, ix) in drop:
                    continue
                blk = np.ascontiguousarray(vol[iz * cz:(iz + 1) * cz, iy * cy:(iy + 1) * cy, ix * cx:(ix + 1) * cx])
                data = blk.tobytes()
                if (iz, iy, ix) in truncate:
                    data = data[:truncate[(iz, iy, ix)]]
                d = root / "0" / str(iz) / str(iy)
                d.mkdir(parents=True, exist_ok=True)
                with open(d / str(ix), "wb") as f:
                    f.write(data)
    return root


def expected_region(vol: np.ndarray, chunk, region, out: np.ndarray, fill=0, drop=(), truncate=None):
    """The assembly rule restated in numpy (zarr_io.c:288-320): each in-volume voxel takes byte
    (lz*ey + ly)*ex + lx of its chunk's stored bytes, or `fill` past their end or for a missing
    chunk; voxels outside the volume keep out's prior contents."""
    z0, y0, x0, dz, dy, dx = region
    nz, ny, nx = vol.shape
    c0, c1, c2 = chunk
    gz, gy, gx = (np.arange(a, min(a + d, n)) for a, d, n in ((z0, dz, nz), (y0, dy, ny), (x0, dx, nx)))
    if not (gz.size and gy.size and gx.size):
        return out
    kz, ky, kx = gz // c0, gy // c1, gx // c2
    ey, ex = np.minimum(ny - ky * c1, c1), np.minimum(nx - kx * c2, c2)
    off = (((gz - kz * c0)[:, None, None] * ey[None, :, None] + (gy - ky * c1)[None, :, None]) * ex[None, None, :]
           + (gx - kx * c2)[None, None, :])
    v = vol[np.ix_(gz, gy, gx)].copy()
    chunk_of = lambda k: ((kz == k[0])[:, None, None] & (ky == k[1])[None, :, None] & (kx == k[2])[None, None, :])
    for k in drop:
        v[chunk_of(k)] = fill
    for k, keep in (truncate or {}).items():
        v[chunk_of(k) & (off >= keep)] = fill
    out[np.ix_(gz - z0, gy - y0, gx - x0)] = v
    return out
