"""Generate tests/golden/reference_golden.npz from the reference library.

Run where the reference sources exist (they are compiled by `make -C oracle ref`):

    python tests/golden/make_golden.py

Every input is a seeded recipe from tests/_recipes.py (the reference tests' own LCG
recipes), so only the reference's OUTPUTS are stored. The GPU parity tests and the oracle
pins fall back to these vectors where oracle/_ref/libfysics_ref.so is absent.
"""
import ctypes as C
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
from oracle import p, ref, ref_physics  # noqa: E402
from tests import _recipes as R  # noqa: E402

OUT = Path(__file__).resolve().parent / "reference_golden.npz"


def main():
    L = ref()
    g = {}
    vol = R.deconv_equivalence_input()
    g["deconv_equiv"] = oracle.ref_deconvolve(vol, ref_physics(), 0.015)
    g["deconv_matched"] = oracle.ref_deconvolve(
        vol, ref_physics(psf_sigma_vox=1.0, psf_sigma_z_vox=1.17), 0.05, matched=True)

    gv = R.guided_step_input()
    nz, ny, nx = gv.shape
    ws = np.empty(4 * gv.size, np.float32)
    out = np.empty_like(gv)
    L.fy_guided_denoise_ws(p(gv), p(out), nz, ny, nx, 2, 0.0004, p(ws))
    g["guided_exact"] = out.copy()
    L.fy_guided_denoise_fast_ws(p(gv), p(out), nz, ny, nx, 2, 0.0004, 2, p(ws))
    g["guided_fast"] = out.copy()

    nv = R.noise_input(0.05, 12345)
    nm = oracle.RefNoise()
    L.fy_estimate_noise(p(nv), *nv.shape, 5, 10.0, 0.5, C.byref(nm))
    g["noise_model"] = np.array([nm.g, nm.b, nm.noise_ref, nm.n_bins_used])

    dv, cy, cx = R.dering_input()
    nz, ny, nx = dv.shape
    d, t = oracle.RefDering(), oracle.RefDering()
    L.fy_dering_init(C.byref(d), nz, ny, nx, -1, -1, 64, 8)
    L.fy_dering_tile_init(C.byref(t), C.byref(d))
    L.fy_dering_accumulate_u8(C.byref(t), p(dv), 0, 0, nz, ny, nx, 1)
    L.fy_dering_merge_tile(C.byref(d), 0, C.byref(t))
    L.fy_dering_finalize(C.byref(d), 15, 50, 2.0, 15.0)
    rg = np.ctypeslib.as_array(d.ring, shape=(d.nr,)).astype(np.float64).copy()
    cnt = np.ctypeslib.as_array(d.cnt, shape=(d.ns * d.nr,)).astype(np.float64).copy()
    sm = np.ctypeslib.as_array(d.sum, shape=(d.ns * d.nr,)).astype(np.float64).copy()
    g["dering"] = np.concatenate([rg, cnt, sm])
    fa = (dv * np.float32(1.0 / 255.0)).astype(np.float32)
    L.fy_dering_apply(C.byref(d), p(fa), 0, 0, 0, nz, ny, nx, 1.0 / 255.0)
    g["dering_apply_slice0"] = fa[0].copy()
    L.fy_dering_free(C.byref(t))
    L.fy_dering_free(C.byref(d))

    f = R.phasecorr_texture()
    for i, s in enumerate(R.PHASECORR_CASES):
        m = R.fourier_shift(f, s)
        sh = (C.c_double * 3)()
        pk = C.c_double()
        L.fy_phase_correlate(p(f), p(m), *f.shape, sh, C.byref(pk), 0)
        g[f"phasecorr_{i}"] = np.array(sh[:] + [pk.value])

    u8 = np.arange(256, dtype=np.uint8)
    wins = [(-0.03, 0.21), (0.0, 1.0), (-1.5, 2.25), (0.1, 0.1000001), (1e-3, 7.0)]
    g["dewindow_windows"] = np.array(wins)
    g["dewindow"] = np.stack([oracle.ref_u8_to_phys(u8, a, b) for a, b in wins])
    rv = np.random.default_rng(7).uniform(-0.5, 1.5, 4096).astype(np.float32)
    g["requant_in"] = rv
    g["requant"] = np.stack([oracle.ref_phys_to_u8(rv, a, b) for a, b in wins])
    np.savez_compressed(OUT, **g)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes, {len(g)} arrays)")


if __name__ == "__main__":
    main()
