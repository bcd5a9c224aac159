"""Oracle bindings -- TEST INFRASTRUCTURE ONLY (the checker, never the product).

Only tests/, __graft_entry__.smoke() and bench.py's CPU legs import this package.

Two CPU implementations of the fysics restoration path:
  * ref():  the unmodified reference C sources compiled by oracle/Makefile into
            oracle/_ref/libfysics_ref.so (exactly fysics.h's entry points). This is "the
            reference's own CPU path" for bit-exact checks and the CPU baseline timing.
  * o64():  oracle/_build/libfy_oracle64.so, the FP64 restatement (fy_oracle64.c).
Both are plain ctypes handles; helpers below take/return numpy arrays.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_SO = HERE / "_ref" / "libfysics_ref.so"
O64_SO = HERE / "_build" / "libfy_oracle64.so"


class RefPhysics(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("delta_beta", "energy_kev", "distance_mm", "pixel_um",
                                          "unsharp_sigma", "unsharp_coeff", "psf_sigma_vox",
                                          "psf_sigma_z_vox")]


class RefNoise(C.Structure):
    _fields_ = [("g", C.c_double), ("b", C.c_double), ("noise_ref", C.c_double),
                ("ref_intensity", C.c_double), ("n_bins_used", C.c_int)]


class RefDering(C.Structure):
    _fields_ = [("Z", C.c_long), ("Y", C.c_long), ("X", C.c_long),
                ("cy", C.c_double), ("cx", C.c_double),
                ("slab_z", C.c_int), ("nslab", C.c_int), ("ns", C.c_int), ("nr", C.c_int),
                ("sum", C.POINTER(C.c_float)), ("cnt", C.POINTER(C.c_uint)),
                ("ring", C.POINTER(C.c_float)), ("have_rings", C.c_int)]


class RefHist(C.Structure):
    """fy_hist_state (fysics.h:54): 256 u8 counts and their total."""
    _fields_ = [("hist", C.c_long * 256), ("total", C.c_long)]


class RefZarr(C.Structure):
    """fy_zarr (fysics.h:376-381)."""
    _fields_ = [("root", C.c_char * 1024), ("shape", C.c_long * 3), ("chunk", C.c_long * 3), ("fill", C.c_ubyte)]


class RefPipelineCfg(C.Structure):
    """fy_pipeline_cfg (fysics.h:436-491), field for field."""
    _fields_ = ([(n, C.c_double) for n in ("delta_beta", "energy_kev", "distance_mm", "pixel_um", "unsharp_sigma",
                                           "unsharp_coeff", "machine_current_start", "machine_current_stop",
                                           "window_lo", "window_hi")] +
                [("do_deconv", C.c_int), ("use_matched_deconv", C.c_int), ("psf_sigma_vox", C.c_double),
                 ("deconv_tikhonov", C.c_double), ("guided_eps", C.c_double), ("do_air_zero", C.c_int),
                 ("air_cut_u8", C.c_int), ("air_cut_band", C.c_int), ("air_thresh", C.c_double),
                 ("air_cut_aggr", C.c_double), ("air_min_component", C.c_int), ("denoise_k", C.c_double),
                 ("scratch_passes", C.c_int), ("do_normalize", C.c_int), ("norm_lo", C.c_int), ("norm_hi", C.c_int),
                 ("do_zdrift", C.c_int), ("zdrift_factor", C.POINTER(C.c_float)), ("do_dering", C.c_int),
                 ("calib_budget_gb", C.c_double), ("dering_cy", C.c_double), ("dering_cx", C.c_double),
                 ("psf_p5", C.c_double), ("psf_med", C.c_double), ("do_musica", C.c_int), ("musica_p", C.c_double),
                 ("musica_levels", C.c_int), ("musica_core", C.c_double), ("guided_subsample", C.c_int),
                 ("no_dither", C.c_int), ("halo", C.c_int), ("have_norm", C.c_int), ("have_zdrift", C.c_int),
                 ("have_dec_range", C.c_int), ("have_dering", C.c_int), ("dering", C.POINTER(RefDering)),
                 ("psf_z_ratio", C.c_double), ("have_eps_r", C.c_int), ("eps_fn_a", C.c_double),
                 ("eps_fn_b", C.c_double), ("eps_fn_med", C.c_double), ("dec_lo", C.c_double),
                 ("dec_hi", C.c_double), ("vol_z", C.c_long), ("noise_floor", C.c_double),
                 ("occ", C.c_void_p), ("occ_ncz", C.c_long), ("occ_ncy", C.c_long), ("occ_ncx", C.c_long),
                 ("occ_cz", C.c_long), ("occ_cy", C.c_long), ("occ_cx", C.c_long)])


class OtTileCfg(C.Structure):
    """ot_tile_cfg (fy_oracle_tile.h): the fields the tile chain reads, resolved."""
    _fields_ = ([(n, C.c_double) for n in ("delta_beta", "energy_kev", "distance_mm", "pixel_um", "unsharp_sigma",
                                           "unsharp_coeff", "window_lo", "window_hi")] +
                [("do_deconv", C.c_int), ("use_matched_deconv", C.c_int), ("psf_sigma_vox", C.c_double),
                 ("deconv_tikhonov", C.c_double), ("psf_z_ratio", C.c_double), ("have_dec_range", C.c_int),
                 ("dec_lo", C.c_double), ("dec_hi", C.c_double), ("guided_eps", C.c_double),
                 ("guided_subsample", C.c_int), ("tile_eps", C.c_double), ("do_air_zero", C.c_int),
                 ("air_cut_u8", C.c_int), ("air_cut_band", C.c_int), ("air_thresh", C.c_double),
                 ("air_cut_aggr", C.c_double), ("air_min_component", C.c_int), ("scratch_passes", C.c_int),
                 ("have_norm", C.c_int), ("norm_lo", C.c_int), ("norm_hi", C.c_int), ("do_musica", C.c_int),
                 ("no_dither", C.c_int), ("ring", C.POINTER(C.c_float)), ("nslab", C.c_int), ("nr", C.c_int),
                 ("slab_z", C.c_int), ("ring_cy", C.c_double), ("ring_cx", C.c_double),
                 ("zdrift", C.POINTER(C.c_float))])


_P, _i, _l, _d, _sz = C.c_void_p, C.c_int, C.c_long, C.c_double, C.c_size_t
_PP = C.POINTER(RefPhysics)
_PDB = C.POINTER(C.c_double)

REF_SIGS = {
    "fy_next_fft_size": (_i, [_i]),
    "fy_fft1d": (None, [_P, _P, _i, _i]),
    "fy_fft3d": (None, [_P, _P, _i, _i, _i, _i]),
    "fy_fft3d_normalize": (None, [_P, _P, _i, _i, _i]),
    "fy_u8_to_float": (None, [_P, _P, _sz]),
    "fy_float_to_u8": (None, [_P, _P, _sz]),
    "fy_u8_to_phys": (None, [_P, _P, _sz, _d, _d]),
    "fy_phys_to_u8": (None, [_P, _P, _sz, _d, _d]),
    "fy_phys_to_u8_level": (C.c_float, [_d, _d, _d]),
    "fy_paganin_transfer": (_d, [_d, _PP]),
    "fy_unsharp_transfer": (_d, [_d, _PP]),
    "fy_recon_transfer": (_d, [_d, _PP]),
    "fy_auto_deltabeta_scale": (_d, [_PP]),
    "fy_kernel_halo": (_i, [_PP]),
    "fy_deconvolve": (_i, [_P, _P, _i, _i, _i, _PP, _d]),
    "fy_deconvolve_matched": (_i, [_P, _P, _i, _i, _i, _PP, _d]),
    "fy_guided_denoise_ws": (_i, [_P, _P, _i, _i, _i, _i, _d, _P]),
    "fy_guided_denoise_fast_ws": (_i, [_P, _P, _i, _i, _i, _i, _d, _i, _P]),
    "fy_guided_ws_floats": (_sz, [_i, _i, _i]),
    "fy_box_smooth": (None, [_P, _P, _P, _i, _i, _i, _i]),
    "fy_guided_eps_for_noise": (_d, [_d]),
    "fy_estimate_noise": (_i, [_P, _i, _i, _i, _i, _d, _d, C.POINTER(RefNoise)]),
    "fy_dering_init": (_i, [C.POINTER(RefDering), _l, _l, _l, _d, _d, _i, _i]),
    "fy_dering_free": (None, [C.POINTER(RefDering)]),
    "fy_dering_tile_init": (_i, [C.POINTER(RefDering), C.POINTER(RefDering)]),
    "fy_dering_tile_reset": (None, [C.POINTER(RefDering)]),
    "fy_dering_accumulate_u8": (None, [C.POINTER(RefDering), _P, _l, _l, _l, _l, _l, _i]),
    "fy_dering_merge_tile": (None, [C.POINTER(RefDering), _i, C.POINTER(RefDering)]),
    "fy_dering_finalize": (_l, [C.POINTER(RefDering), _i, C.c_uint, _d, _d]),
    "fy_dering_apply": (None, [C.POINTER(RefDering), _P, _l, _l, _l, _l, _l, _l, _d]),
    "fy_phase_correlate": (_i, [_P, _P, _i, _i, _i, _PDB, _PDB, _i]),
    "fy_hist_init": (None, [C.POINTER(RefHist)]),
    "fy_hist_accumulate_u8": (None, [C.POINTER(RefHist), _P, _sz]),
    "fy_hist_merge": (None, [C.POINTER(RefHist), C.POINTER(RefHist)]),
    "fy_hist_percentile_u8": (_i, [C.POINTER(RefHist), _d]),
    "fy_hist_percentile_u8_inner": (_i, [C.POINTER(RefHist), _d]),
    "fy_flat_noise": (_d, [_P, _i, _i, _i, _i]),
    "fy_noise_aniso": (_i, [_P, _i, _i, _i, _PDB, _PDB]),
    "fy_valley_depth": (_d, [_P, C.POINTER(_i), C.POINTER(_i), C.POINTER(_i)]),
    "fy_box_smooth": (None, [_P, _P, _P, _i, _i, _i, _i]),
    "fy_zarr_open": (_i, [C.POINTER(RefZarr), C.c_char_p]),
    "fy_zarr_read": (_i, [C.POINTER(RefZarr), _l, _l, _l, _l, _l, _l, _P]),
    "fy_zarr_create": (_i, [C.POINTER(RefZarr), C.c_char_p, C.POINTER(_l), C.POINTER(_l)]),
    "fy_zarr_write_chunk": (_i, [C.POINTER(RefZarr), _l, _l, _l, _P, _l, _l, _l]),
    "fy_calibrate": (_i, [C.c_char_p, C.POINTER(RefPipelineCfg), _i, _i]),
    "fy_process_chunk": (_i, [C.POINTER(RefZarr), C.POINTER(RefPipelineCfg), _l, _l, _l, _i, _P, C.POINTER(_i),
                              C.POINTER(_i), C.POINTER(_i), C.POINTER(_i)]),
    "fy_process_buffer": (_i, [C.POINTER(RefPipelineCfg), _P, _l, _l, _l, _l, _l, _l, _l, _l, _l, _l, _l, _l,
                               _l, _l, _P, C.POINTER(_i)]),
}

O64_SIGS = {
    "o64_next_fft_size": (_i, [_i]),
    "o64_fft1d": (None, [_P, _i, _i]),
    "o64_u8_to_phys": (None, [_P, _P, _sz, _d, _d]),
    "o64_paganin_transfer": (_d, [_d, _PP]),
    "o64_recon_transfer": (_d, [_d, _PP]),
    "o64_auto_deltabeta_scale": (_d, [_PP]),
    "o64_deconvolve": (_i, [_P, _P, _i, _i, _i, _PP, _d, _i, _d, _i]),
    "o64_box_mean": (None, [_P, _P, _i, _i, _i, _i]),
    "o64_guided": (_i, [_P, _P, _i, _i, _i, _i, _d]),
    "o64_guided_fast": (_i, [_P, _P, _i, _i, _i, _i, _d, _i]),
    "o64_estimate_noise": (_i, [_P, _i, _i, _i, _i, _d, _d, C.POINTER(RefNoise)]),
    "o64_estimate_noise64": (_i, [_P, _i, _i, _i, _i, _d, _d, C.POINTER(RefNoise)]),
    "o64_guided_eps_for_noise": (_d, [_d]),
    "o64_dering_nr": (_i, [_l, _l, _d, _d]),
    "o64_dering_accumulate_u8": (None, [_P, _l, _l, _l, _l, _l, _i, _d, _d, _i, _i, _P, _P]),
    "o64_dering_finalize": (_l, [_P, _P, _i, _i, _i, _i, C.c_uint, _d, _d, _P, C.POINTER(_i)]),
    "o64_dering_apply": (None, [_P, _i, _i, _i, _d, _d, _P, _l, _l, _l, _l, _l, _l, _d]),
    "o64_phase_correlate": (_i, [_P, _P, _i, _i, _i, _PDB, _PDB, _i, C.POINTER(_l)]),
    "o64_fit_radial_eps": (_i, [_P, _P, _i, _PDB, _PDB, _PDB]),
    "o64_median_floor": (C.c_double, [_P, _i]),
    "o64_hist_u8": (None, [_P, _sz, _P]),
    "o64_flat_noise": (_d, [_P, _i, _i, _i, _i]),
    "o64_noise_aniso": (_i, [_P, _i, _i, _i, _PDB, _PDB]),
    "ot_valley_depth": (_d, [_P, C.POINTER(_i), C.POINTER(_i), C.POINTER(_i)]),
    "ot_box_smooth": (None, [_P, _P, _i, _i, _i, _i]),
    "ot_cc_despeckle": (_l, [_P, _i, _i, _i, _i]),
    "ot_dither01": (C.c_float, [_l, _l, _l]),
    "ot_quant_u8": (C.c_uint8, [C.c_float, _l, _l, _l, _i]),
    "ot_air_cuts": (None, [_P, _i, _i, _d, _d, C.POINTER(_i), C.POINTER(_i), C.POINTER(_i)]),
    "ot_measure_psf_sigma": (_d, [_P, _i, _i, _i, C.POINTER(_i)]),
    "ot_process_buffer": (_i, [C.POINTER(OtTileCfg), _P, _l, _l, _l, _l, _l, _l, _l, _l, _l, _l, _l, _l, _P,
                               C.POINTER(_i), _P, _P]),
    "o64_radial_tile_eps": (C.c_double, [_i, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                                         C.c_double, C.c_long, C.c_long, C.c_long, C.c_long]),
}

_ref = None
_o64 = None


def _bind(path: Path, sigs: dict) -> C.CDLL:
    lib = C.CDLL(str(path), mode=C.RTLD_LOCAL)
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype, fn.argtypes = res, args
    return lib


def have_ref() -> bool:
    return REF_SO.exists()


def ref() -> C.CDLL:
    """The reference library compiled from its own sources (oracle/Makefile)."""
    global _ref
    if _ref is None:
        if not REF_SO.exists():
            raise FileNotFoundError(f"{REF_SO} missing: run `make -C oracle ref REF_DIR=<reference checkout>` "
                                    "where the reference sources are available")
        _ref = _bind(REF_SO, REF_SIGS)
    return _ref


def o64() -> C.CDLL:
    """The FP64 restatement; built on first use if gcc is available."""
    global _o64
    if _o64 is None:
        if not O64_SO.exists():
            subprocess.run(["make", "-C", str(HERE), "oracle64"], check=True,
                           capture_output=True)
        _o64 = _bind(O64_SO, O64_SIGS)
    return _o64


def p(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


def ref_physics(**kw) -> RefPhysics:
    d = dict(delta_beta=1000.0, energy_kev=78.0, distance_mm=220.0, pixel_um=2.4,
             unsharp_sigma=1.2, unsharp_coeff=4.0, psf_sigma_vox=0.0, psf_sigma_z_vox=0.0)
    d.update(kw)
    return RefPhysics(*[d[n] for n, _ in RefPhysics._fields_])


# ------------------------------------------------------------- numpy helpers: reference
def ref_u8_to_phys(u8, lo, hi):
    a = np.ascontiguousarray(u8, np.uint8)
    out = np.empty(a.shape, np.float32)
    ref().fy_u8_to_phys(p(a), p(out), a.size, lo, hi)
    return out


def ref_phys_to_u8(v, lo, hi):
    a = np.ascontiguousarray(v, np.float32)
    out = np.empty(a.shape, np.uint8)
    ref().fy_phys_to_u8(p(a), p(out), a.size, lo, hi)
    return out


def ref_deconvolve(vol, phys, reg, matched=False):
    a = np.ascontiguousarray(vol, np.float32)
    out = np.empty_like(a)
    fn = ref().fy_deconvolve_matched if matched else ref().fy_deconvolve
    rc = fn(p(a), p(out), *a.shape, C.byref(phys), reg)
    assert rc == 0
    return out


# ------------------------------------------------------------- numpy helpers: FP64 oracle
def o64_deconvolve(vol, phys, param, kind=0, fz2_scale=1.0, use_lut=True):
    a = np.ascontiguousarray(vol, np.float64)
    out = np.empty_like(a)
    rc = o64().o64_deconvolve(p(a), p(out), *a.shape, C.byref(phys), param, kind, fz2_scale,
                              1 if use_lut else 0)
    assert rc == 0
    return out


# ------------------------------------------------------------- the per-tile chain (f1)
def pipeline_defaults(**kw) -> dict:
    """A fy_pipeline_cfg as a dict: the export tool's settings (mca_export.c:1001-1015) with
    the reference physics; keys are fy_pipeline_cfg field names."""
    d = {n: 0 for n, _ in RefPipelineCfg._fields_}
    d.update(dict(delta_beta=1000.0, energy_kev=78.0, distance_mm=220.0, pixel_um=2.4, unsharp_sigma=1.2,
                  unsharp_coeff=4.0, window_lo=0.0, window_hi=0.0, do_deconv=0, use_matched_deconv=1,
                  psf_sigma_vox=1.0, deconv_tikhonov=0.05, guided_eps=0.0, do_air_zero=1, air_cut_u8=-1,
                  air_cut_band=8, air_thresh=0.05, air_cut_aggr=0.5, air_min_component=0, scratch_passes=5,
                  guided_subsample=0, no_dither=0, halo=8, dering_cy=-1.0, dering_cx=-1.0))
    d.update(kw)
    return d


def ref_pipeline_cfg(d: dict, dering=None, zdrift=None) -> RefPipelineCfg:
    """Fill the reference struct; `dering` is a RefDering, `zdrift` a float32 array (kept alive
    by the caller)."""
    c = RefPipelineCfg()
    for n, t in RefPipelineCfg._fields_:
        if n in ("zdrift_factor", "dering", "occ"):
            continue
        setattr(c, n, d.get(n, 0))
    if zdrift is not None:
        c.zdrift_factor = zdrift.ctypes.data_as(C.POINTER(C.c_float))
    if dering is not None:
        c.dering = C.pointer(dering)
    return c


def tile_eps(d: dict, y0, x0, ty, tx, vol_y, vol_x) -> float:
    """eps_for_tile (pipeline.c:447-456) with the rotation-axis default of fy_process_buffer."""
    ecy = d["dering_cy"] if d["dering_cy"] > 0 else (vol_y - 1) / 2.0
    ecx = d["dering_cx"] if d["dering_cx"] > 0 else (vol_x - 1) / 2.0
    return o64().o64_radial_tile_eps(int(d["have_eps_r"]), d["eps_fn_a"], d["eps_fn_b"], d["eps_fn_med"],
                                     d["guided_eps"], ecy, ecx, y0, x0, ty, tx)


def ot_tile_cfg(d: dict, geo, ring=None, ring_geo=None, zdrift=None) -> OtTileCfg:
    """Resolve a cfg dict for the oracle. geo = (y0, x0, ty, tx, vol_y, vol_x); ring is the
    float32 [nslab][nr] table with ring_geo = (nslab, nr, slab_z, cy, cx)."""
    c = OtTileCfg()
    for n, _ in OtTileCfg._fields_:
        if n in d:
            setattr(c, n, d[n])
    c.tile_eps = tile_eps(d, *geo)
    if ring is not None and d.get("have_dering"):
        c.ring = ring.ctypes.data_as(C.POINTER(C.c_float))
        c.nslab, c.nr, c.slab_z, c.ring_cy, c.ring_cx = ring_geo
    if zdrift is not None and d.get("have_zdrift"):
        c.zdrift = zdrift.ctypes.data_as(C.POINTER(C.c_float))
    return c


def ref_process_buffer(d: dict, u8, org, inner, vol_yx, dering=None, zdrift=None):
    """The reference's fy_process_buffer on a haloed u8 buffer at global origin org=(rz0,ry0,rx0);
    inner = (z0, y0, x0, tz, ty, tx). Returns (out u8 [tz,ty,tx], all_air)."""
    u8 = np.ascontiguousarray(u8, np.uint8)
    z0, y0, x0, tz, ty, tx = inner
    out = np.full((tz, ty, tx), 0xCD, np.uint8)
    air = C.c_int(-1)
    cfg = ref_pipeline_cfg(d, dering, zdrift)
    rc = ref().fy_process_buffer(C.byref(cfg), p(u8), *org, *u8.shape, z0, y0, x0, tz, ty, tx, *vol_yx, p(out),
                                 C.byref(air))
    assert rc == 0
    return out, air.value


def ot_process_buffer(d: dict, u8, org, inner, vol_yx, ring=None, ring_geo=None, zdrift=None, state=False):
    """The oracle restatement of fy_process_buffer; with state=True also the air-cut histogram
    and (cut, uniform cut, textured cut)."""
    u8 = np.ascontiguousarray(u8, np.uint8)
    z0, y0, x0, tz, ty, tx = inner
    out = np.full((tz, ty, tx), 0xCD, np.uint8)
    air = C.c_int(-1)
    hist = np.zeros(256, np.int64)
    cuts = np.zeros(3, np.int32)
    cfg = ot_tile_cfg(d, (y0, x0, ty, tx, *vol_yx), ring, ring_geo, zdrift)
    rc = o64().ot_process_buffer(C.byref(cfg), p(u8), *org, *u8.shape, z0, y0, x0, tz, ty, tx, p(out),
                                 C.byref(air), p(hist), p(cuts))
    assert rc == 0, rc
    return (out, air.value, hist, cuts) if state else (out, air.value)


PSF_SO = HERE / "_ref" / "libref_psf.so"
_psf = None


def ref_psf():
    """The reference's static measure_tile_psf_sigma (pipeline.c:107-196) through the shim
    oracle/ref_psf_shim.c; None where the reference was not built."""
    global _psf
    if _psf is None and PSF_SO.exists():
        _psf = C.CDLL(str(PSF_SO), mode=C.RTLD_LOCAL)
        _psf.ref_measure_tile_psf_sigma.restype = C.c_double
        _psf.ref_measure_tile_psf_sigma.argtypes = [_P, _i, _i, _i]
    return _psf
