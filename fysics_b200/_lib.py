"""ctypes binding of libfysics_b200.so (include/fysics_b200.h).

The shared library is the product: every call below runs hand-written sm_100a kernels.
There is no Python or CPU fallback -- if the library is missing, import fails loudly, and
without a CUDA device every entry point returns FY_ENODEV.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libfysics_b200.so"

FY_OK, FY_EINVAL, FY_ENOMEM, FY_ECUDA, FY_ENODEV = 0, 1, 2, 3, 4
FY_EUNSUPPORTED, FY_ETIMEDOUT, FY_EBUSY, FY_EDEGENERATE, FY_EIO = 5, 6, 7, 8, 9


class Physics(C.Structure):
    """fy_physics (fysics.h:23-35): 8 doubles."""
    _fields_ = [("delta_beta", C.c_double), ("energy_kev", C.c_double),
                ("distance_mm", C.c_double), ("pixel_um", C.c_double),
                ("unsharp_sigma", C.c_double), ("unsharp_coeff", C.c_double),
                ("psf_sigma_vox", C.c_double), ("psf_sigma_z_vox", C.c_double)]


class NoiseModel(C.Structure):
    """fy_noise_model (fysics.h:191-197)."""
    _fields_ = [("g", C.c_double), ("b", C.c_double), ("noise_ref", C.c_double),
                ("ref_intensity", C.c_double), ("n_bins_used", C.c_int)]


class HistState(C.Structure):
    """fy_hist_state (fysics.h:54): 256 u8 counts and their total."""
    _fields_ = [("hist", C.c_long * 256), ("total", C.c_long)]


class AnisoResult(C.Structure):
    """fy_aniso_result (include/fysics_b200.h)."""
    _fields_ = [("rho_z", C.c_double), ("rho_xy", C.c_double), ("status", C.c_int)]


class RestoreCfg(C.Structure):
    """fy_restore_cfg (include/fysics_b200.h)."""
    _fields_ = [("deconv_kind", C.c_int), ("deconv_param", C.c_double), ("fz2_scale", C.c_double),
                ("noise_win", C.c_int), ("noise_flat_pct", C.c_double), ("noise_ref_intensity", C.c_double),
                ("guided_eps", C.c_double), ("guided_radius", C.c_int), ("guided_s", C.c_int),
                ("dering", C.c_void_p), ("dering_accumulate", C.c_int), ("dering_ss", C.c_int),
                ("dering_hp_win", C.c_int), ("dering_min_cnt", C.c_uint), ("dering_min_amp", C.c_double),
                ("dering_max_amp", C.c_double), ("dering_scale", C.c_double),
                ("z0", C.c_long), ("y0", C.c_long), ("x0", C.c_long),
                ("radial", C.c_void_p), ("radial_cy", C.c_double), ("radial_cx", C.c_double)]


class PipelineCfg(C.Structure):
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
                 ("have_dec_range", C.c_int), ("have_dering", C.c_int), ("dering", C.c_void_p),
                 ("psf_z_ratio", C.c_double), ("have_eps_r", C.c_int), ("eps_fn_a", C.c_double),
                 ("eps_fn_b", C.c_double), ("eps_fn_med", C.c_double), ("dec_lo", C.c_double),
                 ("dec_hi", C.c_double), ("vol_z", C.c_long), ("noise_floor", C.c_double),
                 ("occ", C.c_void_p), ("occ_ncz", C.c_long), ("occ_ncy", C.c_long), ("occ_ncx", C.c_long),
                 ("occ_cz", C.c_long), ("occ_cy", C.c_long), ("occ_cx", C.c_long)])


class ServerCfg(C.Structure):
    """fy_server_cfg (include/fysics_b200.h)."""
    _fields_ = [("hbm_budget_bytes", C.c_size_t), ("workers", C.c_int), ("device", C.c_int),
                ("priority_voxels", C.c_size_t), ("small_workers", C.c_int),
                ("reserve_nz", C.c_int), ("reserve_ny", C.c_int), ("reserve_nx", C.c_int)]


class Request(C.Structure):
    """fy_request (include/fysics_b200.h)."""
    _fields_ = [("u8", C.c_void_p), ("out", C.c_void_p), ("nz", C.c_int), ("ny", C.c_int), ("nx", C.c_int),
                ("f32_min", C.c_double), ("f32_max", C.c_double), ("phys", Physics), ("cfg", RestoreCfg)]


class BatchCube(C.Structure):
    """fy_batch_cube (include/fysics_b200.h)."""
    _fields_ = [("u8", C.c_void_p), ("out", C.c_void_p), ("nz", C.c_int), ("ny", C.c_int), ("nx", C.c_int),
                ("f32_min", C.c_double), ("f32_max", C.c_double), ("phys", Physics)]


class RequestResult(C.Structure):
    """fy_request_result (include/fysics_b200.h)."""
    _fields_ = [("status", C.c_int), ("queue_ms", C.c_double), ("run_ms", C.c_double), ("latency_ms", C.c_double),
                ("h2d_ms", C.c_double), ("chain_ms", C.c_double), ("d2h_ms", C.c_double)]


class ServerStats(C.Structure):
    """fy_server_stats (include/fysics_b200.h)."""
    _fields_ = [("completed", C.c_longlong), ("voxels", C.c_double), ("mvox_per_s", C.c_double),
                ("p50_ms", C.c_double), ("p99_ms", C.c_double), ("inflight", C.c_int), ("queued", C.c_int)]


class RadialEps(C.Structure):
    """fy_radial_eps (include/fysics_b200.h)."""
    _fields_ = [("a", C.c_double), ("b", C.c_double), ("corr", C.c_double), ("median", C.c_double),
                ("guided_eps", C.c_double), ("have", C.c_int), ("n", C.c_int)]


class Dering(C.Structure):
    """fy_dering (fysics.h:406-415)."""
    _fields_ = [("Z", C.c_long), ("Y", C.c_long), ("X", C.c_long),
                ("cy", C.c_double), ("cx", C.c_double),
                ("slab_z", C.c_int), ("nslab", C.c_int), ("ns", C.c_int), ("nr", C.c_int),
                ("sum", C.POINTER(C.c_float)), ("cnt", C.POINTER(C.c_uint)),
                ("ring", C.POINTER(C.c_float)), ("have_rings", C.c_int)]


class Zarr(C.Structure):
    """fy_zarr (fysics.h:376-381)."""
    _fields_ = [("root", C.c_char * 1024), ("shape", C.c_long * 3), ("chunk", C.c_long * 3), ("fill", C.c_ubyte)]


_P = C.c_void_p
_i, _l, _d, _f, _sz = C.c_int, C.c_long, C.c_double, C.c_float, C.c_size_t
_PP = C.POINTER(Physics)
_PN = C.POINTER(NoiseModel)
_PD = C.POINTER(Dering)
_PDBL = C.POINTER(C.c_double)

# name -> (restype, argtypes): every symbol declared in include/fysics_b200.h
SIGNATURES = {
    "fy_is_pow2": (_i, [_i]),
    "fy_next_pow2": (_i, [_i]),
    "fy_next_fft_size": (_i, [_i]),
    "fy_fft1d": (None, [_P, _P, _i, _i]),
    "fy_fft3d": (None, [_P, _P, _i, _i, _i, _i]),
    "fy_fft3d_normalize": (None, [_P, _P, _i, _i, _i]),
    "fy_u8_to_float": (None, [_P, _P, _sz]),
    "fy_float_to_u8": (None, [_P, _P, _sz]),
    "fy_u8_to_phys": (None, [_P, _P, _sz, _d, _d]),
    "fy_phys_to_u8": (None, [_P, _P, _sz, _d, _d]),
    "fy_phys_to_u8_level": (_f, [_d, _d, _d]),
    "fy_paganin_transfer": (_d, [_d, _PP]),
    "fy_unsharp_transfer": (_d, [_d, _PP]),
    "fy_recon_transfer": (_d, [_d, _PP]),
    "fy_auto_reg": (_d, [_PP, _d]),
    "fy_auto_deltabeta_scale": (_d, [_PP]),
    "fy_kernel_halo": (_i, [_PP]),
    "fy_deconvolve": (_i, [_P, _P, _i, _i, _i, _PP, _d]),
    "fy_deconvolve_matched": (_i, [_P, _P, _i, _i, _i, _PP, _d]),
    "fy_guided_denoise": (_i, [_P, _P, _i, _i, _i, _i, _d]),
    "fy_guided_denoise_ws": (_i, [_P, _P, _i, _i, _i, _i, _d, _P]),
    "fy_guided_ws_floats": (_sz, [_i, _i, _i]),
    "fy_guided_denoise_fast_ws": (_i, [_P, _P, _i, _i, _i, _i, _d, _i, _P]),
    "fy_box_smooth": (None, [_P, _P, _P, _i, _i, _i, _i]),
    "fy_guided_eps_for_noise": (_d, [_d]),
    "fy_estimate_noise": (_i, [_P, _i, _i, _i, _i, _d, _d, _PN]),
    "fy_dering_init": (_i, [_PD, _l, _l, _l, _d, _d, _i, _i]),
    "fy_dering_free": (None, [_PD]),
    "fy_dering_tile_init": (_i, [_PD, _PD]),
    "fy_dering_tile_reset": (None, [_PD]),
    "fy_dering_accumulate_u8": (None, [_PD, _P, _l, _l, _l, _l, _l, _i]),
    "fy_dering_merge_tile": (None, [_PD, _i, _PD]),
    "fy_dering_finalize": (_l, [_PD, _i, C.c_uint, _d, _d]),
    "fy_dering_apply": (None, [_PD, _P, _l, _l, _l, _l, _l, _l, _d]),
    "fy_phase_correlate": (_i, [_P, _P, _i, _i, _i, _PDBL, _PDBL, _i]),
    "fy_hist_init": (None, [C.POINTER(HistState)]),
    "fy_hist_accumulate_u8": (None, [C.POINTER(HistState), _P, _sz]),
    "fy_hist_merge": (None, [C.POINTER(HistState), C.POINTER(HistState)]),
    "fy_hist_percentile_u8": (_i, [C.POINTER(HistState), _d]),
    "fy_hist_percentile_u8_inner": (_i, [C.POINTER(HistState), _d]),
    "fy_flat_noise": (_d, [_P, _i, _i, _i, _i]),
    "fy_noise_aniso": (_i, [_P, _i, _i, _i, _PDBL, _PDBL]),
    "fy_gpu_hist_accumulate_u8": (_i, [_P, _sz, _P, _P]),
    "fy_gpu_calib_scratch_bytes": (_sz, [_i, _i, _i, _i]),
    "fy_gpu_flat_noise": (_i, [_P, _i, _i, _i, _i, _P, _P, _P]),
    "fy_gpu_noise_aniso": (_i, [_P, _i, _i, _i, _P, _P, _P]),
    "fy_valley_depth": (_d, [_P, C.POINTER(_i), C.POINTER(_i), C.POINTER(_i)]),
    "fy_measure_psf_sigma": (_d, [_P, _i, _i, _i, C.POINTER(_i)]),
    "fy_gpu_measure_psf_sigma": (_i, [_P, _i, _i, _i, _P, _P]),
    "fy_process_buffer": (_i, [C.POINTER(PipelineCfg), _P, _l, _l, _l, _l, _l, _l, _l, _l, _l, _l, _l, _l, _l, _l,
                               _P, C.POINTER(_i)]),
    "fy_gpu_process_buffer": (_i, [C.POINTER(PipelineCfg), _P, _l, _l, _l, _l, _l, _l, _l, _l, _l, _l, _l, _l, _l,
                                   _l, _P, C.POINTER(_i), _P]),
    "fy_process_buffer_air_state": (_i, [_P, _P]),
    "fy_zarr_open": (_i, [C.POINTER(Zarr), C.c_char_p]),
    "fy_zarr_read": (_i, [C.POINTER(Zarr), _l, _l, _l, _l, _l, _l, _P]),
    "fy_process_chunk": (_i, [C.POINTER(Zarr), C.POINTER(PipelineCfg), _l, _l, _l, _i, _P, C.POINTER(_i),
                              C.POINTER(_i), C.POINTER(_i), C.POINTER(_i)]),
    "fy_gpu_zarr_read": (_i, [C.POINTER(Zarr), _l, _l, _l, _l, _l, _l, _P, _P]),
    "fy_gpu_autotune": (_i, [_i, _i, _i, _i]),
    "fy_gpu_tune_load": (_i, [C.c_char_p]),
    "fy_gpu_tune_value": (_i, [C.c_char_p]),
    "fy_gpu_zarr_cache_limit": (_i, [_sz]),
    "fy_gpu_zarr_cache_stats": (None, [C.POINTER(C.c_ulonglong), C.POINTER(C.c_ulonglong),
                                       C.POINTER(C.c_ulonglong)]),
    # ---- fy_gpu_* extension
    "fy_gpu_init": (_i, [_i]),
    "fy_gpu_last_status": (_i, []),
    "fy_gpu_last_error": (C.c_char_p, []),
    "fy_gpu_release": (None, []),
    "fy_gpu_kernel_launches": (C.c_ulonglong, []),
    "fy_gpu_kernel_timeouts": (_i, []),
    "fy_gpu_test_box_first_wait": (_i, [_i]),
    "fy_gpu_test_noise_paths": (_i, [_i, C.POINTER(C.c_int)]),
    "fy_gpu_u8_to_phys": (_i, [_P, _P, _sz, _d, _d, _P]),
    "fy_gpu_phys_to_u8": (_i, [_P, _P, _sz, _d, _d, _P]),
    "fy_gpu_deconvolve_ex": (_i, [_P, _i, _d, _d, _P, _i, _i, _i, _PP, _d, _i, _d, _P]),
    "fy_gpu_guided": (_i, [_P, _P, _i, _i, _i, _i, _d, _i, _P]),
    "fy_gpu_guided_scratch_bytes": (_sz, [_i, _i, _i, _i, _i]),
    "fy_gpu_noise_scratch_bytes": (_sz, [_i, _i, _i]),
    "fy_gpu_estimate_noise": (_i, [_P, _i, _i, _i, _i, _d, _d, _P, _P]),
    "fy_gpu_noise_model": (_i, [_P, _i, _i, _i, _PN, _P]),
    "fy_gpu_noise_eps": (_P, [_P, _i, _i, _i]),
    "fy_server_cfg_default": (None, [C.POINTER(ServerCfg)]),
    "fy_server_create": (_i, [C.POINTER(_P), C.POINTER(ServerCfg)]),
    "fy_server_submit": (_i, [_P, C.POINTER(Request), C.POINTER(C.c_longlong)]),
    "fy_server_wait": (_i, [_P, C.c_longlong, _d, C.POINTER(RequestResult)]),
    "fy_server_get_stats": (_i, [_P, C.POINTER(ServerStats)]),
    "fy_server_reset_stats": (None, [_P]),
    "fy_server_destroy": (None, [_P]),
    "fy_gpu_fit_radial_eps": (_i, [_P, _P, _i, _d, _P, _P]),
    "fy_fit_radial_eps": (_i, [_P, _P, _i, _d, C.POINTER(RadialEps)]),
    "fy_radial_tile_eps": (_d, [C.POINTER(RadialEps), _d, _d, _d, _l, _l, _l, _l]),
    "fy_gpu_estimate_noise_noalloc": (_i, [_P, _i, _i, _i, _i, _d, _d, _P, _P, _P]),
    "fy_gpu_dering_create": (_i, [C.POINTER(_P), _l, _l, _l, _d, _d, _i, _i]),
    "fy_gpu_dering_destroy": (None, [_P]),
    "fy_gpu_dering_reset": (_i, [_P, _P]),
    "fy_gpu_dering_accumulate_u8": (_i, [_P, _P, _l, _l, _l, _l, _l, _l, _i, _P]),
    "fy_gpu_dering_finalize": (_i, [_P, _i, C.c_uint, _d, _d, _P]),
    "fy_gpu_dering_apply": (_i, [_P, _P, _l, _l, _l, _l, _l, _l, _d, _P]),
    "fy_gpu_dering_download": (_i, [_P, _PD, C.POINTER(_l), _P]),
    "fy_gpu_phase_correlate_scratch_bytes": (_sz, [_i, _i, _i]),
    "fy_restore_cfg_default": (None, [C.c_void_p]),
    "fy_gpu_restore_u8": (_i, [_P, _P, _i, _i, _i, _d, _d, _PP, C.c_void_p, _P]),
    "fy_gpu_restore_u8_batch": (_i, [C.POINTER(BatchCube), _i, C.c_void_p, _P]),
    "fy_gpu_profile_start": (_i, [_i, _P]),
    "fy_gpu_profile_stop": (_i, []),
    "fy_gpu_profile_read": (_i, [_i, C.POINTER(C.c_char_p), C.POINTER(C.c_float)]),
    "fy_gpu_profile_select": (_i, [C.c_char_p]),
    "fy_gpu_phase_correlate_batch": (_i, [_P, _P, _i, _i, _i, _i, _i, _P, _PDBL, _PDBL,
                                          C.POINTER(C.c_longlong), C.POINTER(_i), _P]),
}

_lib = None


def load(path: str | os.PathLike | None = None) -> C.CDLL:
    """Load the CUDA library (once). Raises if it was not built: no fallback exists."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise ImportError(f"{p} is missing: build it with `python -m fysics_b200.build` "
                          "(fysics_b200 has no CPU fallback)")
    lib = C.CDLL(str(p), mode=C.RTLD_LOCAL)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


class FysicsError(RuntimeError):
    def __init__(self, rc: int, where: str):
        msg = load().fy_gpu_last_error()
        super().__init__(f"{where} failed with status {rc}: {msg.decode() if msg else ''}")
        self.rc = rc


def check(rc: int, where: str) -> int:
    if rc != 0:
        raise FysicsError(rc, where)
    return rc


def check_void(where: str) -> None:
    """For void entry points: raise if the call recorded a failure."""
    lib = load()
    st = lib.fy_gpu_last_status()
    if st != 0:
        raise FysicsError(st, where)
