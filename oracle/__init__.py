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
            raise FileNotFoundError(f"{REF_SO} missing: run `make -C oracle ref` where the "
                                    "reference sources are available")
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
