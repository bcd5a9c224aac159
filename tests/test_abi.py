"""C-ABI surface (CPU): the library loads, exports every symbol include/fysics_b200.h
declares, and -- with no usable GPU -- refuses to compute instead of falling back."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from tests.conftest import has_cuda

HEADER = Path(__file__).resolve().parents[1] / "include" / "fysics_b200.h"


def declared():
    src = HEADER.read_text()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = set(re.findall(r"\b(fy_[a-z0-9_]+)\s*\(", src))
    return sorted(names)


def test_header_declares_the_drop_in_set():
    names = set(declared())
    # the fysics.h entry points on the restoration path
    required = {
        "fy_u8_to_phys", "fy_phys_to_u8", "fy_float_to_u8", "fy_u8_to_float", "fy_phys_to_u8_level",
        "fy_fft1d", "fy_fft3d", "fy_fft3d_normalize", "fy_next_fft_size", "fy_is_pow2",
        "fy_next_pow2", "fy_paganin_transfer", "fy_unsharp_transfer", "fy_recon_transfer",
        "fy_auto_reg", "fy_auto_deltabeta_scale", "fy_kernel_halo", "fy_deconvolve",
        "fy_deconvolve_matched", "fy_guided_denoise", "fy_guided_denoise_ws",
        "fy_guided_denoise_fast_ws", "fy_guided_ws_floats", "fy_box_smooth",
        "fy_estimate_noise", "fy_guided_eps_for_noise", "fy_dering_init", "fy_dering_free",
        "fy_dering_tile_init", "fy_dering_tile_reset", "fy_dering_accumulate_u8",
        "fy_dering_merge_tile", "fy_dering_finalize", "fy_dering_apply", "fy_phase_correlate",
        # the per-tile export chain and the pass-1 calibration helpers
        "fy_process_buffer", "fy_valley_depth", "fy_hist_accumulate_u8", "fy_flat_noise", "fy_noise_aniso",
    }
    assert required <= names, sorted(required - names)


def test_library_exports_every_declared_symbol(fy):
    lib = fy.load()
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_ctypes_signatures_cover_header(fy):
    assert set(declared()) <= set(fy.SIGNATURES), sorted(set(declared()) - set(fy.SIGNATURES))


def test_struct_layouts_match_reference():
    import fysics_b200 as fb
    assert C.sizeof(fb.Physics) == 64                      # fysics.h:23-35, 8 doubles
    assert C.sizeof(fb.NoiseModel) == 40                    # 4 doubles + int (+pad)
    assert fb.Dering.ring.offset == 72 and C.sizeof(fb.Dering) == 88
    # fy_pipeline_cfg (fysics.h:436-491): 440 bytes on LP64, the ring handle at 304
    assert C.sizeof(fb.PipelineCfg) == 440 and fb.PipelineCfg.dering.offset == 304
    import oracle
    assert [(n, getattr(fb.PipelineCfg, n).offset) for n, _ in fb.PipelineCfg._fields_] == \
        [(n, getattr(oracle.RefPipelineCfg, n).offset) for n, _ in oracle.RefPipelineCfg._fields_]


def test_scalar_helpers_match_reference(fy):
    """Plan-time scalar helpers are host math; compare with the reference's values."""
    import oracle
    lib = fy.load()
    assert [lib.fy_next_fft_size(n) for n in (176, 128, 160, 97)] == [192, 128, 192, 128]
    assert lib.fy_is_pow2(64) and not lib.fy_is_pow2(96) and lib.fy_next_pow2(97) == 128
    ph = fy.physics()
    if oracle.have_ref():
        rph = oracle.ref_physics()
        R = oracle.ref()
        # FP64 scalars: the -Ofast reference build reassociates/contracts, so agree to 1e-14
        for f in (0.0, 0.05, 0.1, 0.25, 0.5, 0.7):
            for fn in ("fy_paganin_transfer", "fy_unsharp_transfer", "fy_recon_transfer"):
                a, b = getattr(lib, fn)(f, C.byref(ph)), getattr(R, fn)(f, C.byref(rph))
                assert abs(a - b) <= 1e-14 * abs(b), (fn, f, a, b)
        a, b = lib.fy_auto_deltabeta_scale(C.byref(ph)), R.fy_auto_deltabeta_scale(C.byref(rph))
        assert abs(a - b) <= 1e-14 * abs(b)
        for args in ((0.0, -0.03, 0.145), (0.1, -0.03, 0.21), (0.5, 0.0, 0.0)):
            assert lib.fy_phys_to_u8_level(*args) == R.fy_phys_to_u8_level(*args)
    assert lib.fy_guided_eps_for_noise(0.0) == 1e-8
    assert abs(lib.fy_guided_eps_for_noise(0.01) - 9e-4) < 1e-18


@pytest.mark.skipif(has_cuda(), reason="a GPU is present: the no-device contract is not observable")
def test_no_cpu_fallback_without_gpu(fy):
    lib = fy.load()
    a = np.ones((4, 4, 4), np.float32)
    out = np.full_like(a, -7.0)
    rc = lib.fy_deconvolve(a.ctypes.data, out.ctypes.data, 4, 4, 4, C.byref(fy.physics()), 0.015)
    assert rc == fy.FY_ENODEV
    assert b"no CPU fallback" in lib.fy_gpu_last_error()
    assert (out == -7.0).all()                              # nothing computed on the host
    u8 = np.arange(16, dtype=np.uint8)
    f = np.full(16, -1.0, np.float32)
    lib.fy_u8_to_phys(u8.ctypes.data, f.ctypes.data, 16, 0.0, 1.0)
    assert lib.fy_gpu_last_status() == fy.FY_ENODEV and (f == -1.0).all()


@pytest.mark.skipif(has_cuda(), reason="a GPU is present: the no-device contract is not observable")
def test_server_refuses_without_gpu(fy):
    lib = fy.load()
    h = C.c_void_p(123)
    cfg = fy.ServerCfg()
    lib.fy_server_cfg_default(C.byref(cfg))
    assert cfg.workers == 8 and cfg.small_workers == 2 and cfg.hbm_budget_bytes == 150 << 30
    assert lib.fy_server_create(C.byref(h), C.byref(cfg)) == fy.FY_ENODEV
    assert h.value is None                                  # no handle, no worker threads


@pytest.mark.skipif(has_cuda(), reason="a GPU is present: the no-device contract is not observable")
def test_tile_chain_and_psf_refuse_without_gpu(fy):
    """The per-tile chain and the PSF edge fit have no CPU fallback either."""
    lib = fy.load()
    cfg = fy.PipelineCfg()
    cfg.do_air_zero = 1
    buf = np.full((12, 12, 12), 90, np.uint8)
    out = np.full((8, 8, 8), 0xCD, np.uint8)
    air = C.c_int(-7)
    rc = lib.fy_process_buffer(C.byref(cfg), buf.ctypes.data, 0, 0, 0, 12, 12, 12, 2, 2, 2, 8, 8, 8, 12, 12,
                               out.ctypes.data, C.byref(air))
    assert rc == fy.FY_ENODEV and (out == 0xCD).all() and air.value == -7
    assert lib.fy_process_buffer(C.byref(cfg), buf.ctypes.data, 0, 0, 0, 12, 12, 12, 2, 2, 2, 8, 8, 11, 12, 12,
                                 out.ctypes.data, C.byref(air)) == fy.FY_EINVAL   # geometry is checked first
    n = C.c_int(-3)
    assert np.isnan(lib.fy_measure_psf_sigma(buf.ctypes.data, 12, 12, 12, C.byref(n)))
    assert lib.fy_gpu_last_status() == fy.FY_ENODEV and n.value == -3
