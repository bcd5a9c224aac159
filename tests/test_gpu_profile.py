"""Per-pass CUDA-event marks (fy_gpu_profile_*): every instrumented pass of the chain records a
mark, and fy_gpu_profile_select keeps only the named ones, whose spans then cover everything
since the previous kept mark (the sum of the spans is the same chain either way)."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _chain(fb, lib, u8, out, names):
    import torch
    cfg = fb.RestoreCfg()
    lib.fy_restore_cfg_default(C.byref(cfg))
    cfg.deconv_kind, cfg.deconv_param = 1, 0.05
    cfg.noise_win, cfg.noise_flat_pct, cfg.noise_ref_intensity = 5, 10.0, 0.4
    cfg.guided_radius, cfg.guided_s = 2, 1
    phys = fb.physics(delta_beta=500.0, energy_kev=110.0, distance_mm=1200.0, pixel_um=2.4, unsharp_sigma=0.8,
                      unsharp_coeff=0.5, psf_sigma_vox=1.0, psf_sigma_z_vox=1.17)
    assert lib.fy_gpu_profile_select(names) == 0
    assert lib.fy_gpu_profile_start(64, None) == 0
    rc = lib.fy_gpu_restore_u8(C.c_void_p(u8.data_ptr()), C.c_void_p(out.data_ptr()), *u8.shape, 0.0, 1.0,
                               C.byref(phys), C.byref(cfg), None)
    assert rc == 0, lib.fy_gpu_last_error()
    torch.cuda.synchronize()
    cnt = lib.fy_gpu_profile_stop()
    marks = []
    for i in range(1, cnt):
        nm, ms = C.c_char_p(), C.c_float()
        assert lib.fy_gpu_profile_read(i, C.byref(nm), C.byref(ms)) == 0
        marks.append((nm.value.decode(), ms.value))
    assert lib.fy_gpu_profile_select(None) == 0
    return marks


def test_profile_select_keeps_named_marks(gpu):
    import torch
    import fysics_b200.phantom as ph
    lib = gpu.load()
    shape = (64, 72, 80)
    u8 = ph.phantom(shape, seed=3, delta_beta=500.0, pixel_um=2.4, fz2_scale=1.17 ** 2, device="cuda")
    out = torch.empty(shape, dtype=torch.float32, device="cuda")
    _chain(gpu, lib, u8, out, None)                               # warm-up: tables, workspaces
    every = _chain(gpu, lib, u8, out, None)
    names = [n for n, _ in every]
    for want in ("deconv.x_fwd", "deconv.z_weight", "deconv.x_inv", "noise.stats", "noise", "guided"):
        assert want in names, names
    assert all(ms >= 0 for _, ms in every)
    ref = out.clone()
    kept = _chain(gpu, lib, u8, out, b"noise, guided")
    assert [n for n, _ in kept] == ["noise", "guided"], kept
    assert all(ms > 0 for _, ms in kept)
    assert torch.equal(out, ref)                                  # marks change no result
    # the guided pass's own span is the same pass either way (events around it in both runs)
    g_every = dict(every)["guided"]
    g_kept = dict(kept)["guided"]
    assert 0.2 * g_every <= g_kept <= 5 * g_every + 0.05, (g_every, g_kept)
