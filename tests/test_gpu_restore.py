"""The per-cube restoration chain (fy_gpu_restore_u8) and the radial eps model.

Chain order as the reference's per-tile path: u8 dewindow -> matched Wiener deconvolution
-> noise model -> guided filter with eps = fy_guided_eps_for_noise(noise_ref) -> ring
subtraction (pipeline.c:252-443 order; each stage's own tolerance is stated in its test
file). Here the chain is checked
  - against the same stages called one by one through the device entry points: the
    kernels are the same, so the chain must match to 1e-6;
  - against the reference library's stages on the host, within 2e-3 absolute on [0, 1]
    data (deconvolution ~1e-6, noise_ref within 1e-3 relative moves eps, guided 3e-5).
Radial eps (pipeline.c:851-891, 445-456): fit, median and tile eps against the FP64 oracle.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from oracle import o64, p

pytestmark = pytest.mark.gpu

SHAPE = (40, 64, 72)


def phys(fb):
    return fb.physics(delta_beta=175.0, energy_kev=110.0, distance_mm=1200.0, pixel_um=2.4, unsharp_sigma=0.8,
                      unsharp_coeff=0.5, psf_sigma_vox=1.0, psf_sigma_z_vox=1.17)


def cube():
    import fysics_b200.phantom as ph
    u = ph.phantom(SHAPE, seed=11, delta_beta=175.0, pixel_um=2.4, fz2_scale=1.17 ** 2, rings=6, device="cpu")
    return np.ascontiguousarray(u.numpy() if hasattr(u, "numpy") else u)


def cfg_for(fb, dering):
    cfg = fb.RestoreCfg()
    fb.load().fy_restore_cfg_default(C.byref(cfg))
    cfg.deconv_kind = 1
    cfg.deconv_param = 0.05
    cfg.noise_win, cfg.noise_flat_pct, cfg.noise_ref_intensity = 5, 10.0, 0.4
    cfg.guided_radius, cfg.guided_s = 2, 1
    cfg.dering = dering
    cfg.dering_accumulate = 1 if dering else 0
    cfg.dering_ss, cfg.dering_hp_win, cfg.dering_min_cnt = 2, 15, 20
    cfg.dering_min_amp, cfg.dering_max_amp, cfg.dering_scale = 0.5, 6.0, 1.0 / 255.0
    return cfg


def run_chain(fb, u8, cfg_mod=None, with_rings=True):
    import torch
    lib = fb.load()
    nz, ny, nx = u8.shape
    d_in = torch.from_numpy(u8).cuda()
    d_out = torch.empty(u8.shape, dtype=torch.float32, device="cuda")
    h = C.c_void_p()
    if with_rings:
        assert lib.fy_gpu_dering_create(C.byref(h), nz, ny, nx, -1.0, -1.0, 512, 8) == 0
    cfg = cfg_for(fb, h if with_rings else None)
    if cfg_mod:
        cfg_mod(cfg)
    ph = phys(fb)
    torch.cuda.synchronize()
    rc = lib.fy_gpu_restore_u8(C.c_void_p(d_in.data_ptr()), C.c_void_p(d_out.data_ptr()), nz, ny, nx, 0.0, 1.0,
                               C.byref(ph), C.byref(cfg), None)
    assert rc == 0, lib.fy_gpu_last_error()
    torch.cuda.synchronize()
    if with_rings:
        lib.fy_gpu_dering_destroy(h)
    return d_out.cpu().numpy()


def run_steps(fb, u8):
    """The same stages through the individual device entry points."""
    import torch
    lib = fb.load()
    nz, ny, nx = u8.shape
    d_in = torch.from_numpy(u8).cuda()
    dec = torch.empty(u8.shape, dtype=torch.float32, device="cuda")
    ph = phys(fb)
    assert lib.fy_gpu_deconvolve_ex(C.c_void_p(d_in.data_ptr()), 1, 0.0, 1.0, C.c_void_p(dec.data_ptr()),
                                    nz, ny, nx, C.byref(ph), 0.05, 1, 1.0, None) == 0
    scratch = torch.empty(lib.fy_gpu_noise_scratch_bytes(nz, ny, nx), dtype=torch.uint8, device="cuda")
    assert lib.fy_gpu_estimate_noise(C.c_void_p(dec.data_ptr()), nz, ny, nx, 5, 10.0, 0.4,
                                     C.c_void_p(scratch.data_ptr()), None) == 0
    nm = fb.NoiseModel()
    assert lib.fy_gpu_noise_model(C.c_void_p(scratch.data_ptr()), nz, ny, nx, C.byref(nm), None) == 0
    eps = float(np.float32(lib.fy_guided_eps_for_noise(nm.noise_ref)))
    out = torch.empty_like(dec)
    assert lib.fy_gpu_guided(C.c_void_p(dec.data_ptr()), C.c_void_p(out.data_ptr()), nz, ny, nx, 2, eps, 1,
                             None) == 0
    torch.cuda.synchronize()
    return out.cpu().numpy(), nm


def ref_chain(u8, rings=True):
    L = oracle.ref()
    nz, ny, nx = u8.shape
    n = u8.size
    ph = oracle.ref_physics(delta_beta=175.0, energy_kev=110.0, distance_mm=1200.0, pixel_um=2.4,
                            unsharp_sigma=0.8, unsharp_coeff=0.5, psf_sigma_vox=1.0, psf_sigma_z_vox=1.17)
    f = np.empty(u8.shape, np.float32)
    L.fy_u8_to_phys(p(u8), p(f), n, 0.0, 1.0)
    d = np.empty_like(f)
    assert L.fy_deconvolve_matched(p(f), p(d), nz, ny, nx, C.byref(ph), 0.05) == 0
    nm = oracle.RefNoise()
    assert L.fy_estimate_noise(p(d), nz, ny, nx, 5, 10.0, 0.4, C.byref(nm)) == 0
    eps = L.fy_guided_eps_for_noise(nm.noise_ref)
    ws = np.empty(4 * n, np.float32)
    out = np.empty_like(f)
    assert L.fy_guided_denoise_ws(p(d), p(out), nz, ny, nx, 2, eps, p(ws)) == 0
    if rings:
        dr, dt = oracle.RefDering(), oracle.RefDering()
        assert L.fy_dering_init(C.byref(dr), nz, ny, nx, -1, -1, 512, 8) == 0
        assert L.fy_dering_tile_init(C.byref(dt), C.byref(dr)) == 0
        L.fy_dering_accumulate_u8(C.byref(dt), p(u8), 0, 0, nz, ny, nx, 2)
        L.fy_dering_merge_tile(C.byref(dr), 0, C.byref(dt))
        L.fy_dering_finalize(C.byref(dr), 15, 20, 0.5, 6.0)
        L.fy_dering_apply(C.byref(dr), p(out), 0, 0, 0, nz, ny, nx, 1.0 / 255.0)
        L.fy_dering_free(C.byref(dt))
        L.fy_dering_free(C.byref(dr))
    return out, nm


def test_chain_equals_stages(gpu):
    u8 = cube()
    chain = run_chain(gpu, u8, with_rings=False)
    steps, _ = run_steps(gpu, u8)
    assert np.abs(chain - steps).max() <= 1e-6


def test_chain_ring_subtraction_matches_separate_apply(gpu):
    """The chain folds the ring subtraction into the guided output pass; the result must
    equal the chain without rings followed by fy_gpu_dering_apply (dering.c:200-248)."""
    import torch
    lib = gpu.load()
    u8 = cube()
    nz, ny, nx = u8.shape
    fused = run_chain(gpu, u8, with_rings=True)
    plain = torch.from_numpy(run_chain(gpu, u8, with_rings=False)).cuda()
    d_u8 = torch.from_numpy(u8).cuda()
    h = C.c_void_p()
    assert lib.fy_gpu_dering_create(C.byref(h), nz, ny, nx, -1.0, -1.0, 512, 8) == 0
    assert lib.fy_gpu_dering_accumulate_u8(h, C.c_void_p(d_u8.data_ptr()), 0, 0, 0, nz, ny, nx, 2, None) == 0
    assert lib.fy_gpu_dering_finalize(h, 15, 20, 0.5, 6.0, None) == 0
    assert lib.fy_gpu_dering_apply(h, C.c_void_p(plain.data_ptr()), 0, 0, 0, nz, ny, nx, 1.0 / 255.0, None) == 0
    torch.cuda.synchronize()
    lib.fy_gpu_dering_destroy(h)
    sep = plain.cpu().numpy()
    assert np.array_equal(fused, sep)


@pytest.mark.skipif(not oracle.have_ref(), reason="reference library not built")
def test_chain_vs_reference(gpu):
    u8 = cube()
    got = run_chain(gpu, u8, with_rings=True)
    want, _ = ref_chain(u8, rings=True)
    assert np.isfinite(got).all()
    err = np.abs(got - want)
    assert err.max() <= 2e-3, err.max()
    assert err.mean() <= 5e-5, err.mean()


def test_chain_radial_eps_scales_guided(gpu):
    """A radial model in the chain equals a fixed eps pre-scaled by fy_radial_tile_eps."""
    import torch
    lib = gpu.load()
    u8 = cube()
    r = np.linspace(20.0, 900.0, 64)
    floors = 0.004 + 1.5e-5 * r
    fit = gpu.RadialEps()
    assert lib.fy_fit_radial_eps(p(r), p(floors), r.size, 3.0, C.byref(fit)) == 0
    assert fit.have == 1
    d_fit = torch.from_numpy(np.frombuffer(bytes(fit), np.uint8).copy()).cuda()
    base = 2.0 ** -9                                   # exactly representable: both paths round once
    cy, cx, y0, x0 = 700.0, 650.0, 96, 160
    tile = lib.fy_radial_tile_eps(C.byref(fit), base, cy, cx, y0, x0, SHAPE[1], SHAPE[2])
    assert tile > 0 and tile != base

    def radial(cfg):
        cfg.guided_eps = base
        cfg.radial = d_fit.data_ptr()
        cfg.radial_cy, cfg.radial_cx = cy, cx
        cfg.y0, cfg.x0 = y0, x0

    def fixed(cfg):
        cfg.guided_eps = tile
        cfg.y0, cfg.x0 = y0, x0

    a = run_chain(gpu, u8, radial, with_rings=False)
    b = run_chain(gpu, u8, fixed, with_rings=False)
    assert np.array_equal(a, b)
    c = run_chain(gpu, u8, lambda cfg: setattr(cfg, "guided_eps", base), with_rings=False)
    assert not np.array_equal(a, c)


def o64_fit(r, f):
    a, b, cc = C.c_double(), C.c_double(), C.c_double()
    have = o64().o64_fit_radial_eps(p(r), p(f), r.size, C.byref(a), C.byref(b), C.byref(cc))
    return have, a.value, b.value, cc.value


def close(x, y, rel=1e-12):
    return abs(x - y) <= rel * max(abs(y), 1e-300)


@pytest.mark.parametrize("case", ["rising", "flat", "few", "none", "noisy", "ties"])
def test_radial_fit_vs_oracle(gpu, case):
    lib = gpu.load()
    rng = np.random.default_rng(5)
    r = np.sort(rng.uniform(10, 1200, 200))
    f = {"rising": 0.01 + 2e-5 * r,
         "flat": 0.01 + 1e-6 * np.sin(r),
         "few": (0.01 + 2e-5 * r)[:7],
         "none": np.zeros(0),
         "noisy": 0.01 + 2e-5 * r + rng.normal(0, 2e-3, r.size),
         "ties": np.round(0.01 + 2e-5 * r, 3)}[case]
    r = r[:f.size].copy()
    f = np.ascontiguousarray(f)
    fit = gpu.RadialEps()
    assert lib.fy_fit_radial_eps(p(r), p(f), r.size, 0.0, C.byref(fit)) == 0, lib.fy_gpu_last_error()
    have, a, b, cc = o64_fit(r, f)
    assert fit.n == r.size and fit.have == have
    if r.size >= 8:
        # a, b: well conditioned; corr in [-1, 1] carries the cancellation of nn*srf - sr*sf
        # (flat floors), where FMA contraction alone moves it by ~1e-10
        assert close(fit.a, a, 1e-9) and close(fit.b, b, 1e-9) and abs(fit.corr - cc) <= 1e-7
    med = o64().o64_median_floor(p(f), f.size)
    assert fit.median == med                                   # order statistic: exact
    assert close(fit.guided_eps, (4.2 * med) ** 2)


def test_radial_device_form_and_disabled_denoise(gpu):
    import torch
    lib = gpu.load()
    r = np.linspace(10, 1000, 256)
    f = 0.008 + 3e-5 * r
    d_r, d_f = torch.from_numpy(r).cuda(), torch.from_numpy(f).cuda()
    d_fit = torch.zeros(C.sizeof(gpu.RadialEps), dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    assert lib.fy_gpu_fit_radial_eps(C.c_void_p(d_r.data_ptr()), C.c_void_p(d_f.data_ptr()), 256, -1.0,
                                     C.c_void_p(d_fit.data_ptr()), None) == 0
    torch.cuda.synchronize()
    fit = gpu.RadialEps.from_buffer_copy(d_fit.cpu().numpy().tobytes())
    have, a, b, cc = o64_fit(r, f)
    assert fit.have == have == 1 and close(fit.a, a, 1e-9) and close(fit.b, b, 1e-9)
    assert fit.guided_eps == 0.0                               # denoise_k < 0: disabled
    assert lib.fy_gpu_fit_radial_eps(C.c_void_p(d_r.data_ptr()), C.c_void_p(d_f.data_ptr()), 257, 0.0,
                                     C.c_void_p(d_fit.data_ptr()), None) == 1   # FY_EINVAL: > 256 samples
