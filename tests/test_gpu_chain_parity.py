"""The whole restoration chain at the benchmark configurations, against the reference's chain
and the FP64 oracle's chain.

Bar (written here, the hot path's float bar): max abs error <= 1e-4 of the window range on
the chain's float output, against BOTH
  - the reference library's chain (its public calls in the configuration order: dewindow,
    fy_deconvolve or fy_deconvolve_matched, fy_estimate_noise, fy_guided_denoise_ws with
    eps = fy_guided_eps_for_noise(noise_ref), then fy_dering_accumulate_u8 / finalize /
    apply), and
  - the FP64 oracle's chain (the same stages in double, each fed the previous double stage).
The GPU output is the fused chain fy_gpu_restore_u8. Every stage's error against both is
printed (a `CHAIN_ERR {json}` line under `pytest -s`): the device entry points run the
same kernels stage by stage, each fed the GPU's own previous stage, so errors carry
through the noise model's percentile and bin decisions into eps exactly as in the chain.
The ring vote (detected count) must be equal.

Workloads (seeded phantoms of the benchmark recipe):
  config 1   128^3, isotropic Paganin + unsharp (delta_beta 500, 110 keV, 1.2 m, 7.91 um,
             unsharp 0.5 / 0.8), fy_deconvolve reg 0.015, noise (5, 10, 0.4), guided r 2;
  config 2   the 512^3 configuration's recipe on a 256^3 cube: pixel 2.4 um, delta_beta x
             fy_auto_deltabeta_scale, matched anisotropic PSF 1.0 / 1.17 (gamma 0.05),
             40 rings about the axis, dering (ss 2; vote 15, 100, 0.5, 6.0; scale 1/255).
"""
import ctypes as C
import json

import numpy as np
import pytest

import oracle
from oracle.chain import ChainSpec, o64_restore, ref_restore

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not oracle.have_ref(), reason="reference library not built")]

TOL = 1e-4          # of the window range


def spec_for(name, fb):
    if name == "config1":
        phys = dict(delta_beta=500.0, energy_kev=110.0, distance_mm=1200.0, pixel_um=7.91, unsharp_sigma=0.8,
                    unsharp_coeff=0.5)
        return (128, 128, 128), ChainSpec(phys=phys, matched=False, deconv_param=0.015), dict(rings=0)
    phys = dict(delta_beta=500.0, energy_kev=110.0, distance_mm=1200.0, pixel_um=2.4, unsharp_sigma=0.8,
                unsharp_coeff=0.5, psf_sigma_vox=1.0, psf_sigma_z_vox=1.17)
    fp = fb.physics(**phys)
    phys["delta_beta"] *= fb.load().fy_auto_deltabeta_scale(C.byref(fp))
    dering = dict(ss=2, hp_win=15, min_cnt=100, min_amp=0.5, max_amp=6.0, slab_z=512, ns=8)
    return (256, 256, 256), ChainSpec(phys=phys, matched=True, deconv_param=0.05, dering=dering), \
        dict(rings=40, fz2_scale=1.17 ** 2)


def make_cube(shape, spec, extra, seed):
    import fysics_b200.phantom as ph
    import torch
    u = ph.phantom(shape, seed=seed, delta_beta=spec.phys["delta_beta"], energy_kev=spec.phys["energy_kev"],
                   distance_mm=spec.phys["distance_mm"], pixel_um=spec.phys["pixel_um"],
                   unsharp_sigma=spec.phys["unsharp_sigma"], unsharp_coeff=spec.phys["unsharp_coeff"],
                   fz2_scale=extra.get("fz2_scale", 1.0), rings=extra["rings"], device="cuda")
    torch.cuda.synchronize()
    return np.ascontiguousarray(u.cpu().numpy())


def gpu_chain(fb, u8, spec):
    """fy_gpu_restore_u8 (the fused chain) and the same stages through the device entry
    points; returns the fused output and the staged intermediates."""
    import torch
    lib = fb.load()
    nz, ny, nx = u8.shape
    ph = fb.physics(**spec.phys)
    d_in = torch.from_numpy(u8).cuda()
    out = torch.empty(u8.shape, dtype=torch.float32, device="cuda")
    h = C.c_void_p()
    cfg = fb.RestoreCfg()
    lib.fy_restore_cfg_default(C.byref(cfg))
    cfg.deconv_kind = 1 if spec.matched else 0
    cfg.deconv_param = spec.deconv_param
    cfg.noise_win, cfg.noise_flat_pct, cfg.noise_ref_intensity = spec.noise_win, spec.noise_pct, spec.noise_ref
    cfg.guided_radius, cfg.guided_s = spec.guided_r, 1
    g = spec.dering
    if g:
        assert lib.fy_gpu_dering_create(C.byref(h), nz, ny, nx, -1.0, -1.0, g["slab_z"], g["ns"]) == 0
        cfg.dering = h
        cfg.dering_accumulate = 1
        cfg.dering_ss, cfg.dering_hp_win, cfg.dering_min_cnt = g["ss"], g["hp_win"], g["min_cnt"]
        cfg.dering_min_amp, cfg.dering_max_amp, cfg.dering_scale = g["min_amp"], g["max_amp"], spec.ring_scale()
    torch.cuda.synchronize()
    rc = lib.fy_gpu_restore_u8(C.c_void_p(d_in.data_ptr()), C.c_void_p(out.data_ptr()), nz, ny, nx, *spec.window,
                               C.byref(ph), C.byref(cfg), None)
    assert rc == 0, lib.fy_gpu_last_error()
    torch.cuda.synchronize()
    res = {"out": out.cpu().numpy()}
    if g:
        d = fb.Dering()
        assert lib.fy_dering_init(C.byref(d), nz, ny, nx, -1, -1, g["slab_z"], g["ns"]) == 0
        det = C.c_long()
        assert lib.fy_gpu_dering_download(h, C.byref(d), C.byref(det), None) == 0
        res["detected"] = det.value
        lib.fy_dering_free(C.byref(d))
        lib.fy_gpu_dering_destroy(h)
    # the stages one by one (same kernels), each fed the GPU's previous stage
    dec = torch.empty(u8.shape, dtype=torch.float32, device="cuda")
    assert lib.fy_gpu_deconvolve_ex(C.c_void_p(d_in.data_ptr()), 1, *spec.window, C.c_void_p(dec.data_ptr()),
                                    nz, ny, nx, C.byref(ph), spec.deconv_param, 1 if spec.matched else 0, 1.0,
                                    None) == 0
    scratch = torch.empty(lib.fy_gpu_noise_scratch_bytes(nz, ny, nx), dtype=torch.uint8, device="cuda")
    assert lib.fy_gpu_estimate_noise(C.c_void_p(dec.data_ptr()), nz, ny, nx, spec.noise_win, spec.noise_pct,
                                     spec.noise_ref, C.c_void_p(scratch.data_ptr()), None) == 0
    nm = fb.NoiseModel()
    assert lib.fy_gpu_noise_model(C.c_void_p(scratch.data_ptr()), nz, ny, nx, C.byref(nm), None) == 0
    del scratch
    eps = float(np.float32(lib.fy_guided_eps_for_noise(nm.noise_ref)))
    gd = torch.empty_like(dec)
    assert lib.fy_gpu_guided(C.c_void_p(dec.data_ptr()), C.c_void_p(gd.data_ptr()), nz, ny, nx, spec.guided_r, eps, 1,
                             None) == 0
    torch.cuda.synchronize()
    res.update(deconv=dec.cpu().numpy(), noise=nm, guided=gd.cpu().numpy())
    return res


def rel(a, b):
    return abs(a - b) / max(abs(b), 1e-300)


@pytest.mark.parametrize("name", ["config1", "config2_256"])
def test_chain_vs_reference_and_fp64(gpu, name):
    shape, spec, extra = spec_for(name, gpu)
    u8 = make_cube(shape, spec, extra, seed=2026)
    g = gpu_chain(gpu, u8, spec)
    r = ref_restore(u8, spec)
    o = o64_restore(u8, spec)
    span = spec.window[1] - spec.window[0]
    err = {}
    for st in ("deconv", "guided", "out"):
        err[st] = {"gpu_vs_ref": float(np.abs(g[st] - r[st]).max() / span),
                   "gpu_vs_fp64": float(np.abs(g[st] - o[st]).max() / span),
                   "ref_vs_fp64": float(np.abs(r[st] - o[st]).max() / span)}
    err["out"]["gpu_vs_ref_mean"] = float(np.abs(g["out"] - r["out"]).mean() / span)
    err["noise_ref_rel"] = {"gpu_vs_ref": rel(g["noise"].noise_ref, r["noise"].noise_ref),
                            "gpu_vs_fp64": rel(g["noise"].noise_ref, o["noise"].noise_ref),
                            "ref_vs_fp64": rel(r["noise"].noise_ref, o["noise"].noise_ref)}
    err["bins"] = [g["noise"].n_bins_used, r["noise"].n_bins_used, o["noise"].n_bins_used]
    if spec.dering:
        err["detected"] = [g["detected"], r["detected"], o["detected"]]
    print("CHAIN_ERR " + json.dumps({"case": name, "shape": shape, **err}))
    assert np.isfinite(g["out"]).all()
    assert g["noise"].n_bins_used == r["noise"].n_bins_used == o["noise"].n_bins_used
    if spec.dering:
        assert g["detected"] == r["detected"] == o["detected"] and g["detected"] >= 2
    # the fused chain equals its stages (ring subtraction aside: it is folded into the output pass)
    if not spec.dering:
        assert np.abs(g["out"] - g["guided"]).max() <= 1e-6 * span
    assert err["out"]["gpu_vs_ref"] <= TOL, err
    assert err["out"]["gpu_vs_fp64"] <= TOL, err
