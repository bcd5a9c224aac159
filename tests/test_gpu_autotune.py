"""Autotuner (fy_gpu_autotune): measured launch shapes cached per GPU.

Every knob only changes how work is split over CTAs (lines per CTA of the deconvolution X
passes, z chunks of the box passes), so the chain's output must stay bit-identical whatever
the cache holds: checked with forced, non-default values loaded from a cache file, and after a
real tuning run, whose cache file must then hold this device's entries and reload."""
import ctypes as C
import json

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPE = (96, 200, 320)          # an uneven-cube shape of the batched configuration (x pads to 384)


def chain(fb, u8):
    import torch
    lib = fb.load()
    nz, ny, nx = u8.shape
    d_in = torch.from_numpy(u8).cuda()
    out = torch.empty(u8.shape, dtype=torch.float32, device="cuda")
    ph = fb.physics(delta_beta=175.0, energy_kev=110.0, distance_mm=1200.0, pixel_um=2.4, unsharp_sigma=0.8,
                    unsharp_coeff=0.5, psf_sigma_vox=1.0, psf_sigma_z_vox=1.17)
    cfg = fb.RestoreCfg()
    lib.fy_restore_cfg_default(C.byref(cfg))
    cfg.deconv_kind, cfg.deconv_param = 1, 0.05
    torch.cuda.synchronize()
    assert lib.fy_gpu_restore_u8(C.c_void_p(d_in.data_ptr()), C.c_void_p(out.data_ptr()), nz, ny, nx, 0.0, 1.0,
                                 C.byref(ph), C.byref(cfg), None) == 0, lib.fy_gpu_last_error()
    torch.cuda.synchronize()
    return out.cpu().numpy()


def cube():
    import fysics_b200.phantom as ph
    u = ph.phantom(SHAPE, seed=4, delta_beta=175.0, pixel_um=2.4, fz2_scale=1.17 ** 2, device="cpu")
    return np.ascontiguousarray(u.numpy() if hasattr(u, "numpy") else u)


def test_forced_shapes_are_bit_identical(gpu, tmp_path, monkeypatch):
    lib = gpu.load()
    empty = tmp_path / "none.json"
    assert lib.fy_gpu_tune_load(str(empty).encode()) == 0
    u8 = cube()
    want = chain(gpu, u8)
    # a tuning run into a scratch cache gives this device's key; then a cache with that key
    # and non-default values for every knob of the shape
    path = tmp_path / "seed.json"
    monkeypatch.setenv("FY_TUNE_CACHE", str(tmp_path / "probe.json"))
    assert lib.fy_gpu_tune_load(str(tmp_path / "probe.json").encode()) == 0
    assert lib.fy_gpu_autotune(*SHAPE, 1) == 0, lib.fy_gpu_last_error()
    lines = [json.loads(ln) for ln in (tmp_path / "probe.json").read_text().splitlines()]
    dev = lines[0]["device"]
    assert all(ln["device"] == dev for ln in lines)
    knobs = {ln["knob"] for ln in lines}
    assert knobs == {"x1.384", "x5.384"}
    forced = {"x1.384": 2, "x5.384": 1}
    path.write_text("".join(json.dumps({"device": dev, "knob": k, "value": v, "ms": 0.0}) + "\n"
                            for k, v in forced.items()))
    assert lib.fy_gpu_tune_load(str(path).encode()) == 2
    for k, v in forced.items():
        assert lib.fy_gpu_tune_value(k.encode()) == v
    got = chain(gpu, u8)
    assert np.array_equal(got, want)
    # another device's entries are ignored
    path.write_text(json.dumps({"device": "other|sm1|drv1|rt1", "knob": "x1.384", "value": 1, "ms": 0}) + "\n")
    assert lib.fy_gpu_tune_load(str(path).encode()) == 1
    assert lib.fy_gpu_tune_value(b"x1.384") == 0
    assert np.array_equal(chain(gpu, u8), want)


def test_tuning_run_keeps_results(gpu, tmp_path, monkeypatch):
    lib = gpu.load()
    path = tmp_path / "tune.json"
    monkeypatch.setenv("FY_TUNE_CACHE", str(path))
    assert lib.fy_gpu_tune_load(str(path).encode()) == 0
    u8 = cube()
    want = chain(gpu, u8)
    assert lib.fy_gpu_autotune(*SHAPE, 0) == 0, lib.fy_gpu_last_error()
    entries = [json.loads(ln) for ln in path.read_text().splitlines()]
    assert len(entries) == 2 and all(e["value"] > 0 and e["ms"] > 0 for e in entries)
    assert np.array_equal(chain(gpu, u8), want)
    assert lib.fy_gpu_tune_load(str(path).encode()) == 2           # reloads what it wrote
    assert lib.fy_gpu_autotune(*SHAPE, 0) == 0                      # cached: no re-measurement
    assert [json.loads(ln) for ln in path.read_text().splitlines()] == entries
    assert lib.fy_gpu_tune_load(str(tmp_path / "absent.json").encode()) == 0   # leave the defaults on
