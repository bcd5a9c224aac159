"""Per-stage error of the plain 128^3 chain on the GPU, against the reference and the FP64 oracle.

The chain is the CPU-runnable benchmark recipe: a seeded 128^3 scroll phantom (pixel
7.91 um, delta_beta 500, Poisson-Gaussian noise, window [0, 1]), u8 -> phys, Wiener
deconvolution (reg 0.015), noise model (win 5, 10th percentile, ref 0.4), guided filter
(r 2, eps = (3 noise_ref)^2). Every stage runs on the reference's output of the stage
before it, so each stage's error is its own and errors do not compound.

Bars (the window range is 1): u8 -> phys bit-exact; deconvolution and guided filter max
abs error <= 1e-4 against both the reference and the FP64 oracle; noise_ref within 1e-3
relative and the bin count exact. Each stage prints its measured errors (pytest -s).
"""
import ctypes as C

import numpy as np
import pytest

import fysics_b200.phantom as ph
import oracle
from oracle import p
from tests.test_gpu_guided import gpu_guided, o64_guided, ref_guided
from tests.test_gpu_noise import close, gpu_noise, o64_noise, ref_noise

pytestmark = pytest.mark.gpu
TOL = 1e-4


def rphys(phy):
    return oracle.RefPhysics(*[getattr(phy, n) for n, _ in phy._fields_])


@pytest.mark.skipif(not oracle.have_ref(), reason="needs the compiled reference")
def test_stage_errors_plain_128(gpu):
    u8 = ph.phantom((128, 128, 128), seed=20260101, device="cpu")
    u8 = np.ascontiguousarray(u8.numpy() if hasattr(u8, "numpy") else u8, np.uint8)
    lib = gpu.load()
    report = {}

    # u8 -> phys
    got = np.empty(u8.shape, np.float32)
    lib.fy_u8_to_phys(p(u8), p(got), u8.size, 0.0, 1.0)
    ref_f = oracle.ref_u8_to_phys(u8, 0.0, 1.0)
    assert np.array_equal(got, ref_f)
    o64_f = np.empty(u8.shape, np.float64)
    oracle.o64().o64_u8_to_phys(p(u8), p(o64_f), u8.size, 0.0, 1.0)
    report["u8_to_phys"] = (0.0, float(np.abs(got - o64_f).max()))
    assert report["u8_to_phys"][1] < 1e-7                      # float rounding of u8/255

    # Wiener deconvolution
    phy = gpu.physics(delta_beta=500.0, energy_kev=110.0, distance_mm=1200.0, pixel_um=7.91,
                      unsharp_sigma=0.8, unsharp_coeff=0.5)
    got = gpu.deconvolve(ref_f, phy, 0.015)
    ref_d = oracle.ref_deconvolve(ref_f, rphys(phy), 0.015)
    o64_d = oracle.o64_deconvolve(ref_f, rphys(phy), 0.015, kind=0)
    report["deconvolve"] = (float(np.abs(got - ref_d).max()), float(np.abs(got - o64_d).max()))
    assert max(report["deconvolve"]) < TOL

    # noise model
    g, r, o = gpu_noise(gpu, ref_d, 5, 10.0, 0.4), ref_noise(ref_d, 5, 10.0, 0.4), o64_noise(ref_d, 5, 10.0, 0.4)
    assert g.n_bins_used == r.n_bins_used == o.n_bins_used
    assert close(g.noise_ref, r.noise_ref) and close(g.noise_ref, o.noise_ref)
    report["noise_ref (rel)"] = (abs(g.noise_ref - r.noise_ref) / r.noise_ref,
                                 abs(g.noise_ref - o.noise_ref) / o.noise_ref)

    # guided filter with the reference's eps
    eps = float(np.float32(oracle.ref().fy_guided_eps_for_noise(r.noise_ref)))
    got = gpu_guided(gpu, ref_d, 2, eps)
    report["guided"] = (float(np.abs(got - ref_guided(ref_d, 2, eps)).max()),
                        float(np.abs(got - o64_guided(ref_d, 2, eps)).max()))
    assert max(report["guided"]) < TOL

    for stage, (er, eo) in report.items():
        print(f"STAGE {stage:16s} vs reference {er:.3e}  vs FP64 oracle {eo:.3e}")
