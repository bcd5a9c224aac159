"""The drop-in link test: the reference's own pipeline.c (its fy_process_buffer,
pipeline.c:467-510) compiled unmodified and linked against libfysics_b200 first
(oracle/_ref/libpipeline_b200.so, oracle/Makefile). Its calls to fy_deconvolve*,
fy_guided_denoise_fast_ws, fy_box_smooth, fy_valley_depth and fy_dering_apply then run on
the GPU library; its output is compared with the all-reference build's.
"""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

import oracle
from tests.conftest import has_cuda
from tests.test_tile_oracle import MISMATCH_FRAC, VOL, tile_of
from tests._tiles import scroll_volume

LINKED = Path(oracle.__file__).resolve().parent / "_ref" / "libpipeline_b200.so"
pytestmark = pytest.mark.skipif(not (LINKED.exists() and oracle.have_ref()),
                                reason="needs the reference sources relinked against the library")


def linked():
    import fysics_b200
    fysics_b200.load()                      # the GPU library first in the process
    lib = C.CDLL(str(LINKED), mode=C.RTLD_LOCAL)
    lib.fy_process_buffer.restype = C.c_int
    lib.fy_process_buffer.argtypes = ([C.POINTER(oracle.RefPipelineCfg), C.c_void_p] + [C.c_long] * 14 +
                                      [C.c_void_p, C.POINTER(C.c_int)])
    return lib


def run(lib, d, buf, org, inner):
    z0, y0, x0, tz, ty, tx = inner
    out = np.full((tz, ty, tx), 0xCD, np.uint8)
    air = C.c_int(-1)
    cfg = oracle.ref_pipeline_cfg(d)
    rc = lib.fy_process_buffer(C.byref(cfg), oracle.p(buf), *org, *buf.shape, z0, y0, x0, tz, ty, tx, *VOL[1:],
                               oracle.p(out), C.byref(air))
    return rc, out, air.value


@pytest.mark.skipif(has_cuda(), reason="a GPU is present: the no-device path is not observable")
def test_reference_pipeline_binds_the_gpu_library(fy):
    """Without a device the relinked pipeline's guided-filter call reaches the GPU library,
    which refuses (FY_ENODEV, recorded for the thread); the reference then skips the stage,
    as pipeline.c:295 does on a nonzero return."""
    lib = linked()
    buf, org, inner = tile_of(scroll_volume(VOL, seed=11))
    d = oracle.pipeline_defaults(do_air_zero=0, guided_eps=8e-4)
    rc, out, _ = run(lib, d, buf, org, inner)
    assert rc == 0
    assert fy.load().fy_gpu_last_status() == fy.FY_ENODEV
    skipped, _ = oracle.ref_process_buffer(oracle.pipeline_defaults(do_air_zero=0), buf, org, inner, VOL[1:])
    assert np.array_equal(out, skipped)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["guided_air_cc_norm", "deconv_guided_air"])
def test_reference_pipeline_on_the_gpu_library(gpu, case):
    lib = linked()
    kw = {"guided_air_cc_norm": dict(guided_eps=8e-4, air_min_component=40, have_norm=1, norm_lo=40, norm_hi=200),
          "deconv_guided_air": dict(do_deconv=1, guided_eps=8e-4, window_lo=-0.02, window_hi=0.3)}[case]
    d = oracle.pipeline_defaults(**kw)
    buf, org, inner = tile_of(scroll_volume(VOL, seed=11))
    launches0 = gpu.load().fy_gpu_kernel_launches()
    rc, got, air = run(lib, d, buf, org, inner)
    assert rc == 0 and air == 0
    assert gpu.load().fy_gpu_kernel_launches() > launches0      # the stages ran on the GPU
    ref, _ = oracle.ref_process_buffer(d, buf, org, inner, VOL[1:])
    diff = np.abs(got.astype(int) - ref.astype(int))
    print(f"LINK {case}: {np.count_nonzero(diff)} of {diff.size} voxels differ, max {diff.max()}")
    # The relinked pipeline's air-cut scratch is the GPU fy_box_smooth (not the reference's
    # CPU-dependent reciprocals), so an air decision can flip where a smoothed value ties a
    # cut; the bar is the fraction of voxels only.
    assert np.count_nonzero(diff) / diff.size <= MISMATCH_FRAC
