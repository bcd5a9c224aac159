"""Failure detection of the box passes' bounded waits, without a GPU fault.

The z-sliding box passes (guided filter and noise statistics) stage their planes with
tensor copies and wait for each on an mbarrier with a bounded number of polls. When a wait
gives up, the CTA raises a flag, waits under the normal bound for every copy it issued, and
returns with its part of the output unfinished; fy_gpu_kernel_timeouts() reports it and the
context stays usable. Here the test hook fy_gpu_test_box_first_wait(0) gives every CTA's
first wait zero polls, so it expires at once; the copies it drains were issued and land.
Then the normal bound is restored and the next calls must be correct again.

Collected after the other GPU tests (the file name sorts late), so its first assertion also
checks that no wait expired while they ran.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def guided_dev(lib, d, out, shape):
    assert lib.fy_gpu_guided(C.c_void_p(d.data_ptr()), C.c_void_p(out.data_ptr()), *shape, 2, 2e-3, 1, None) == 0


def test_first_wait_expiry_is_reported_and_recovers(gpu):
    import torch
    lib = gpu.load()
    shape = (40, 48, 64)                         # nx % 4 == 0 and aligned: the tensor-copy path
    vol = np.random.default_rng(11).uniform(0, 1, shape).astype(np.float32)
    d = torch.from_numpy(vol).cuda()
    out = torch.empty_like(d)
    torch.cuda.synchronize()
    assert lib.fy_gpu_kernel_timeouts() == 0     # nothing expired in the tests before this one
    guided_dev(lib, d, out, shape)
    torch.cuda.synchronize()
    want = out.cpu().numpy()
    scratch = torch.empty(lib.fy_gpu_noise_scratch_bytes(*shape), dtype=torch.uint8, device="cuda")
    nm_want = gpu.NoiseModel()
    assert lib.fy_gpu_estimate_noise(C.c_void_p(d.data_ptr()), *shape, 5, 10.0, 0.5,
                                     C.c_void_p(scratch.data_ptr()), None) == 0
    assert lib.fy_gpu_noise_model(C.c_void_p(scratch.data_ptr()), *shape, C.byref(nm_want), None) == 0
    try:
        assert lib.fy_gpu_test_box_first_wait(0) == 0
        out.fill_(-7.0)
        torch.cuda.synchronize()
        guided_dev(lib, d, out, shape)           # every CTA gives up on its first plane
        torch.cuda.synchronize()
        assert lib.fy_gpu_kernel_timeouts() >= 1
        assert (out.cpu().numpy() == -7.0).any()  # the output was left unfinished
        assert lib.fy_gpu_estimate_noise(C.c_void_p(d.data_ptr()), *shape, 5, 10.0, 0.5,
                                         C.c_void_p(scratch.data_ptr()), None) == 0
        torch.cuda.synchronize()                 # the noise statistics pass also returns early
        assert lib.fy_gpu_kernel_timeouts() >= 2
    finally:
        assert lib.fy_gpu_test_box_first_wait(-1) == 0
    assert lib.fy_gpu_kernel_timeouts() == 0
    # the context is usable and the next calls are correct
    guided_dev(lib, d, out, shape)
    nm = gpu.NoiseModel()
    assert lib.fy_gpu_estimate_noise(C.c_void_p(d.data_ptr()), *shape, 5, 10.0, 0.5,
                                     C.c_void_p(scratch.data_ptr()), None) == 0
    assert lib.fy_gpu_noise_model(C.c_void_p(scratch.data_ptr()), *shape, C.byref(nm), None) == 0
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), want)
    assert nm.noise_ref == nm_want.noise_ref and nm.n_bins_used == nm_want.n_bins_used
    assert lib.fy_gpu_kernel_timeouts() == 0
