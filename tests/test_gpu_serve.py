"""The request loop (fy_server_*): continuous batching of restoration requests.

Requests of different sizes and metadata run concurrently on the worker streams. Each
result must equal the same request run alone through fy_gpu_restore_u8: bit-equal, since
the kernels are deterministic and every worker's workspaces are its own. Admission by the
HBM budget is checked by a budget that admits one large request at a time and by a request
larger than the whole budget, which is refused at submission.
"""
import ctypes as C
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPES = [(48, 64, 56), (64, 64, 64), (40, 48, 40), (96, 80, 72), (33, 70, 41), (128, 96, 112),
          (64, 64, 64), (56, 40, 72), (96, 96, 96), (40, 48, 40), (72, 64, 48), (64, 128, 96)]


def phantom(shape, seed):
    import fysics_b200.phantom as ph
    u = ph.phantom(shape, seed=seed, delta_beta=300.0 + 50 * seed, pixel_um=2.4, rings=0, device="cpu")
    return np.ascontiguousarray(u.numpy() if hasattr(u, "numpy") else u)


def request(fy, u8, out, seed):
    r = fy.Request()
    r.u8 = u8.ctypes.data
    r.out = out.ctypes.data
    r.nz, r.ny, r.nx = u8.shape
    r.f32_min, r.f32_max = 0.0, 1.0 + 0.1 * (seed % 3)
    r.phys = fy.physics(delta_beta=300.0 + 50 * seed, energy_kev=110.0, distance_mm=1200.0, pixel_um=2.4,
                        unsharp_sigma=0.8, unsharp_coeff=0.5, psf_sigma_vox=1.0, psf_sigma_z_vox=1.17)
    fy.load().fy_restore_cfg_default(C.byref(r.cfg))
    r.cfg.deconv_kind = seed % 3
    r.cfg.deconv_param = 0.05 if seed % 3 == 1 else 0.015
    r.cfg.fz2_scale = 1.17 ** 2
    return r


def alone(fy, r):
    import torch
    lib = fy.load()
    n = r.nz * r.ny * r.nx
    u8 = np.ctypeslib.as_array(C.cast(r.u8, C.POINTER(C.c_uint8)), (n,)).copy()
    d_in = torch.from_numpy(u8).cuda()
    d_out = torch.empty(n, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    rc = lib.fy_gpu_restore_u8(C.c_void_p(d_in.data_ptr()), C.c_void_p(d_out.data_ptr()), r.nz, r.ny, r.nx,
                               r.f32_min, r.f32_max, C.byref(r.phys), C.byref(r.cfg), None)
    assert rc == 0, lib.fy_gpu_last_error()
    torch.cuda.synchronize()
    return d_out.cpu().numpy().reshape(r.nz, r.ny, r.nx)


def make_server(fy, budget=16 << 30, workers=4):
    lib = fy.load()
    cfg = fy.ServerCfg()
    lib.fy_server_cfg_default(C.byref(cfg))
    cfg.hbm_budget_bytes, cfg.workers = budget, workers
    h = C.c_void_p()
    assert lib.fy_server_create(C.byref(h), C.byref(cfg)) == 0, lib.fy_gpu_last_error()
    return h


def test_mix_equals_alone(gpu):
    lib = gpu.load()
    ins = [phantom(s, i) for i, s in enumerate(SHAPES)]
    outs = [np.full(s, np.nan, np.float32) for s in SHAPES]
    reqs = [request(gpu, u, o, i) for i, (u, o) in enumerate(zip(ins, outs))]
    srv = make_server(gpu)
    tickets = [None] * len(reqs)

    def submit(idx):                                   # submissions from several host threads
        for i in idx:
            t = C.c_longlong()
            assert lib.fy_server_submit(srv, C.byref(reqs[i]), C.byref(t)) == 0
            tickets[i] = t.value

    th = [threading.Thread(target=submit, args=(range(k, len(reqs), 3),)) for k in range(3)]
    for x in th:
        x.start()
    for x in th:
        x.join()
    for t in tickets:
        res = gpu.RequestResult()
        assert lib.fy_server_wait(srv, t, -1.0, C.byref(res)) == 0, lib.fy_gpu_last_error()
        assert res.status == 0 and res.latency_ms >= res.run_ms >= 0
    st = gpu.ServerStats()
    assert lib.fy_server_get_stats(srv, C.byref(st)) == 0
    assert st.completed == len(reqs) and st.queued == 0 and st.inflight == 0
    assert 0 < st.p50_ms <= st.p99_ms and st.mvox_per_s > 0
    lib.fy_server_destroy(srv)
    for r, o in zip(reqs, outs):
        assert np.array_equal(o, alone(gpu, r))


def test_budget_admits_one_at_a_time_and_refuses_oversize(gpu):
    lib = gpu.load()
    shapes = [(96, 96, 96)] * 3
    ins = [phantom(s, 7 + i) for i, s in enumerate(shapes)]
    outs = [np.zeros(s, np.float32) for s in shapes]
    reqs = [request(gpu, u, o, 7 + i) for i, (u, o) in enumerate(zip(ins, outs))]
    n = 96 ** 3
    srv = make_server(gpu, budget=48 * n, workers=3)  # one 96^3 request's footprint (~40 B/voxel), not two
    ts = []
    for r in reqs:
        t = C.c_longlong()
        assert lib.fy_server_submit(srv, C.byref(r), C.byref(t)) == 0
        ts.append(t.value)
    for t in ts:
        assert lib.fy_server_wait(srv, t, -1.0, None) == 0
    big = np.zeros((256, 256, 256), np.uint8)
    bo = np.zeros(big.shape, np.float32)
    t = C.c_longlong(-1)
    assert lib.fy_server_submit(srv, C.byref(request(gpu, big, bo, 0)), C.byref(t)) == 5   # FY_EUNSUPPORTED
    assert b"HBM budget" in lib.fy_gpu_last_error()
    assert lib.fy_server_wait(srv, 987654, 0.0, None) == 1                                 # unknown ticket
    lib.fy_server_destroy(srv)
    for r, o in zip(reqs, outs):
        assert np.array_equal(o, alone(gpu, r))


def test_device_resident_requests_equal_alone(gpu):
    """Requests whose input and output are device memory run the chain in place (no link
    copies); results equal the single-cube call, several requests at once."""
    import torch
    lib = gpu.load()
    shapes = SHAPES[:6]
    ins = [torch.from_numpy(phantom(s, 20 + i)).cuda() for i, s in enumerate(shapes)]
    outs = [torch.full(s, float("nan"), dtype=torch.float32, device="cuda") for s in shapes]
    reqs = []
    for i, (u, o) in enumerate(zip(ins, outs)):
        r = request(gpu, np.zeros(shapes[i], np.uint8), np.zeros(1, np.float32), 20 + i)
        r.u8, r.out = u.data_ptr(), o.data_ptr()
        reqs.append(r)
    torch.cuda.synchronize()
    srv = make_server(gpu)
    ts = []
    for r in reqs:
        t = C.c_longlong()
        assert lib.fy_server_submit(srv, C.byref(r), C.byref(t)) == 0
        ts.append(t.value)
    for t in ts:
        res = gpu.RequestResult()
        assert lib.fy_server_wait(srv, t, -1.0, C.byref(res)) == 0, lib.fy_gpu_last_error()
        assert res.status == 0 and res.h2d_ms == 0 and res.d2h_ms == 0
    lib.fy_server_destroy(srv)
    for i, r in enumerate(reqs):
        host = ins[i].cpu().numpy()
        r.u8 = host.ctypes.data
        assert np.array_equal(outs[i].cpu().numpy(), alone(gpu, r))
