#!/usr/bin/env python
"""Benchmark of the fysics restoration path on B200 (one JSON line on stdout, rank 0).

Workload: the production-size drop-in configuration -- one 512^3 u8 cube of the seeded
scroll phantom (pixel 2.4 um, delta_beta x fy_auto_deltabeta_scale, anisotropic PSF
sigma_z/sigma_xy = 1.17, 40 synthetic rings), restored by the full chain
  fy_u8_to_phys -> fy_deconvolve_matched (psf 1.0 / 1.17) -> fy_estimate_noise (win 5,
  10th pct, ref 0.4) -> guided filter (r 2, eps = (3*noise_ref)^2) -> ring subtraction
  (accumulate ss=2 on the u8 input, vote(15, 100, 0.5, 6.0), apply),
through fy_gpu_restore_u8. A step is one cube.

  value   Mvox/s with the cube resident in HBM (device-timed with CUDA events, max over ranks)
  e2e     Mvox/s through host buffers: pinned u8 in -> H2D -> chain -> D2H -> pinned f32 out
  --impl reference  the reference's CPU implementation (oracle/_ref, compiled from its own
          sources) on the host cores, same metric, bounded sample

Multi-GPU (torchrun): cubes are independent -- each rank restores its own cube (weak
scaling, no collective on the data path); the barrier and the max of the per-rank times
use torch.distributed.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
# Hardware work queues per context (CUDA default 8). The request loop runs a stream pair per
# worker; with fewer queues than busy streams, unrelated streams share a queue and a small
# request's kernels wait behind a large one's. Must be set before CUDA is initialised.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

METRIC = "Mvoxel/s deconv+denoise and p50/p99 cube latency, served vs plain, same B200"
SHAPE = (512, 512, 512)
WORKLOAD = "512^3 u8 scroll phantom, dewindow->deconv_matched(aniso 1.17)->noise->guided(r2)->dering"


def physics_for(fb):
    import fysics_b200.phantom as ph
    p = fb.physics(delta_beta=500.0, energy_kev=110.0, distance_mm=1200.0, pixel_um=2.4, unsharp_sigma=0.8,
                   unsharp_coeff=0.5, psf_sigma_vox=1.0, psf_sigma_z_vox=1.17)
    scale = fb.load().fy_auto_deltabeta_scale(C.byref(p))
    p.delta_beta *= scale
    del ph
    return p, scale


def restore_cfg(fb, dering_handle):
    cfg = fb.RestoreCfg()
    fb.load().fy_restore_cfg_default(C.byref(cfg))
    cfg.deconv_kind = 1
    cfg.deconv_param = 0.05
    cfg.noise_win = 5
    cfg.noise_flat_pct = 10.0
    cfg.noise_ref_intensity = 0.4
    cfg.guided_radius = 2
    cfg.guided_s = 1
    cfg.dering = dering_handle
    cfg.dering_accumulate = 1
    cfg.dering_ss = 2
    cfg.dering_hp_win = 15
    cfg.dering_min_cnt = 100
    cfg.dering_min_amp = 0.5
    cfg.dering_max_amp = 6.0
    cfg.dering_scale = 1.0 / 255.0
    return cfg


# ------------------------------------------------------------------------------ clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "25"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            t0 = time.perf_counter()              # the timed region starts once samples flow
            while not self.lines and time.perf_counter() - t0 < 3.0 and self.proc.poll() is None:
                time.sleep(0.005)
            self.lines.clear()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------------------ roofline
def algorithmic_bytes(name: str, n: int, geo: dict) -> float | None:
    """Bytes a kernel must move per launch (read once + written once), 512^3 u8 chain."""
    nz, ny, nx = geo["shape"]
    px = geo["px"]
    hx = px // 2 + 1
    half = nz * ny * hx * 8            # one stored half-spectrum (nz planes)
    table = {
        "deconv.x_fwd": n * 1 + half,
        "deconv.y_fwd": half + nz * geo["py"] * hx * 8,
        "deconv.z_weight": 2 * nz * geo["py"] * hx * 8,
        "deconv.y_inv": nz * geo["py"] * hx * 8 + half,
        "deconv.x_inv": half + n * 4,
        # box pass: I read, mean + var written (+ the guided (mean, var) pairs when the noise
        # window is the guided window: the chain then skips the guided a/b pass)
        "noise.stats": n * (20 if geo.get("shared_window") else 12),
        "noise.lohi": n * 4,                   # one window pass over mean (candidates ~1%: small)
        "noise.bin_select": n * 8,             # one pass over mean + var (the bins' window; candidates ~5%)
        # (mean, var) pairs + I -> out (16 B); without the shared window I -> a, b (12 B) first
        "guided": n * (16 if geo.get("shared_window") else 28),
        "dering.accumulate+vote": n * 1,
        "dering.apply": n * 8,
    }
    return table.get(name)


# marks recorded inside the timed loop: "noise" closes the span before the guided output pass,
# "guided" closes the pass itself (the dominant kernel of the chain)
TIMED_MARKS = "noise,guided"

# DRAM bytes per voxel of each instrumented span: dram__bytes_read.sum + dram__bytes_write.sum
# of its kernel's launch in an ncu capture of this chain on a 384^3 cube (one kernel per
# capture, on the smaller cube; every span's traffic grows with the voxel count), divided by
# its voxels. The two selection spans give their counting pass only: their other launches
# run over candidate lists of a few percent of the voxels.
DRAM_BYTES_PER_VOXEL = {
    "deconv.x_fwd": 4.087, "deconv.y_fwd": 7.599, "deconv.z_weight": 8.198, "deconv.y_inv": 7.602,
    "deconv.x_inv": 7.539, "noise.stats": 19.142, "noise.lohi": 4.108, "noise.bin_select": 8.227,
    "guided": 15.954,
}


def read_profile(lib):
    cnt = lib.fy_gpu_profile_stop()
    per = {}
    for i in range(1, cnt):
        nm = C.c_char_p()
        ms = C.c_float()
        if lib.fy_gpu_profile_read(i, C.byref(nm), C.byref(ms)) == 0:
            per.setdefault(nm.value.decode(), []).append(ms.value)
    return per


# ------------------------------------------------------------------------------ CPU legs
def chain_spec(db_scale: float):
    """The benchmark chain's settings for the CPU chain runner (oracle.chain): the same
    physics, deconvolution, noise, guided and ring settings as restore_cfg()."""
    from oracle.chain import ChainSpec
    phys = dict(delta_beta=500.0 * db_scale, energy_kev=110.0, distance_mm=1200.0, pixel_um=2.4, unsharp_sigma=0.8,
                unsharp_coeff=0.5, psf_sigma_vox=1.0, psf_sigma_z_vox=1.17)
    return ChainSpec(phys=phys, matched=True, deconv_param=0.05, noise_win=5, noise_pct=10.0, noise_ref=0.4,
                     guided_r=2, dering=dict(ss=2, hp_win=15, min_cnt=100, min_amp=0.5, max_amp=6.0, slab_z=512,
                                             ns=8))


def host_memory_bytes() -> int | None:
    """Memory this process may still use on the host: MemAvailable, capped by a cgroup limit."""
    avail = None
    try:
        for ln in open("/proc/meminfo"):
            if ln.startswith("MemAvailable:"):
                avail = int(ln.split()[1]) * 1024
    except OSError:
        pass
    try:
        lim = open("/sys/fs/cgroup/memory.max").read().strip()
        if lim != "max":
            used = int(open("/sys/fs/cgroup/memory.current").read().strip())
            room = int(lim) - used
            avail = room if avail is None else min(avail, room)
    except (OSError, ValueError):
        pass
    return avail


# Peak host memory of one reference chain per voxel: the noise model's three double fields,
# its float squares, the sorted copy of the means and qsort's merge buffer (44 B), plus the
# chain's float volumes (dewindowed, deconvolved, output) alive meanwhile; rounded up.
REF_CHAIN_BYTES_PER_VOXEL = 64


def cpu_reference_chain(u8_host: np.ndarray, spec, threads: int | None = None, warmup: int = 3,
                        keep_output: bool = True) -> dict:
    """The reference's chain (oracle/_ref, compiled from its own sources) on the WHOLE
    benchmark cube: one chain per host thread, each thread restoring its own copy of the
    same cube -- the reference's own parallelism, one tile or cube chain per worker
    (pipeline.c:1008-1020); its entry points are single-threaded per call. The thread count
    is the host's cores, or fewer where host memory holds fewer chains at once. Warm-up: the
    same chain on a 128^3 corner crop, `warmup` times per thread. Returns Mvox/s over the
    timed cubes, their count (the steps) and one thread's output for the error check."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle.chain import ref_restore
    n = u8_host.size
    cores = os.cpu_count() or 1
    mem = host_memory_bytes()
    by_mem = max(1, int(0.8 * mem) // (REF_CHAIN_BYTES_PER_VOXEL * n)) if mem else 1
    nthr = threads or max(1, min(cores, by_mem))
    crop = np.ascontiguousarray(u8_host[:128, :128, :128])
    with ThreadPoolExecutor(max_workers=nthr) as ex:
        for _ in range(warmup):
            list(ex.map(lambda i: ref_restore(crop, spec, keep_stages=False), range(nthr)))
    kept = {}
    per = [0.0] * nthr

    def one(i):
        t0 = time.perf_counter()
        r = ref_restore(u8_host, spec, keep_stages=False)
        per[i] = time.perf_counter() - t0
        if i == 0 and keep_output:
            kept.update(out=r["out"], noise_ref=r["noise"].noise_ref, detected=r["detected"])
        return r["detected"]

    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=nthr) as ex:
        detected = list(ex.map(one, range(nthr)))
    wall = time.perf_counter() - t0
    shape = "x".join(map(str, u8_host.shape))
    res = {"value": nthr * n / wall / 1e6, "unit": "Mvoxel/s", "cores": nthr, "kind": "reference",
           "cubes": nthr, "wall_s": wall, "ms_per_cube_single_thread": 1e3 * min(per),
           "sample": f"{nthr} full {shape} chains of the benchmark cube, one per host thread ({cores} cores, "
                     f"{nthr} threads, host memory {mem / 2**30:.0f} GiB free)" if mem else
                     f"{nthr} full {shape} chains of the benchmark cube, one per host thread ({cores} cores)",
           "warmup": f"{warmup} chains on a 128^3 corner crop per thread",
           "detected_rings": detected[0]}
    if keep_output:
        res["_out"] = kept
    return res


def cpu_reference_crops(u8_host: np.ndarray, spec, crop: int = 128, budget_s: float = 10.0) -> dict:
    """Secondary figure: the reference chain on 128^3 crops of the cube, one crop per host
    thread. Each crop votes its own rings about its own centre and runs crop-sized FFTs and
    sorts, so this is not the benchmark's configuration."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle.chain import ref_restore
    cores = os.cpu_count() or 1
    crops = [(z, y, x) for z in range(u8_host.shape[0] // crop) for y in range(u8_host.shape[1] // crop)
             for x in range(u8_host.shape[2] // crop)]

    def one(i):
        z, y, x = crops[i % len(crops)]
        sub = np.ascontiguousarray(u8_host[z * crop:(z + 1) * crop, y * crop:(y + 1) * crop, x * crop:(x + 1) * crop])
        ref_restore(sub, spec, keep_stages=False)
        return sub.size

    t0 = time.perf_counter()
    one(0)
    t_one = time.perf_counter() - t0
    jobs = cores * max(1, min(int(budget_s / max(t_one, 1e-3)), 4))
    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=cores) as ex:
        vox = sum(ex.map(one, range(jobs)))
    dt = time.perf_counter() - t0
    return {"value": vox / dt / 1e6, "unit": "Mvoxel/s", "cores": cores,
            "sample": f"{jobs} crops of {crop}^3, one per host thread; not the benchmark configuration (each crop "
                      f"votes its own rings, crop-sized FFTs and sorts); single-thread {t_one * 1e3:.0f} ms per crop"}


# ------------------------------------------------------------------------------ serving
def _req(fb, u8_pinned, out_pinned, db, span, scale):
    r = fb.Request()
    r.u8 = u8_pinned.data_ptr()
    r.out = out_pinned.data_ptr()
    r.nz, r.ny, r.nx = u8_pinned.shape
    r.f32_min, r.f32_max = 0.0, span
    r.phys = fb.physics(delta_beta=db * scale, energy_kev=110.0, distance_mm=1200.0, pixel_um=2.4,
                        unsharp_sigma=0.8, unsharp_coeff=0.5, psf_sigma_vox=1.0, psf_sigma_z_vox=1.17)
    fb.load().fy_restore_cfg_default(C.byref(r.cfg))
    r.cfg.deconv_kind = 1
    r.cfg.deconv_param = 0.05
    r.cfg.noise_win, r.cfg.noise_flat_pct, r.cfg.noise_ref_intensity = 5, 10.0, 0.4
    r.cfg.guided_radius, r.cfg.guided_s = 2, 1
    return r


def _plain(fb, lib, reqs, dev):
    """The same requests one at a time through the plain per-cube path: pinned H2D, the
    chain (fy_gpu_restore_u8), D2H, synchronise; returns Mvox/s over the wall time."""
    import torch
    vox = 0
    d_in = {}
    d_out = {}
    t0 = time.perf_counter()
    for r in reqs:
        shp = (r.nz, r.ny, r.nx)
        if shp not in d_in:
            d_in[shp] = torch.empty(shp, dtype=torch.uint8, device=f"cuda:{dev}")
            d_out[shp] = torch.empty(shp, dtype=torch.float32, device=f"cuda:{dev}")
        n = r.nz * r.ny * r.nx
        src = torch.frombuffer((C.c_uint8 * n).from_address(r.u8), dtype=torch.uint8).view(shp)
        d_in[shp].copy_(src, non_blocking=True)
        fb.check(lib.fy_gpu_restore_u8(C.c_void_p(d_in[shp].data_ptr()), C.c_void_p(d_out[shp].data_ptr()),
                                       r.nz, r.ny, r.nx, r.f32_min, r.f32_max, C.byref(r.phys), C.byref(r.cfg),
                                       C.c_void_p(torch.cuda.current_stream().cuda_stream)), "fy_gpu_restore_u8")
        dst = torch.frombuffer((C.c_float * n).from_address(r.out), dtype=torch.float32).view(shp)
        dst.copy_(d_out[shp], non_blocking=True)
        torch.cuda.synchronize()
        vox += n
    return vox / (time.perf_counter() - t0) / 1e6


def served_and_batched(fb, lib, dev, seed, db_scale, n_requests=400, rates=(500.0, 2000.0), n_batch=96):
    """Config-5 sample (Poisson arrivals, 64:128:256:512 = 40:30:25:5) through the request
    loop, and a config-3 sample (uneven cubes, dims per axis from {96..320}) submitted at
    once; each next to the same requests on the plain per-cube path."""
    import torch
    import fysics_b200.phantom as ph
    rng = np.random.default_rng(seed)
    scfg = fb.ServerCfg()
    lib.fy_server_cfg_default(C.byref(scfg))
    scfg.reserve_nz = scfg.reserve_ny = scfg.reserve_nx = 512      # resident workspaces: largest cube
    srv = C.c_void_p()
    fb.check(lib.fy_server_create(C.byref(srv), C.byref(scfg)), "fy_server_create")

    def pinned_phantom(shape, s):
        u = ph.phantom(shape, seed=s, delta_beta=500.0 * db_scale, pixel_um=2.4, fz2_scale=1.17 ** 2,
                       device=f"cuda:{dev}")
        h = torch.empty(shape, dtype=torch.uint8, pin_memory=True)
        h.copy_(u.cpu())
        return h

    def run_all(reqs, arrivals=None):
        lat = [0.0] * len(reqs)
        phases = [None] * len(reqs)
        tickets = [None] * len(reqs)
        done = threading.Event()

        def waiter():
            for i in range(len(reqs)):
                while tickets[i] is None:
                    time.sleep(1e-4)
                res = fb.RequestResult()
                fb.check(lib.fy_server_wait(srv, tickets[i], -1.0, C.byref(res)), "fy_server_wait")
                lat[i] = res.latency_ms
                phases[i] = (res.queue_ms, res.h2d_ms, res.chain_ms, res.d2h_ms)
            done.set()

        lib.fy_server_reset_stats(srv)
        th = threading.Thread(target=waiter)
        th.start()
        t0 = time.perf_counter()
        for i, r in enumerate(reqs):
            if arrivals is not None:
                dt = arrivals[i] - (time.perf_counter() - t0)
                if dt > 0:
                    time.sleep(dt)
            t = C.c_longlong()
            fb.check(lib.fy_server_submit(srv, C.byref(r), C.byref(t)), "fy_server_submit")
            tickets[i] = t.value
        th.join()
        wall = time.perf_counter() - t0
        st = fb.ServerStats()
        lib.fy_server_get_stats(srv, C.byref(st))
        return lat, wall, st, phases

    # ---- config-5 sample at a latency point and a saturating throughput point
    sizes = [64, 128, 256, 512]
    src = {s: pinned_phantom((s,) * 3, seed + s) for s in sizes}
    outs = {s: [torch.empty((s,) * 3, dtype=torch.float32, pin_memory=True) for _ in range(6)] for s in sizes}
    pick = rng.choice(len(sizes), n_requests, p=[0.40, 0.30, 0.25, 0.05])
    reqs = []
    for i, k in enumerate(pick):
        s = sizes[k]
        reqs.append(_req(fb, src[s], outs[s][i % 6], rng.uniform(200, 1000), float(rng.uniform(0.9, 1.1)), db_scale))
    run_all([_req(fb, src[s], outs[s][0], 500.0, 1.0, db_scale) for s in sizes] * scfg.workers)   # warm-up
    vox = sum(r.nz * r.ny * r.nx for r in reqs)
    points = []
    for rate in rates:
        arrivals = np.cumsum(rng.exponential(1.0 / rate, n_requests))
        lat, wall, st, phases = run_all(reqs, arrivals)
        by, ph_by = {}, {}
        for r, l, f in zip(reqs, lat, phases):
            by.setdefault(r.nz, []).append(l)
            ph_by.setdefault(r.nz, []).append(f)
        points.append({
            "arrival_rps": rate, "offered_mvox_per_s": vox / arrivals[-1] / 1e6, "mvox_per_s": vox / wall / 1e6,
            "p50_ms": st.p50_ms, "p99_ms": st.p99_ms,
            "p50_ms_by_size": {f"{k}^3": float(np.percentile(v, 50)) for k, v in sorted(by.items())},
            "p99_ms_by_size": {f"{k}^3": float(np.percentile(v, 99)) for k, v in sorted(by.items())},
            # per-size p50/p99 of each phase: queue wait, H2D, chain (incl. waiting for the GPU), D2H
            "phases_ms_by_size": {f"{k}^3": {name: [round(float(np.percentile(col, q)), 3) for q in (50, 99)]
                                             for name, col in zip(("queue", "h2d", "chain", "d2h"), zip(*v))}
                                  for k, v in sorted(ph_by.items())}})
    plain = _plain(fb, lib, reqs[: min(len(reqs), 120)], dev)
    served = {
        "workload": f"{n_requests} requests per point, Poisson arrivals, sizes 64^3:128^3:256^3:512^3 = "
                    "40:30:25:5, per-request delta_beta U[200,1000] and window span U[0.9,1.1]; host pinned "
                    "buffers, H2D + chain + D2H per request",
        "workers": scfg.workers, "small_workers": scfg.small_workers, "resident_workspaces": "512^3",
        "hbm_budget_gb": scfg.hbm_budget_bytes / 2 ** 30,
        "cuda_device_max_connections": int(os.environ.get("CUDA_DEVICE_MAX_CONNECTIONS", "8")),
        "points": points,
        "mvox_per_s": max(pt["mvox_per_s"] for pt in points),
        "plain_mvox_per_s": plain,
        "plain": "the first 120 requests one at a time: pinned H2D, fy_gpu_restore_u8, D2H, synchronise",
    }
    if n_batch <= 0:
        lib.fy_server_destroy(srv)
        return served, None
    # ---- config-3: uneven cubes submitted at once, device-resident and through host buffers
    dims = [96, 128, 160, 200, 240, 256, 320]
    bre, dre = [], []
    keep = []
    for i in range(n_batch):
        shape = tuple(int(d) for d in rng.choice(dims, 3))
        u = ph.phantom(shape, seed=seed + 1000 + i, delta_beta=500.0 * db_scale, pixel_um=2.4, fz2_scale=1.17 ** 2,
                       device=f"cuda:{dev}")
        h = torch.empty(shape, dtype=torch.uint8, pin_memory=True)
        h.copy_(u.cpu())
        o = torch.empty(shape, dtype=torch.float32, pin_memory=True)
        do = torch.empty(shape, dtype=torch.float32, device=f"cuda:{dev}")
        keep += [h, o, u, do]
        db = rng.uniform(200, 1000)
        bre.append(_req(fb, h, o, db, 1.0, db_scale))
        r = _req(fb, h, o, db, 1.0, db_scale)
        r.u8, r.out = u.data_ptr(), do.data_ptr()
        dre.append(r)
    bvox = sum(r.nz * r.ny * r.nx for r in bre)
    torch.cuda.synchronize()
    run_all(dre[:8])                                                                       # warm-up
    _, dwall, _, _ = run_all(dre)
    # the plain per-cube path on device buffers: one fy_gpu_restore_u8 after another, one stream
    st = torch.cuda.Stream(device=dev)
    spp = C.c_void_p(st.cuda_stream)

    def plain_device():
        for r in dre:
            fb.check(lib.fy_gpu_restore_u8(C.c_void_p(r.u8), C.c_void_p(r.out), r.nz, r.ny, r.nx, r.f32_min,
                                           r.f32_max, C.byref(r.phys), C.byref(r.cfg), spp), "fy_gpu_restore_u8")
        st.synchronize()

    plain_device()
    t0 = time.perf_counter()
    plain_device()
    pdev = bvox / (time.perf_counter() - t0) / 1e6
    # the same device-resident cubes through the batch entry point: one call for all of them
    items = (fb.BatchCube * n_batch)()
    for i, r in enumerate(dre):
        q = items[i]
        q.u8, q.out, q.nz, q.ny, q.nx = r.u8, r.out, r.nz, r.ny, r.nx
        q.f32_min, q.f32_max, q.phys = r.f32_min, r.f32_max, r.phys

    def batch_call():
        fb.check(lib.fy_gpu_restore_u8_batch(items, n_batch, C.byref(dre[0].cfg), spp), "fy_gpu_restore_u8_batch")

    batch_call()                                                                           # warm-up
    st.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    bms = []
    for _ in range(3):
        ev0.record(st)
        batch_call()
        ev1.record(st)
        ev1.synchronize()
        bms.append(ev0.elapsed_time(ev1))
    bapi = bvox / (statistics.median(bms) * 1e-3) / 1e6
    run_all(bre[:4])                                                                       # warm-up
    _, bwall, _, _ = run_all(bre)
    batched = {
        "workload": f"{n_batch} cubes, dims per axis from {dims} ({bvox / 1e6:.0f} Mvoxel), per-cube delta_beta "
                    "U[200,1000]",
        "batch_api": {"mvox_per_s": bapi, "ms": statistics.median(bms),
                      "api": "fy_gpu_restore_u8_batch, one call over the device-resident cubes (deconvolutions on "
                             "8 streams, the two box passes as work-queue launches over all cubes' tiles, the "
                             "noise selection as one launch per step for all cubes); CUDA events on its stream, "
                             "median of 3 calls"},
        "resident": {"mvox_per_s": bvox / dwall / 1e6, "plain_mvox_per_s": pdev,
                     "api": "request loop on device-resident cubes submitted at once (no link copies) vs the "
                            "plain per-cube fy_gpu_restore_u8 one after another on one stream"},
        "host": {"mvox_per_s": bvox / bwall / 1e6, "plain_mvox_per_s": _plain(fb, lib, bre, dev),
                 "api": "host pinned buffers: request loop vs plain per-cube H2D + chain + D2H"},
        "mvox_per_s": max(bapi, bvox / dwall / 1e6),
        "plain_mvox_per_s": pdev,
    }
    lib.fy_server_destroy(srv)
    return served, batched


# ------------------------------------------------------------------------------ registration
class WorkerPool:
    """`n` persistent host threads. run(fn, items) hands out 0..items-1 through a shared
    counter and returns the wall time; run_each(fn) runs fn once on every thread (the
    warm-up, so that each thread's library workspaces exist before anything is timed).
    fn(worker, item) returns 0 or an error code. close() releases every thread's library
    workspaces (fy_gpu_release) and joins the threads."""

    def __init__(self, n, lib):
        self.n, self.lib = n, lib
        self.go, self.done = threading.Barrier(n + 1), threading.Barrier(n + 1)
        self.lock = threading.Lock()
        self.fn, self.items, self.next, self.each, self.errs = None, 0, 0, False, []
        self.threads = [threading.Thread(target=self._loop, args=(w,), daemon=True) for w in range(n)]
        for t in self.threads:
            t.start()

    def _loop(self, w):
        while True:
            self.go.wait()
            if self.fn is None:
                self.lib.fy_gpu_release()
                self.done.wait()
                return
            if self.each:
                rc = self.fn(w, w)
                if rc:
                    self.errs.append(rc)
            else:
                while True:
                    with self.lock:
                        k = self.next
                        self.next += 1
                    if k >= self.items:
                        break
                    rc = self.fn(w, k)
                    if rc:
                        self.errs.append(rc)
            self.done.wait()

    def _start(self, fn, items, each):
        self.fn, self.items, self.next, self.each, self.errs = fn, items, 0, each, []
        t0 = time.perf_counter()
        self.go.wait()
        self.done.wait()
        dt = time.perf_counter() - t0
        if self.errs:
            raise RuntimeError(f"worker call failed: {self.errs[:3]} {self.lib.fy_gpu_last_error()}")
        return dt

    def run(self, fn, items):
        return self._start(fn, items, False)

    def run_each(self, fn):
        return self._start(fn, self.n, True)

    def close(self):
        self.fn = None
        self.go.wait()
        self.done.wait()
        for t in self.threads:
            t.join()


def tiles_sample(fb, lib, dev, seed, threads=8, passes=3, cpu_budget_s=10.0):
    """The export tool's per-tile chain (fy_process_buffer, pipeline.c:467-510) as its worker
    pool calls it (mca_export.c:634-660): 16 inner tiles of 128^3 with an 8-voxel halo
    (144^3 u8 buffers) from a synthetic 144 x 528 x 528 scroll band, with the export
    settings: no deconvolution, guided eps 8e-4 on 2x-subsampled coefficients, air cut,
    despeckle of islands under 64 voxels, recenter [40, 200], dithered u8.
      e2e       `threads` host threads take tiles from a shared queue and call
                fy_process_buffer on pageable host buffers (copies inside the timing);
      resident  the same threads call fy_gpu_process_buffer on device-resident buffers,
                one CUDA stream each;
      reference the reference's fy_process_buffer, one tile per host thread (bounded)."""
    import torch
    import fysics_b200.phantom as ph
    vol = ph.scroll_volume((144, 528, 528), seed=seed)
    halo, T = 8, 128
    tiles = []
    for ty in range(4):
        for tx in range(4):
            z0, y0, x0 = halo, halo + T * ty, halo + T * tx
            org = (z0 - halo, y0 - halo, x0 - halo)
            buf = np.ascontiguousarray(vol[org[0]:z0 + T + halo, org[1]:y0 + T + halo, org[2]:x0 + T + halo])
            tiles.append((buf, org, (z0, y0, x0, T, T, T)))
    vyx = vol.shape[1:]
    cfgd = dict(delta_beta=1000.0, energy_kev=78.0, distance_mm=220.0, pixel_um=2.4, unsharp_sigma=1.2,
                unsharp_coeff=4.0, use_matched_deconv=1, psf_sigma_vox=1.0, deconv_tikhonov=0.05, guided_eps=8e-4,
                do_air_zero=1, air_cut_u8=-1, air_cut_band=8, air_thresh=0.05, air_cut_aggr=0.5,
                air_min_component=64, scratch_passes=5, have_norm=1, norm_lo=40, norm_hi=200, halo=halo,
                dering_cy=-1.0, dering_cx=-1.0)
    cfg = fb.PipelineCfg()
    for k, v in cfgd.items():
        setattr(cfg, k, v)
    inner_vox = T ** 3

    outs = [np.empty((T, T, T), np.uint8) for _ in range(len(tiles))]

    def host_work(wid, k):
        buf, org, inner = tiles[k % len(tiles)]
        air = C.c_int()
        return lib.fy_process_buffer(C.byref(cfg), buf.ctypes.data, *org, *buf.shape, *inner, *vyx,
                                     outs[k % len(tiles)].ctypes.data, C.byref(air))

    d_bufs = [torch.from_numpy(t[0]).to(f"cuda:{dev}") for t in tiles]
    d_outs = [torch.empty((T, T, T), dtype=torch.uint8, device=f"cuda:{dev}") for _ in range(threads)]
    streams = [torch.cuda.Stream(device=dev) for _ in range(threads)]
    torch.cuda.synchronize()

    def dev_work(wid, k):
        buf, org, inner = tiles[k % len(tiles)]
        k = k % len(tiles)
        air = C.c_int()
        return lib.fy_gpu_process_buffer(C.byref(cfg), C.c_void_p(d_bufs[k].data_ptr()), *org, *buf.shape, *inner,
                                         *vyx, C.c_void_p(d_outs[wid].data_ptr()), C.byref(air),
                                         C.c_void_p(streams[wid].cuda_stream))

    # the same band as a local zarr v2 tree of 128^3 chunks (the export's chunking), read through
    # fy_process_chunk: chunk files -> pinned -> device chunk cache -> GPU assembly -> tile chain
    import shutil
    import tempfile
    zdir = tempfile.mkdtemp(prefix="fy_band_")
    zroot = Path(zdir) / "band.zarr"
    (zroot / "0").mkdir(parents=True)
    (zroot / "0" / ".zarray").write_text(
        '{"chunks":[128,128,128],"compressor":null,"dtype":"|u1","fill_value":0,"order":"C",'
        f'"shape":[{vol.shape[0]},{vol.shape[1]},{vol.shape[2]}],"zarr_format":2,"dimension_separator":"/"}}')
    for cz in range(-(-vol.shape[0] // 128)):
        for cy in range(-(-vol.shape[1] // 128)):
            for cx in range(-(-vol.shape[2] // 128)):
                d = zroot / "0" / str(cz) / str(cy)
                d.mkdir(parents=True, exist_ok=True)
                (d / str(cx)).write_bytes(np.ascontiguousarray(
                    vol[cz * 128:(cz + 1) * 128, cy * 128:(cy + 1) * 128, cx * 128:(cx + 1) * 128]).tobytes())
    zin = fb.Zarr()
    fb.check(lib.fy_zarr_open(C.byref(zin), str(zroot).encode()), "fy_zarr_open")
    zouts = [np.empty((T, T, T), np.uint8) for _ in range(len(tiles))]

    def zarr_work(wid, k):
        k = k % len(tiles)
        z0, y0, x0 = tiles[k][2][:3]
        dims = [C.c_int() for _ in range(3)]
        air = C.c_int()
        return lib.fy_process_chunk(C.byref(zin), C.byref(cfg), z0, y0, x0, T, zouts[k].ctypes.data,
                                    *[C.byref(v) for v in dims], C.byref(air))

    def cache_stats():
        v = [C.c_ulonglong() for _ in range(3)]
        lib.fy_gpu_zarr_cache_stats(*[C.byref(x) for x in v])
        return [x.value for x in v]

    n_items = passes * len(tiles)
    pool = WorkerPool(threads, lib)
    try:
        pool.run_each(host_work)                       # warm-up: every thread's workspaces
        pool.run(host_work, len(tiles))
        t_host = pool.run(host_work, n_items)
        pool.run_each(dev_work)
        pool.run(dev_work, len(tiles))
        t_dev = pool.run(dev_work, n_items)
        s0 = cache_stats()
        t_zcold = pool.run(zarr_work, len(tiles))      # first pass: every chunk file read once
        s1 = cache_stats()
        pool.run_each(zarr_work)
        t_zarr = pool.run(zarr_work, n_items)
        s2 = cache_stats()
    finally:
        pool.close()
        shutil.rmtree(zdir, ignore_errors=True)
    res = {"workload": "16 tiles of 128^3 (8-voxel halo, 144^3 u8 buffers) from a synthetic 144x528x528 scroll "
                       "band; export settings: no deconvolution, guided eps 8e-4 subsample 2, air cut, despeckle "
                       "< 64 voxels, recenter [40, 200], dithered u8",
           "threads": threads, "tiles_timed": n_items,
           "e2e": {"tiles_per_s": n_items / t_host, "mvox_per_s": n_items * inner_vox / t_host / 1e6,
                   "ms_per_tile": t_host * 1e3 / n_items, "api": "fy_process_buffer, pageable host buffers"},
           "resident": {"tiles_per_s": n_items / t_dev, "mvox_per_s": n_items * inner_vox / t_dev / 1e6,
                        "ms_per_tile": t_dev * 1e3 / n_items, "api": "fy_gpu_process_buffer, one stream per thread"},
           "zarr": {"tiles_per_s": n_items / t_zarr, "mvox_per_s": n_items * inner_vox / t_zarr / 1e6,
                    "ms_per_tile": t_zarr * 1e3 / n_items, "first_pass_ms_per_tile": t_zcold * 1e3 / len(tiles),
                    "chunk_files_read_first_pass": s1[1] - s0[1], "bytes_read_first_pass": s1[2] - s0[2],
                    "chunk_cache_hits_timed": s2[0] - s1[0], "chunk_files_read_timed": s2[1] - s1[1],
                    "haloed_bytes_assembled_per_tile": int(np.prod(tiles[0][0].shape)),
                    "outputs_equal_fy_process_buffer": all(np.array_equal(zouts[k], outs[k]) for k in range(len(tiles))),
                    "api": "fy_process_chunk on a local zarr v2 tree of 128^3 chunk files (same band): chunk files "
                           "read whole into pinned memory, kept in the device chunk cache, haloed tile assembled on "
                           "the GPU, then the tile chain; the first pass reads every chunk file once"}}
    try:
        import oracle
        from concurrent.futures import ThreadPoolExecutor
        if oracle.have_ref() and cpu_budget_s > 0:
            L = oracle.ref()
            rcfg = oracle.ref_pipeline_cfg(oracle.pipeline_defaults(**cfgd))
            ref_out = [np.empty((T, T, T), np.uint8) for _ in range(len(tiles))]

            def one(k):
                buf, org, inner = tiles[k % len(tiles)]
                air = C.c_int()
                L.fy_process_buffer(C.byref(rcfg), oracle.p(buf), *org, *buf.shape, *inner, *vyx,
                                    oracle.p(ref_out[k % len(tiles)]), C.byref(air))
                return 1

            t1 = time.perf_counter()
            one(0)
            t_one = time.perf_counter() - t1
            cores = os.cpu_count() or 1
            jobs = max(1, min(len(tiles), int(cpu_budget_s / max(t_one, 1e-3)) * cores // 2, cores))
            t1 = time.perf_counter()
            with ThreadPoolExecutor(max_workers=cores) as ex:
                done = sum(ex.map(one, range(jobs)))
            dt = time.perf_counter() - t1
            res["cpu_reference"] = {"tiles_per_s": done / dt, "mvox_per_s": done * inner_vox / dt / 1e6,
                                    "cores": cores, "kind": "reference",
                                    "sample": f"{done} tiles, one per host thread; single-thread {t_one * 1e3:.0f} ms "
                                              "per tile"}
            same = [np.count_nonzero(ref_out[k] != outs[k]) for k in range(min(done, len(tiles)))]
            res["u8_voxels_differing_from_reference"] = {"tiles": len(same), "voxels": int(sum(same)),
                                                         "of": len(same) * inner_vox}
    except Exception as exc:          # reported, never required
        res["cpu_reference"] = {"error": str(exc)[:200]}
    return res


def viewer_slab_sample(fb, lib, dev, seed, reps=40, cpu_budget_s=5.0):
    """The viewer path (README.md:109-118, :190): fy_deconvolve (auto reg) on 8x512x512 f32
    slabs with the reference physics, as an interactive caller issues it. Host API on pageable
    buffers, one call at a time (copies inside each call), and the device form on resident
    buffers; beside them the reference's fy_deconvolve on the host."""
    import torch
    rng = np.random.default_rng(seed)
    shape = (8, 512, 512)
    n = int(np.prod(shape))
    slab = rng.uniform(0.0, 1.0, shape).astype(np.float32)
    out = np.empty_like(slab)
    ph = fb.physics()
    t_host = []
    for i in range(reps + 3):
        t0 = time.perf_counter()
        fb.check(lib.fy_deconvolve(slab.ctypes.data, out.ctypes.data, *shape, C.byref(ph), -1.0), "fy_deconvolve")
        if i >= 3:
            t_host.append(time.perf_counter() - t0)
    d_in = torch.from_numpy(slab).to(f"cuda:{dev}")
    d_out = torch.empty_like(d_in)
    st = torch.cuda.Stream(device=dev)
    args = (C.c_void_p(d_in.data_ptr()), 0, 0.0, 0.0, C.c_void_p(d_out.data_ptr()), *shape, C.byref(ph), -1.0, 0, 1.0,
            C.c_void_p(st.cuda_stream))
    for _ in range(3):
        fb.check(lib.fy_gpu_deconvolve_ex(*args), "fy_gpu_deconvolve_ex")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(st)
    for _ in range(reps):
        lib.fy_gpu_deconvolve_ex(*args)
    e1.record(st)
    e1.synchronize()
    dev_ms = e0.elapsed_time(e1) / reps
    p50 = float(np.percentile(t_host, 50)) * 1e3
    res = {"workload": "fy_deconvolve, auto reg, reference physics, 8x512x512 f32 slab (uniform [0,1])",
           "e2e": {"ms_p50": p50, "ms_p99": float(np.percentile(t_host, 99)) * 1e3, "mvox_per_s": n / p50 / 1e3,
                   "api": "fy_deconvolve, pageable host buffers, one call at a time",
                   "h2d_bytes": 4 * n, "d2h_bytes": 4 * n},
           "resident": {"ms_per_slab": dev_ms, "mvox_per_s": n / dev_ms / 1e3,
                        "api": "fy_gpu_deconvolve_ex, device buffers, back to back on one stream"}}
    try:
        import oracle
        if oracle.have_ref() and cpu_budget_s > 0:
            rph = oracle.RefPhysics(*[getattr(ph, k) for k, _ in ph._fields_])
            ts = []
            t_end = time.perf_counter() + cpu_budget_s
            while time.perf_counter() < t_end and len(ts) < 20:
                t0 = time.perf_counter()
                oracle.ref_deconvolve(slab, rph, -1.0)
                ts.append(time.perf_counter() - t0)
            ms = float(np.median(ts)) * 1e3
            res["cpu_reference"] = {"ms_per_slab": ms, "mvox_per_s": n / ms / 1e3, "cores": os.cpu_count(),
                                    "kind": "reference",
                                    "sample": f"{len(ts)} calls of the reference's fy_deconvolve (its own "
                                              "OpenMP threads), median"}
    except Exception as exc:          # reported, never required
        res["cpu_reference"] = {"error": str(exc)[:200]}
    return res


def phasecorr_sample(fb, lib, dev, seed, db_scale, npairs=64, n=256, distinct=8, cpu_budget_s=10.0):
    """Config-4 sample: npairs pairs of n^3 f32 volumes; the moving volume is an FP64 Fourier
    shift of the fixed one (integer U[-40,40] + subvoxel U[-0.5,0.5] per axis), each with
    independent noise var = 0.002*I + 1e-4. `distinct` different pairs are tiled to npairs.
    One batched call (fy_gpu_phase_correlate_batch, window 0) is timed; the reference CPU path
    runs a bounded sample of the same pairs, one per host thread."""
    import torch
    import fysics_b200.phantom as ph
    rng = np.random.default_rng(seed)
    g = torch.Generator(device=f"cuda:{dev}").manual_seed(int(seed))
    u = ph.phantom((n, n, n), seed=seed, delta_beta=500.0 * db_scale, pixel_um=2.4, device=f"cuda:{dev}")
    f = u.to(torch.float64) / 255.0
    F = torch.fft.fftn(f)
    k = torch.fft.fftfreq(n, device=f"cuda:{dev}", dtype=torch.float64) * n
    k[n // 2] = n // 2                           # the reference keeps k = n/2 positive
    truths, fixed, moving = [], [], []
    for i in range(distinct):
        s = rng.integers(-40, 41, 3) + rng.uniform(-0.5, 0.5, 3)
        ph_ = -2 * np.pi * (k[:, None, None] * s[0] + k[None, :, None] * s[1] + k[None, None, :] * s[2]) / n
        m = torch.fft.ifftn(F * torch.exp(1j * ph_)).real
        noise = lambda v: v + torch.sqrt(0.002 * v.clamp(min=0) + 1e-4) * torch.randn(v.shape, generator=g,
                                                                                      device=v.device, dtype=v.dtype)
        fixed.append(noise(f).float())
        moving.append(noise(m).float())
        truths.append(s)
    del F
    d_fixed = torch.stack([fixed[i % distinct] for i in range(npairs)])
    d_moving = torch.stack([moving[i % distinct] for i in range(npairs)])
    scratch = torch.empty(lib.fy_gpu_phase_correlate_scratch_bytes(n, n, n), dtype=torch.uint8, device=f"cuda:{dev}")
    sh = (C.c_double * (3 * npairs))()
    pk = (C.c_double * npairs)()
    st = (C.c_int * npairs)()
    args = (C.c_void_p(d_fixed.data_ptr()), C.c_void_p(d_moving.data_ptr()), npairs, n, n, n, 0,
            C.c_void_p(scratch.data_ptr()), sh, pk, None, st, None)
    torch.cuda.synchronize()
    fb.check(lib.fy_gpu_phase_correlate_batch(*args[:2], min(npairs, 2), *args[3:]), "phase correlate warm-up")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    fb.check(lib.fy_gpu_phase_correlate_batch(*args), "fy_gpu_phase_correlate_batch")
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    got = np.array(sh[:]).reshape(npairs, 3)
    want = np.array([truths[i % distinct] for i in range(npairs)])
    err = np.abs(got - want)
    res = {"workload": f"{npairs} pairs of {n}^3 f32 ({distinct} distinct pairs tiled), FP64 Fourier shift "
                       "integer U[-40,40] + subvoxel U[-0.5,0.5] per axis, noise var = 0.002*I + 1e-4, window 0; "
                       "inputs resident on the device, one batched call",
           "pairs_per_s": npairs / dt, "mvox_pairs_per_s": npairs * n ** 3 / dt / 1e6,
           "ms_per_pair": dt * 1e3 / npairs, "status_ok": int(sum(1 for i in range(npairs) if st[i] == 0)),
           "integer_exact": int(np.sum(np.all(np.round(got) == np.round(want), axis=1))),
           "mean_abs_err_vox": float(err.mean()), "max_abs_err_vox": float(err.max())}
    # reference CPU path on a bounded sample: one pair per host thread
    try:
        import oracle
        from concurrent.futures import ThreadPoolExecutor
        if oracle.have_ref() and cpu_budget_s > 0:
            L = oracle.ref()
            hf = [fixed[i].cpu().numpy() for i in range(distinct)]
            hm = [moving[i].cpu().numpy() for i in range(distinct)]

            def one(i):
                s3 = (C.c_double * 3)()
                p1 = C.c_double()
                L.fy_phase_correlate(oracle.p(hf[i % distinct]), oracle.p(hm[i % distinct]), n, n, n, s3, C.byref(p1), 0)
                return 1

            t1 = time.perf_counter()
            one(0)
            t_one = time.perf_counter() - t1
            cores = os.cpu_count() or 1
            jobs = cores if t_one < cpu_budget_s else 1      # one wave of pairs, one per thread
            t1 = time.perf_counter()
            with ThreadPoolExecutor(max_workers=cores) as ex:
                done = sum(ex.map(one, range(jobs)))
            res["cpu_reference"] = {"pairs_per_s": done / (time.perf_counter() - t1), "cores": cores,
                                    "sample": f"{done} pairs, one per host thread; single-thread {t_one:.2f} s per pair"}
    except Exception as exc:             # reported, never required
        res["cpu_reference"] = {"error": str(exc)[:200]}
    return res


# ------------------------------------------------------------------------------ main
def dist_setup(n_gpus: int, backend: str = "nccl"):
    """One process per GPU (torchrun env). Replicas only: the only collectives are the
    barrier and the max over ranks of the timed regions."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world <= 1:
        return 0, 1, 0, None
    import torch
    import torch.distributed as dist
    rank = int(os.environ["RANK"])
    local = int(os.environ.get("LOCAL_RANK", rank))
    if backend == "nccl":
        torch.cuda.set_device(local)
    import datetime
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return rank, world, local, dist


def max_over_ranks(value: float, dist, device=None) -> float:
    """The job's time is the slowest rank's (max over ranks); identity on one process."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_mvox_per_s(world: int, vox_per_rank: int, steps: int, total_ms: float) -> float:
    """Whole-job throughput: every rank processes its own cubes (weak scaling)."""
    return world * vox_per_rank * steps / (total_ms * 1e-3) / 1e6


def bench_config(db_scale: float, world: int) -> dict:
    """The workload's description; both arms print the same one."""
    return {"workload": WORKLOAD, "cube": f"{SHAPE[0]}^3 u8", "deltabeta_scale": db_scale,
            "l2": "inputs and working set (~3 GB) larger than the 126 MB L2",
            "parallelism": f"replicas x{world} (one cube per GPU, no collective)"}


def benchmark_cube(args, rank: int, delta_beta: float, device: str):
    """The benchmark's seeded phantom cube (the same in both arms: same seed, recipe, device)."""
    import fysics_b200.phantom as ph
    return ph.phantom(SHAPE, seed=args.seed + rank, delta_beta=delta_beta, energy_kev=110.0, distance_mm=1200.0,
                      pixel_um=2.4, unsharp_sigma=0.8, unsharp_coeff=0.5, fz2_scale=1.17 ** 2, rings=40,
                      device=device)


def run_reference(args, rank, world):
    """The reference's own CPU chain on the benchmark cube (rank 0 only; the other ranks exit)."""
    if rank != 0:
        return
    import oracle
    if not oracle.have_ref():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libfysics_ref.so not built"}))
        return
    rph = oracle.ref_physics(delta_beta=500.0, energy_kev=110.0, distance_mm=1200.0, pixel_um=2.4, unsharp_sigma=0.8,
                             unsharp_coeff=0.5, psf_sigma_vox=1.0, psf_sigma_z_vox=1.17)
    db_scale = oracle.ref().fy_auto_deltabeta_scale(C.byref(rph))
    import torch
    dev = "cuda" if torch.cuda.is_available() and not args.cpu_phantom else "cpu"
    u8 = benchmark_cube(args, 0, 500.0 * db_scale, dev)
    u8 = u8.cpu().numpy() if hasattr(u8, "cpu") else u8
    spec = chain_spec(db_scale)
    res = cpu_reference_chain(u8, spec, threads=args.cpu_threads, warmup=args.warmup, keep_output=False)
    try:
        res["crops_128"] = cpu_reference_crops(u8, spec, budget_s=10.0)
    except Exception as exc:          # secondary figure, reported only
        res["crops_128"] = {"error": str(exc)[:200]}
    line = {"metric": METRIC, "value": res["value"], "unit": "Mvoxel/s", "impl": "reference",
            "n_gpus": world, "steps": res["cubes"], "warmup": args.warmup,
            "ms_per_step": res["wall_s"] * 1e3 / res["cubes"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": bench_config(db_scale, world),
            "timing": f"{res['cubes']} cubes restored concurrently, one per host thread, in {res['wall_s']:.1f} s "
                      "wall (steps = cubes timed, ms_per_step = wall / cubes); warm-up: "
                      f"{args.warmup} chains of a 128^3 crop per thread",
            "cpu_baseline": res,
            "e2e": {"value": res["value"], "unit": "Mvoxel/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


SWEEP_RATES = (200.0, 400.0, 700.0, 1000.0, 1400.0, 2000.0)


def run_serve_sweep(args, rank, local):
    """The serving configuration at its stated scale: `--sweep-requests` requests (sizes
    64^3:128^3:256^3:512^3 = 40:30:25:5, Poisson arrivals) through the request loop at each
    rate of SWEEP_RATES; per rate the throughput and p50/p99 latency overall and per size, and
    the highest rate whose 256^3 p99 stays under 10 ms."""
    if rank != 0:
        return
    import fysics_b200 as fb
    lib = fb.load()
    fb.check(lib.fy_gpu_init(local), "fy_gpu_init")
    import torch
    torch.cuda.set_device(local)
    _, db_scale = physics_for(fb)
    served, _ = served_and_batched(fb, lib, local, args.seed, db_scale, n_requests=args.sweep_requests,
                                   rates=SWEEP_RATES, n_batch=0)
    ok = [pt["arrival_rps"] for pt in served["points"] if pt["p99_ms_by_size"].get("256^3", 1e9) < 10.0]
    line = {"mode": "serve_sweep", "metric": METRIC, "unit": "Mvoxel/s", "requests_per_rate": args.sweep_requests,
            "rates_rps": list(SWEEP_RATES),
            "max_rate_rps_256_p99_under_10ms": max(ok) if ok else None,
            "served": served}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--seed", type=int, default=2026)
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline leg")
    ap.add_argument("--cpu-threads", type=int, default=None,
                    help="host threads of the reference chain (default: cores, bounded by host memory)")
    ap.add_argument("--cpu-phantom", action="store_true")
    ap.add_argument("--size", type=int, default=512, help="cube edge (512 = the benchmark workload)")
    ap.add_argument("--no-serve", action="store_true", help="skip the served / batched samples")
    ap.add_argument("--no-phasecorr", action="store_true", help="skip the registration sample")
    ap.add_argument("--no-tiles", action="store_true", help="skip the per-tile export chain sample")
    ap.add_argument("--no-viewer", action="store_true", help="skip the viewer slab sample")
    ap.add_argument("--serve-sweep", action="store_true",
                    help="the serving configuration at its stated scale instead of the benchmark: 20,000 "
                         "requests per arrival rate over a sweep of 200-2000 req/s (one JSON line)")
    ap.add_argument("--sweep-requests", type=int, default=20000)
    args = ap.parse_args()
    global SHAPE, WORKLOAD
    if args.size != 512:
        SHAPE = (args.size,) * 3
        WORKLOAD = WORKLOAD.replace("512^3", f"{args.size}^3")
    args.warmup = max(args.warmup, 3)
    rank, world, local, dist = dist_setup(args.gpus)
    if args.serve_sweep:
        run_serve_sweep(args, rank, local)
        if dist:
            dist.destroy_process_group()
        return
    if args.impl == "reference":
        run_reference(args, rank, world)
        if dist:
            dist.destroy_process_group()
        return

    import torch
    import fysics_b200 as fb
    import fysics_b200.phantom as ph
    lib = fb.load()
    dev = local
    fb.check(lib.fy_gpu_init(dev), "fy_gpu_init")
    torch.cuda.set_device(dev)
    p, db_scale = physics_for(fb)
    # launch shapes measured for this cube shape on this GPU (cached; set-up, not timed)
    t_tune = time.perf_counter()
    rc_tune = lib.fy_gpu_autotune(*SHAPE, 0)
    t_tune = time.perf_counter() - t_tune
    px = lib.fy_next_fft_size(SHAPE[2])
    tune_knobs = [f"x1.{px}", f"x5.{px}"]
    tuning = {"rc": rc_tune, "seconds": round(t_tune, 2),
              "values": {k: lib.fy_gpu_tune_value(k.encode()) for k in tune_knobs}}
    u8 = benchmark_cube(args, rank, p.delta_beta, f"cuda:{dev}")
    nz, ny, nx = SHAPE
    n = nz * ny * nx
    out = torch.empty(SHAPE, dtype=torch.float32, device=f"cuda:{dev}")
    stream = torch.cuda.Stream(device=dev)
    sp = C.c_void_p(stream.cuda_stream)
    h = C.c_void_p()
    fb.check(lib.fy_gpu_dering_create(C.byref(h), nz, ny, nx, -1.0, -1.0, 512, 8), "fy_gpu_dering_create")
    cfg = restore_cfg(fb, h)

    def step(src_ptr, dst_ptr):
        fb.check(lib.fy_gpu_dering_reset(h, sp), "fy_gpu_dering_reset")
        fb.check(lib.fy_gpu_restore_u8(src_ptr, dst_ptr, nz, ny, nx, 0.0, 1.0, C.byref(p), C.byref(cfg), sp),
                 "fy_gpu_restore_u8")

    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step(C.c_void_p(u8.data_ptr()), C.c_void_p(out.data_ptr()))
    torch.cuda.synchronize()

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- device-resident timed region (per-step events -> latency; profile marks)
    clocks = ClockSampler(dev)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    launches0 = lib.fy_gpu_kernel_launches()
    barrier()
    clocks.start()
    # the timed loop records only the events around the guided output pass (each event between
    # two launches costs them their overlap); the per-pass table comes from a profiled run after
    lib.fy_gpu_profile_select(TIMED_MARKS.encode())
    lib.fy_gpu_profile_start(64 * args.steps + 8, sp)
    with torch.cuda.stream(stream):
        ev[0].record(stream)
        for k in range(args.steps):
            step(C.c_void_p(u8.data_ptr()), C.c_void_p(out.data_ptr()))
            ev[k + 1].record(stream)
    stream.synchronize()
    barrier()
    clock = clocks.stop()
    launches = lib.fy_gpu_kernel_launches() - launches0
    prof_timed = read_profile(lib)
    lib.fy_gpu_profile_select(None)
    # ---- per-pass events: a separate profiled run of the same step (not the timed number)
    prof_steps = max(1, min(args.steps, 5))
    lib.fy_gpu_profile_start(64 * prof_steps + 8, sp)
    with torch.cuda.stream(stream):
        for _ in range(prof_steps):
            step(C.c_void_p(u8.data_ptr()), C.c_void_p(out.data_ptr()))
    stream.synchronize()
    prof = read_profile(lib)
    per_step = [ev[k].elapsed_time(ev[k + 1]) for k in range(args.steps)]
    total_ms = max_over_ranks(ev[0].elapsed_time(ev[args.steps]), dist, f"cuda:{dev}")
    ms_step = total_ms / args.steps
    value = job_mvox_per_s(world, n, args.steps, total_ms)

    # ---- end to end through pinned host buffers: the same chain through the public call,
    # each cube's H2D and D2H inside the timed region. Three streams form a pipeline -- input
    # copies, chains, output copies -- linked by events, over NSLOT buffer slots (device
    # input and output, pinned result and ring handle each). The output link, which bounds
    # this leg (537 MB of f32 per cube), then carries one result after another while the
    # next inputs land and the next chain runs.
    NSLOT = 3
    h_in = torch.empty(SHAPE, dtype=torch.uint8, pin_memory=True)
    h_in.copy_(u8.cpu())
    st_in, st_run, st_out = (torch.cuda.Stream(device=dev) for _ in range(3))
    slots = []
    for _ in range(NSLOT):
        hs = C.c_void_p()
        fb.check(lib.fy_gpu_dering_create(C.byref(hs), nz, ny, nx, -1.0, -1.0, 512, 8), "fy_gpu_dering_create")
        slots.append({"d_in": torch.empty_like(u8), "d_out": torch.empty_like(out),
                      "h_out": torch.empty(SHAPE, dtype=torch.float32, pin_memory=True), "ring": hs,
                      "cfg": restore_cfg(fb, hs)})
    e2e_steps = max(4, min(args.steps, 10))
    spr = C.c_void_p(st_run.cuda_stream)

    def new_events(k):
        return [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(k)]

    def e2e_cube(k, ev):
        """ev[k] = input copy start, input landed, chain done, result landed."""
        sl = slots[k % NSLOT]
        if k >= NSLOT:
            st_in.wait_event(ev[k - NSLOT][2])           # d_in free: the slot's last chain read it
            st_run.wait_event(ev[k - NSLOT][3])          # d_out free: the slot's last result is out
        with torch.cuda.stream(st_in):
            ev[k][0].record(st_in)
            sl["d_in"].copy_(h_in, non_blocking=True)
            ev[k][1].record(st_in)
        st_run.wait_event(ev[k][1])
        with torch.cuda.stream(st_run):
            fb.check(lib.fy_gpu_dering_reset(sl["ring"], spr), "fy_gpu_dering_reset")
            fb.check(lib.fy_gpu_restore_u8(C.c_void_p(sl["d_in"].data_ptr()), C.c_void_p(sl["d_out"].data_ptr()),
                                           nz, ny, nx, 0.0, 1.0, C.byref(p), C.byref(sl["cfg"]), spr),
                     "fy_gpu_restore_u8")
            ev[k][2].record(st_run)
        st_out.wait_event(ev[k][2])
        with torch.cuda.stream(st_out):
            sl["h_out"].copy_(sl["d_out"], non_blocking=True)
            ev[k][3].record(st_out)

    warm = new_events(NSLOT)
    for k in range(NSLOT):                               # warm every slot's buffers
        e2e_cube(k, warm)
    torch.cuda.synchronize()
    ev = new_events(e2e_steps)
    barrier()
    t_e2e = time.perf_counter()
    for k in range(e2e_steps):
        if k >= NSLOT:
            ev[k - NSLOT][3].synchronize()               # the caller has the slot's last result
        e2e_cube(k, ev)
    torch.cuda.synchronize()
    barrier()
    e2e_wall_ms = (time.perf_counter() - t_e2e) * 1e3
    e2e_steps_ms = [ev[k][0].elapsed_time(ev[k][3]) for k in range(e2e_steps)]
    e2e_dev_ms = ev[0][0].elapsed_time(ev[e2e_steps - 1][3])
    for sl in slots:
        lib.fy_gpu_dering_destroy(sl["ring"])
    e2e_ms = max_over_ranks(max(e2e_dev_ms, e2e_wall_ms), dist, f"cuda:{dev}")
    e2e_value = job_mvox_per_s(world, n, e2e_steps, e2e_ms)

    # ---- roofline of the dominant kernel (live event timings above)
    peaks = {}
    try:
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except Exception:
        pass
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    geo = {"shape": SHAPE, "px": fb.load().fy_next_fft_size(nx), "py": fb.load().fy_next_fft_size(ny),
           "shared_window": cfg.noise_win == 2 * cfg.guided_radius + 1 and cfg.guided_s <= 1}
    kernels = {}
    for name, v in prof.items():
        avg = sum(v) / len(v)
        ab = algorithmic_bytes(name, n, geo)
        kernels[name] = {"avg_ms": avg, "launches": len(v), "share": sum(v) / max(sum(map(sum, prof.values())), 1e-9),
                         "gbs": (ab / (avg * 1e-3) / 1e9) if ab else None}
    dom = max((k for k in kernels if kernels[k]["gbs"] is not None), key=lambda k: kernels[k]["avg_ms"], default=None)
    roof = None
    if dom:
        ach = kernels[dom]["gbs"]
        timed_ms = None
        if dom in prof_timed:                 # the dominant pass's events inside the timed loop
            v = prof_timed[dom]
            timed_ms = sum(v) / len(v)
            ach = algorithmic_bytes(dom, n, geo) / (timed_ms * 1e-3) / 1e9
        tpv = DRAM_BYTES_PER_VOXEL.get(dom)
        roof = {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": hbm_peak, "unit": "GB/s",
                "frac": ach / hbm_peak, "traffic": tpv * n if tpv is not None and SHAPE == (512, 512, 512) else None,
                "traffic_source": "ncu DRAM capture of the chain on a 384^3 cube, bytes per voxel x voxels",
                "peak_source": peak_src,
                "algorithmic_bytes_per_launch": algorithmic_bytes(dom, n, geo),
                "duration_ms": timed_ms if timed_ms is not None else kernels[dom]["avg_ms"],
                "duration_source": ("CUDA events around the pass inside the timed loop" if timed_ms is not None
                                    else "CUDA events of the separate profiled run")}

    # ---- the reference's chain on the same cube (host cores), and the benchmark output's
    # error against it: `out` holds the last timed step's result (the chain is deterministic)
    cpu = parity = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            import oracle
            if oracle.have_ref():
                cpu = cpu_reference_chain(u8.cpu().numpy(), chain_spec(db_scale), threads=args.cpu_threads,
                                          warmup=args.warmup)
                ref_out = cpu.pop("_out")
                got = out.cpu().numpy()
                err = np.abs(got - ref_out["out"])
                parity = {"against": "the reference's chain on the same cube (oracle/_ref)",
                          "max_abs_err": float(err.max()), "mean_abs_err": float(err.mean()),
                          "window_range": 1.0, "bar": 1e-4, "within_bar": bool(err.max() <= 1e-4),
                          "detected_rings_ref": ref_out["detected"], "noise_ref_ref": ref_out["noise_ref"]}
                del got, err, ref_out
        except Exception as exc:       # the baseline is reported, never required
            cpu = {"value": None, "error": str(exc)[:200]}

    # the legs' CPU reference samples use every host core: rank 0 of a one-GPU run only, as
    # the cpu_baseline leg
    cpu_legs = rank == 0 and world == 1 and not args.no_cpu
    served = batched = None
    if not args.no_serve:
        try:
            served, batched = served_and_batched(fb, lib, dev, args.seed + 17 * rank, db_scale)
        except Exception as exc:      # reported, never required
            served = {"error": str(exc)[:300]}

    phasecorr = None
    if not args.no_phasecorr:
        try:
            phasecorr = phasecorr_sample(fb, lib, dev, args.seed + 31 * rank, db_scale,
                                         cpu_budget_s=10.0 if cpu_legs else 0.0)
        except Exception as exc:      # reported, never required
            phasecorr = {"error": str(exc)[:300]}

    tiles = None
    if not args.no_tiles:
        try:
            tiles = tiles_sample(fb, lib, dev, args.seed + 43 * rank, cpu_budget_s=10.0 if cpu_legs else 0.0)
        except Exception as exc:      # reported, never required
            tiles = {"error": str(exc)[:300]}

    viewer = None
    if not args.no_viewer:
        try:
            viewer = viewer_slab_sample(fb, lib, dev, args.seed + 59 * rank, cpu_budget_s=5.0 if cpu_legs else 0.0)
        except Exception as exc:      # reported, never required
            viewer = {"error": str(exc)[:300]}

    lat = sorted(per_step)
    line = {
        "metric": METRIC, "value": value, "unit": "Mvoxel/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": bench_config(db_scale, world),
        "tuning": tuning,
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                       "e2e_p50": float(np.percentile(e2e_steps_ms, 50)),
                       "e2e_p99": float(np.percentile(e2e_steps_ms, 99))},
        "e2e": {"value": e2e_value, "unit": "Mvoxel/s", "h2d_bytes_per_step": n, "d2h_bytes_per_step": 4 * n},
        "gpu_launches": int(launches),
        "roofline": roof,
        "kernels": kernels,
        "kernels_source": "CUDA events after each pass in a separate profiled run of the same step "
                          "(the timed loop records only the marks " + TIMED_MARKS + ")",
        "clocks": clock,
        "cpu_baseline": cpu,
        "parity": parity,
        "served": served,
        "batched": batched,
        "phasecorr": phasecorr,
        "tiles": tiles,
        "viewer_slab": viewer,
    }
    lib.fy_gpu_dering_destroy(h)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
