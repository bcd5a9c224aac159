"""The per-cube restoration chain on the CPU, as the checker of the GPU chain.

Test infrastructure only: the tests, smoke() and bench.py's CPU legs call these; the
product library never does.

Chain (the order of the benchmark configurations): u8 dewindow -> Wiener deconvolution
(fy_deconvolve, or fy_deconvolve_matched with its anisotropic z scale) -> noise model
(fy_estimate_noise) -> guided filter with eps = fy_guided_eps_for_noise(noise_ref) ->
optional ring subtraction (accumulate the u8 input, vote, apply with scale span/255).

  ref_restore   the reference library compiled from its own sources (oracle/_ref), through
                its public calls (stream.c:41-46, paganin.c:301-342, noise.c:75-192,
                noise.c:197-202, guided.c:233-241, dering.c:31-248);
  o64_restore   the FP64 restatement (fy_oracle64.c), every stage in double and fed the
                previous stage's double output.

Both return every stage's output so the per-stage errors can be reported.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from oracle import RefDering, RefNoise, RefPhysics, o64, p, ref


@dataclass
class ChainSpec:
    """One chain's settings (the GPU chain's fy_restore_cfg carries the same values)."""
    phys: dict
    window: tuple = (0.0, 1.0)
    matched: bool = False             # False: fy_deconvolve (reg); True: fy_deconvolve_matched (gamma)
    deconv_param: float = 0.015
    noise_win: int = 5
    noise_pct: float = 10.0
    noise_ref: float = 0.4
    guided_r: int = 2
    dering: dict | None = None        # ss, hp_win, min_cnt, min_amp, max_amp, slab_z, ns, cy, cx
    extra: dict = field(default_factory=dict)

    def ref_physics(self) -> RefPhysics:
        d = dict(delta_beta=1000.0, energy_kev=78.0, distance_mm=220.0, pixel_um=2.4, unsharp_sigma=1.2,
                 unsharp_coeff=4.0, psf_sigma_vox=0.0, psf_sigma_z_vox=0.0)
        d.update(self.phys)
        return RefPhysics(*[d[n] for n, _ in RefPhysics._fields_])

    def ring_scale(self) -> float:
        return (self.window[1] - self.window[0]) / 255.0


def ref_restore(u8: np.ndarray, spec: ChainSpec, keep_stages: bool = True) -> dict:
    """The reference's chain; returns {'phys','deconv','noise','eps','guided','out','rings'}."""
    L = ref()
    u8 = np.ascontiguousarray(u8, np.uint8)
    nz, ny, nx = u8.shape
    n = u8.size
    ph = spec.ref_physics()
    f = np.empty(u8.shape, np.float32)
    L.fy_u8_to_phys(p(u8), p(f), n, *spec.window)
    d = np.empty_like(f)
    fn = L.fy_deconvolve_matched if spec.matched else L.fy_deconvolve
    assert fn(p(f), p(d), nz, ny, nx, C.byref(ph), spec.deconv_param) == 0
    nm = RefNoise()
    assert L.fy_estimate_noise(p(d), nz, ny, nx, spec.noise_win, spec.noise_pct, spec.noise_ref, C.byref(nm)) == 0
    eps = L.fy_guided_eps_for_noise(nm.noise_ref)
    ws = np.empty(4 * n, np.float32)
    out = np.empty_like(f)
    assert L.fy_guided_denoise_ws(p(d), p(out), nz, ny, nx, spec.guided_r, eps, p(ws)) == 0
    del ws
    res = {"noise": nm, "eps": eps}
    if keep_stages:
        res.update(phys=f, deconv=d, guided=out.copy())
    if spec.dering:
        g = spec.dering
        dr, dt = RefDering(), RefDering()
        assert L.fy_dering_init(C.byref(dr), nz, ny, nx, g.get("cy", -1.0), g.get("cx", -1.0), g.get("slab_z", 512),
                                g.get("ns", 8)) == 0
        assert L.fy_dering_tile_init(C.byref(dt), C.byref(dr)) == 0
        L.fy_dering_accumulate_u8(C.byref(dt), p(u8), 0, 0, nz, ny, nx, g.get("ss", 2))
        L.fy_dering_merge_tile(C.byref(dr), 0, C.byref(dt))
        res["detected"] = L.fy_dering_finalize(C.byref(dr), g.get("hp_win", 15), g.get("min_cnt", 100),
                                               g.get("min_amp", 0.5), g.get("max_amp", 6.0))
        res["rings"] = np.ctypeslib.as_array(dr.ring, (dr.nslab * dr.nr,)).copy() if dr.have_rings else None
        L.fy_dering_apply(C.byref(dr), p(out), 0, 0, 0, nz, ny, nx, spec.ring_scale())
        L.fy_dering_free(C.byref(dt))
        L.fy_dering_free(C.byref(dr))
    res["out"] = out
    return res


def o64_restore(u8: np.ndarray, spec: ChainSpec) -> dict:
    """The FP64 oracle's chain (double throughout); same keys as ref_restore."""
    O = o64()
    u8 = np.ascontiguousarray(u8, np.uint8)
    nz, ny, nx = u8.shape
    n = u8.size
    ph = spec.ref_physics()
    f = np.empty(u8.shape, np.float64)
    O.o64_u8_to_phys(p(u8), p(f), n, *spec.window)
    d = np.empty_like(f)
    assert O.o64_deconvolve(p(f), p(d), nz, ny, nx, C.byref(ph), spec.deconv_param, 1 if spec.matched else 0,
                            1.0, 1) == 0
    nm = RefNoise()
    assert O.o64_estimate_noise64(p(d), nz, ny, nx, spec.noise_win, spec.noise_pct, spec.noise_ref,
                                  C.byref(nm)) == 0
    eps = O.o64_guided_eps_for_noise(nm.noise_ref)
    g64 = np.empty_like(f)
    assert O.o64_guided(p(d), p(g64), nz, ny, nx, spec.guided_r, eps) == 0
    res = {"phys": f, "deconv": d, "noise": nm, "eps": eps, "guided": g64.copy()}
    if spec.dering:
        g = spec.dering
        cy, cx = g.get("cy", -1.0), g.get("cx", -1.0)
        cy = (ny - 1) / 2.0 if cy < 0 else cy
        cx = (nx - 1) / 2.0 if cx < 0 else cx
        slab_z, ns = g.get("slab_z", 512), g.get("ns", 8)
        nr = O.o64_dering_nr(ny, nx, cy, cx)
        nslab = (nz + slab_z - 1) // slab_z
        sums = np.zeros(nslab * ns * nr, np.uint64)
        cnts = np.zeros(nslab * ns * nr, np.uint64)
        for s in range(nslab):                       # one slab's planes at a time, as the tiles merge
            z0, z1 = s * slab_z, min(nz, (s + 1) * slab_z)
            sub = np.ascontiguousarray(u8[z0:z1])
            O.o64_dering_accumulate_u8(p(sub), 0, 0, z1 - z0, ny, nx, g.get("ss", 2), cy, cx, ns, nr,
                                       p(sums[s * ns * nr:]), p(cnts[s * ns * nr:]))
        ring = np.zeros(nslab * nr, np.float64)
        have = C.c_int()
        res["detected"] = O.o64_dering_finalize(p(sums), p(cnts), nslab, ns, nr, g.get("hp_win", 15),
                                                g.get("min_cnt", 100), g.get("min_amp", 0.5),
                                                g.get("max_amp", 6.0), p(ring), C.byref(have))
        res["rings"] = ring if have.value else None
        if have.value:
            O.o64_dering_apply(p(ring), nslab, nr, slab_z, cy, cx, p(g64), 0, 0, 0, nz, ny, nx, spec.ring_scale())
    res["out"] = g64
    return res
