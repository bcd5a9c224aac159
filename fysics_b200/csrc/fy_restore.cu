// fy_restore.cu -- the per-cube restoration chain on device buffers, in the order of the
// path it replaces: u8 dewindow (fused into the deconvolution's first pass) -> Wiener
// deconvolution -> noise model -> guided filter with eps = fy_guided_eps_for_noise(noise_ref)
// read from device memory -> ring subtraction. No host round trip between stages, so the
// whole chain is one stream-ordered sequence (and capturable as a graph per size class).
#include "fy_context.h"

using fy::ctx;
using fy::fail;
using fy::fail_cuda;

// fy_gpu_dering internals needed here (defined in fy_api_dering.cu)
extern "C" int fy_gpu_dering_accumulate_u8(fy_gpu_dering* h, const unsigned char* d_buf, long z0, long y0, long x0,
                                           long dz, long dy, long dx, int ss, void* stream);
extern "C" int fy_gpu_dering_finalize(fy_gpu_dering* h, int hp_win, unsigned int min_cnt, double min_amp,
                                      double max_amp, void* stream);
extern "C" int fy_gpu_dering_apply(const fy_gpu_dering* h, float* d_f, long z0, long y0, long x0, long dz, long dy,
                                   long dx, double scale, void* stream);
extern "C" int fy_gpu_deconvolve_ex(const void* d_in, int src_u8, double f32_min, double f32_max, float* d_out,
                                    int nz, int ny, int nx, const fy_physics* p, double param, int kind,
                                    double fz2_scale, void* stream);

extern "C" void fy_restore_cfg_default(fy_restore_cfg* c) {
    c->deconv_kind = 0;
    c->deconv_param = 0.015;
    c->fz2_scale = 1.0;
    c->noise_win = 5;
    c->noise_flat_pct = 10.0;
    c->noise_ref_intensity = 0.4;
    c->guided_eps = 0.0;
    c->guided_radius = 2;
    c->guided_s = 1;
    c->dering = nullptr;
    c->dering_accumulate = 0;
    c->dering_ss = 2;
    c->dering_hp_win = 15;
    c->dering_min_cnt = 100;
    c->dering_min_amp = 0.5;
    c->dering_max_amp = 6.0;
    c->dering_scale = 1.0 / 255.0;
    c->z0 = c->y0 = c->x0 = 0;
    c->radial = nullptr;
    c->radial_cy = c->radial_cx = 0.0;
}

extern "C" int fy_gpu_restore_u8(const unsigned char* d_u8, float* d_out, int nz, int ny, int nx, double f32_min,
                                 double f32_max, const fy_physics* p, const fy_restore_cfg* cfg, void* stream) {
    fy::enter();
    const char* what = "fy_gpu_restore_u8";
    if (!d_u8 || !d_out || !p || !cfg) return fail(FY_EINVAL, "%s: null pointer", what);
    if (nz < 1 || ny < 1 || nx < 1) return fail(FY_EINVAL, "%s: bad dims", what);
    int win = cfg->noise_win < 3 ? 5 : cfg->noise_win;
    if (win / 2 > 4) return fail(FY_EUNSUPPORTED, "%s: noise win > 9", what);
    int radius = cfg->guided_radius < 1 ? 2 : cfg->guided_radius;
    if (radius > 4 && cfg->guided_s <= 1) return fail(FY_EUNSUPPORTED, "%s: chained guided radius > 4", what);
    int rc = fy::ensure_ctx();
    if (rc) return rc;
    fy::ThreadCtx& c = ctx();
    cudaStream_t st = (cudaStream_t)stream;
    const size_t n = (size_t)nz * ny * nx;
    // 1. ring statistics from the raw u8 input (the pipeline accumulates u8 in pass 1). They
    // need only the input and only the guided output pass reads them, so they run on the
    // thread's side stream, overlapping the deconvolution and the noise model.
    bool ring_join = false;
    if (cfg->dering && cfg->dering_accumulate) {
        if ((rc = fy::ensure_side())) return rc;
        cudaError_t e0;
        if ((e0 = cudaEventRecord(c.fork_ev, st)) != cudaSuccess || (e0 = cudaStreamWaitEvent(c.side, c.fork_ev, 0)) !=
            cudaSuccess)
            return fail_cuda(e0, what);
        if ((rc = fy_gpu_dering_accumulate_u8(cfg->dering, d_u8, cfg->z0, cfg->y0, cfg->x0, nz, ny, nx,
                                              cfg->dering_ss, c.side)))
            return rc;
        if ((rc = fy_gpu_dering_finalize(cfg->dering, cfg->dering_hp_win, cfg->dering_min_cnt, cfg->dering_min_amp,
                                         cfg->dering_max_amp, c.side)))
            return rc;
        if ((e0 = cudaEventRecord(c.join_ev, c.side)) != cudaSuccess) return fail_cuda(e0, what);
        ring_join = true;
    }
    fy::ws_acquire(st);
    cudaError_t e;
    if ((e = c.aux2.ensure(n * sizeof(float))) != cudaSuccess) return fail_cuda(e, what);
    float* dec = c.aux2.as<float>();
    fy::ws_release(st);      // deconvolve_ex re-acquires the shared workspaces
    // 2. dewindow + deconvolution into `dec`
    if ((rc = fy_gpu_deconvolve_ex(d_u8, 1, f32_min, f32_max, dec, nz, ny, nx, p, cfg->deconv_param,
                                   cfg->deconv_kind, cfg->fz2_scale, stream)))
        return rc;
    fy::ws_acquire(st);
    // 3. noise model on the deconvolved volume -> device eps. When the noise window is the
    // exact guided filter's window, the statistics pass also writes the guided (mean, var)
    // pairs (after the noise scratch), and the guided filter runs its output pass only.
    const float* eps_ptr = nullptr;
    int launches = 0;
    const bool noise = !(cfg->guided_eps > 0);
    const bool shared_window = noise && cfg->guided_s <= 1 && win == 2 * radius + 1;
    const size_t mv_off = fy_noise_scratch_floats(n);
    if (noise) {
        const size_t need = mv_off + (shared_window ? fy_guided_fused_scratch_floats(n) : 0);
        if ((e = c.aux.ensure(need * sizeof(float))) != cudaSuccess) return fail_cuda(e, what);
        if ((e = c.small.ensure(fy_noise_ctl_bytes())) != cudaSuccess) return fail_cuda(e, what);
        double pct = cfg->noise_flat_pct <= 0 ? 10.0 : cfg->noise_flat_pct;
        if ((e = fy_launch_estimate_noise(dec, nz, ny, nx, win, pct, cfg->noise_ref_intensity, c.aux.as<float>(),
                                          c.small.p, c.sms, st, launches,
                                          shared_window ? c.aux.as<float>() + mv_off : nullptr)) != cudaSuccess)
            return fail_cuda(e, what);
        eps_ptr = fy_noise_eps_ptr(c.small.p);
        fy_prof_mark(st, "noise");
    }
    const float eps = (float)(cfg->guided_eps > 0 ? cfg->guided_eps : 0.0);
    if (cfg->radial) {       // radial model: this cube's eps = base eps * clamp((fn(r)/median)^2, 0.4, 8)
        const size_t off = fy_noise_ctl_bytes();
        if ((e = c.small.ensure(off + 256)) != cudaSuccess) return fail_cuda(e, what);
        float* d_eps = (float*)((char*)c.small.p + off);
        if ((e = fy_launch_radial_tile_eps(cfg->radial, eps_ptr, eps, cfg->radial_cy, cfg->radial_cx, cfg->y0, cfg->x0,
                                           ny, nx, d_eps, st)) != cudaSuccess)
            return fail_cuda(e, what);
        launches += 1;
        eps_ptr = d_eps;
    }
    // 4. guided filter dec -> d_out (after the ring statistics, when they ran on the side stream)
    if (ring_join && (e = cudaStreamWaitEvent(st, c.join_ev, 0)) != cudaSuccess) return fail_cuda(e, what);
    bool rings_done = false;
    if (cfg->guided_s > 1) {
        const int s = cfg->guided_s;
        const int lz = (nz + s - 1) / s, ly = (ny + s - 1) / s, lx = (nx + s - 1) / s;
        int rl = radius / s; if (rl < 1) rl = 1;
        if (lz >= 2 && ly >= 2 && lx >= 2 && rl <= 4) {
            if ((e = c.vout.ensure(fy_guided_fast_scratch_floats(lz, ly, lx) * sizeof(float))) != cudaSuccess)
                return fail_cuda(e, what);
            e = fy_launch_guided_fast(dec, d_out, c.vout.as<float>(), nz, ny, nx, radius, eps, s, c.sms, st, launches,
                                      eps_ptr);
        } else {
            if ((e = c.aux.ensure(fy_guided_fused_scratch_floats(n) * sizeof(float))) != cudaSuccess)
                return fail_cuda(e, what);
            e = fy_launch_guided_fused(dec, d_out, nullptr, c.aux.as<float>(), nz, ny, nx, radius, eps, 0, c.sms, st,
                                       eps_ptr);
            launches += 2;
        }
    } else {
        // the ring subtraction is folded into the guided filter's output pass
        RingApply ra;
        if (cfg->dering) fy_dering_ring_args(cfg->dering, cfg->z0, cfg->y0, cfg->x0, cfg->dering_scale, &ra);
        if (shared_window) {
            e = fy_launch_guided_apply_mv(c.aux.as<float>() + mv_off, dec, d_out, nz, ny, nx, radius, eps, c.sms, st,
                                          eps_ptr, cfg->dering ? &ra : nullptr);
            launches += 1;
        } else {
            // a, b reuse the noise statistics' scratch: the model is final by now (stream order)
            if ((e = c.aux.ensure(fy_guided_fused_scratch_floats(n) * sizeof(float))) != cudaSuccess)
                return fail_cuda(e, what);
            e = fy_launch_guided_fused(dec, d_out, nullptr, c.aux.as<float>(), nz, ny, nx, radius, eps, 0, c.sms, st,
                                       eps_ptr, cfg->dering ? &ra : nullptr);
            launches += 2;
        }
        rings_done = cfg->dering != nullptr;
    }
    if (e != cudaSuccess) return fail_cuda(e, what);
    fy_prof_mark(st, "guided");
    fy::count_launch(launches);
    fy::ws_release(st);
    // 5. ring subtraction (no-op on the device when fewer than 2 radii were detected), unless
    // the exact guided filter already applied it
    if (cfg->dering && !rings_done) {
        if ((rc = fy_gpu_dering_apply(cfg->dering, d_out, cfg->z0, cfg->y0, cfg->x0, nz, ny, nx, cfg->dering_scale,
                                      stream)))
            return rc;
        fy_prof_mark(st, "dering.apply");
    }
    return FY_OK;
}

// Size every workspace the chain uses for a cube shape (exact guided path), so later calls
// up to that shape allocate nothing: growing a workspace frees the old buffer, and a free
// synchronises the whole device.
int fy_restore_reserve(int nz, int ny, int nx) {
    int rc = fy_deconv_reserve(nz, ny, nx);
    if (rc) return rc;
    fy::ThreadCtx& c = ctx();
    const size_t n = (size_t)nz * ny * nx;
    size_t aux = fy_noise_scratch_floats(n) + fy_guided_fused_scratch_floats(n);   // noise + guided (mean, var)
    cudaError_t e;
    if ((e = c.aux2.ensure(n * sizeof(float))) != cudaSuccess || (e = c.aux.ensure(aux * sizeof(float))) != cudaSuccess ||
        (e = c.small.ensure(fy_noise_ctl_bytes() + 256)) != cudaSuccess)
        return fail_cuda(e, "fy_restore_reserve");
    return FY_OK;
}
