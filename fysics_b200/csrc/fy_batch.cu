// fy_batch.cu -- the restoration chain of fy_gpu_restore_u8 over a batch of volumes of any
// sizes in one call.
//
// One host-built plan per call, uploaded with one copy: every volume's deconvolution tables,
// the jobs of the two box passes and the selection steps' arguments. Then, in stream order:
//   1. the volumes' deconvolutions, spread over kBatchStreams streams (each with its own
//      half-spectrum workspace), joined back into the caller's stream;
//   2. the noise statistics of every volume in one work-queue launch (k_zbox_queue): the
//      (volume, tile, z chunk) items of all volumes in one index space, taken by persistent
//      CTAs, so small volumes leave no tail;
//   3. the noise model's selection, one launch per step for all volumes (each with the CTAs
//      it needs, numbered per volume);
//   4. the guided filter's output pass of every volume in one work-queue launch.
// Each volume's arithmetic is the single-volume chain's (the same tiles, chunks, kernels and
// order statistics), so its output equals fy_gpu_restore_u8's bit for bit. The batched form
// covers the chain with the noise model's eps and the shared noise/guided window without
// rings or a radial model (the configuration of a batch of independent cubes); other
// configurations, and volumes whose rows are not a multiple of 4 floats (no tensor-copy
// staging), run one volume after another through fy_gpu_restore_u8.
#include <string.h>

#include <algorithm>
#include <atomic>
#include <thread>
#include <vector>

#include "fy_context.h"
#include "fy_zbox.cuh"
#include "fysics_b200.h"

using fy::ctx;
using fy::fail;
using fy::fail_cuda;

// fy_noise.cu: the selection steps of many volumes and the statistics pass's parameters
struct NoiseBatch;
NoiseBatch* fy_noise_batch_record(const float* const* in, const int* dims, float* const* scratch,
                                  void* const* ctl_mem, int nvol, int win, double flat_pct, double ref_intensity,
                                  int sms, cudaError_t* err);
size_t fy_noise_batch_bytes(const NoiseBatch* b);
void fy_noise_batch_pack(const NoiseBatch* b, void* host);
int fy_noise_batch_steps(const NoiseBatch* b);
cudaError_t fy_noise_batch_launch(const NoiseBatch* b, const void* dev, cudaStream_t st);
void fy_noise_batch_free(NoiseBatch* b);
fyzb::Params fy_noise_stats_params(const float* in, int nz, int ny, int nx, int win, float* scratch, float* guided_mv);

namespace {
size_t al256(size_t v) { return (v + 255) & ~(size_t)255; }

int one_by_one(const fy_batch_cube* cubes, int n, const fy_restore_cfg* cfg, void* stream) {
    for (int i = 0; i < n; ++i) {
        const fy_batch_cube& q = cubes[i];
        const int rc = fy_gpu_restore_u8(q.u8, q.out, q.nz, q.ny, q.nx, q.f32_min, q.f32_max, &q.phys, cfg, stream);
        if (rc) return rc;
    }
    return FY_OK;
}

// Frees the recorded selection on every exit path.
struct BatchGuard {
    NoiseBatch* nb = nullptr;
    ~BatchGuard() { if (nb) fy_noise_batch_free(nb); }
};
}  // namespace

int fy_batch_wait_timeouts() { return fyzb::timeouts(); }
cudaError_t fy_batch_set_first_wait_polls(int polls) { return fyzb::set_first_wait_polls(polls); }

extern "C" int fy_gpu_restore_u8_batch(const fy_batch_cube* cubes, int n, const fy_restore_cfg* cfg, void* stream) {
    fy::enter();
    const char* what = "fy_gpu_restore_u8_batch";
    if (n < 0 || (n > 0 && !cubes) || !cfg) return fail(FY_EINVAL, "%s: bad arguments", what);
    for (int i = 0; i < n; ++i) {
        const fy_batch_cube& q = cubes[i];
        if (!q.u8 || !q.out) return fail(FY_EINVAL, "%s: volume %d: null pointer", what, i);
        if (q.nz < 1 || q.ny < 1 || q.nx < 1) return fail(FY_EINVAL, "%s: volume %d: bad dims", what, i);
    }
    if (n == 0) return FY_OK;
    int rc = fy::ensure_ctx();
    if (rc) return rc;
    fy::ThreadCtx& c = ctx();
    cudaStream_t st = (cudaStream_t)stream;
    const int win = cfg->noise_win < 3 ? 5 : cfg->noise_win;
    const int radius = cfg->guided_radius < 1 ? 2 : cfg->guided_radius;
    bool batched = !(cfg->guided_eps > 0) && cfg->guided_s <= 1 && win == 2 * radius + 1 && radius <= 4 &&
                   !cfg->dering && !cfg->radial;
    for (int i = 0; i < n && batched; ++i) batched = cubes[i].nx % 4 == 0;
    if (!batched) return one_by_one(cubes, n, cfg, stream);
    if ((rc = fy::ensure_batch_streams())) return rc;
    const int K = n < fy::ThreadCtx::kBatchStreams ? n : fy::ThreadCtx::kBatchStreams;
    const double pct = cfg->noise_flat_pct <= 0 ? 10.0 : cfg->noise_flat_pct;

    // ---- per-volume buffers (one arena) and the deconvolution launches
    std::vector<size_t> off_dec(n), off_scr(n), off_mv(n), off_ctl(n), off_tab(n);
    std::vector<DeconvLaunch> dl(n);
    std::vector<double> params(n), fz2ss(n);
    size_t arena = 0, spec_max = 0, tab_bytes = 0;
    for (int i = 0; i < n; ++i) {
        const fy_batch_cube& q = cubes[i];
        const size_t vox = (size_t)q.nz * q.ny * q.nx;
        off_dec[i] = arena; arena += al256(vox * sizeof(float));
        off_scr[i] = arena; arena += al256(fy_noise_scratch_floats(vox) * sizeof(float));
        off_mv[i] = arena; arena += al256(fy_guided_fused_scratch_floats(vox) * sizeof(float));
        off_ctl[i] = arena; arena += al256(fy_noise_ctl_bytes());
        params[i] = cfg->deconv_param;
        fz2ss[i] = cfg->fz2_scale;
        if ((rc = fy_deconv_setup(q.nz, q.ny, q.nx, &q.phys, params[i], cfg->deconv_kind, fz2ss[i], q.f32_min,
                                  q.f32_max, dl[i], what)))
            return rc;
        const size_t se = fy_deconv_spec_elems(dl[i].g) * sizeof(float2);
        spec_max = se > spec_max ? se : spec_max;
        off_tab[i] = tab_bytes;
        tab_bytes += al256(fy_deconv_table_bytes(dl[i].g));
    }
    // ---- the uploaded plan: tables, the two passes' jobs, their queue counters, the selection
    const size_t off_jobs_s = al256(tab_bytes);
    const size_t off_jobs_g = off_jobs_s + al256((size_t)n * sizeof(fyzb::BoxJob));
    const size_t off_next = off_jobs_g + al256((size_t)n * sizeof(fyzb::BoxJob));
    const size_t off_packs = off_next + 256;

    fy::ws_acquire(st);
    cudaError_t e;
    if ((e = c.batch.ensure(arena)) != cudaSuccess) return fail_cuda(e, what);
    for (int k = 0; k < K; ++k)
        if ((e = c.bspec[k].ensure(spec_max)) != cudaSuccess) return fail_cuda(e, what);
    unsigned char* A = c.batch.as<unsigned char>();
    std::vector<const float*> in_dec(n);
    std::vector<float*> scr(n);
    std::vector<void*> ctlp(n);
    std::vector<int> dims(3 * (size_t)n);
    for (int i = 0; i < n; ++i) {
        in_dec[i] = reinterpret_cast<float*>(A + off_dec[i]);
        scr[i] = reinterpret_cast<float*>(A + off_scr[i]);
        ctlp[i] = A + off_ctl[i];
        dims[3 * i] = cubes[i].nz; dims[3 * i + 1] = cubes[i].ny; dims[3 * i + 2] = cubes[i].nx;
    }
    BatchGuard guard;
    cudaError_t re = cudaSuccess;
    guard.nb = fy_noise_batch_record(in_dec.data(), dims.data(), scr.data(), ctlp.data(), n, win, pct,
                                     cfg->noise_ref_intensity, c.sms, &re);
    if (!guard.nb) return fail_cuda(re, what);
    const size_t up_bytes = off_packs + fy_noise_batch_bytes(guard.nb);
    if ((e = c.batch_up.ensure(up_bytes)) != cudaSuccess) return fail_cuda(e, what);
    // the staging buffer is rewritten only once the previous batch's upload has been read
    if (c.batch_pending && (e = cudaEventSynchronize(c.batch_done)) != cudaSuccess) return fail_cuda(e, what);
    c.batch_pending = false;
    if ((e = c.batch_pin.ensure(up_bytes)) != cudaSuccess) return fail_cuda(e, what);
    unsigned char* H = (unsigned char*)c.batch_pin.p;
    unsigned char* D = c.batch_up.as<unsigned char>();
    memset(H, 0, off_packs);                              // the queue counters start at 0
    const size_t lut_bytes = ((FY_LUT_N + 1) * sizeof(float) + 15) & ~(size_t)15;
    fyzb::BoxJob* js = reinterpret_cast<fyzb::BoxJob*>(H + off_jobs_s);
    fyzb::BoxJob* jg = reinterpret_cast<fyzb::BoxJob*>(H + off_jobs_g);
    long long total_s = 0, total_g = 0;
    {   // the volumes' tables (FP64 weights: ~0.1 ms each) on the host cores, one volume at a time each
        std::atomic<int> nexti{0};
        auto fill = [&]() {
            for (int i = nexti++; i < n; i = nexti++)
                dl[i].us = fy_deconv_fill_tables(dl[i].g, &cubes[i].phys, params[i], cfg->deconv_kind, fz2ss[i],
                                                 H + off_tab[i]);
        };
        const unsigned hw = std::thread::hardware_concurrency();
        const int nth = std::min(std::min(n, 16), (int)(hw > 1 ? hw : 1)) - 1;
        std::vector<std::thread> th;
        for (int k = 0; k < nth; ++k) th.emplace_back(fill);
        fill();
        for (auto& x : th) x.join();
    }
    for (int i = 0; i < n; ++i) {
        const fy_batch_cube& q = cubes[i];
        DeconvLaunch& d = dl[i];
        unsigned char* tb = D + off_tab[i];
        d.lut = reinterpret_cast<const float*>(tb);
        d.fz2 = reinterpret_cast<const double*>(tb + lut_bytes);
        d.fy2 = d.fz2 + d.g.pz;
        d.fx2 = d.fy2 + d.g.py;
        d.src = q.u8;
        d.src_u8 = 1;
        d.dst = reinterpret_cast<float*>(A + off_dec[i]);
        d.spec = c.bspec[i % K].as<float2>();
        float* mv = reinterpret_cast<float*>(A + off_mv[i]);
        const fyzb::Params ps = fy_noise_stats_params(d.dst, q.nz, q.ny, q.nx, win, scr[i], mv);
        long long items = fyzb::make_job<fyzb::ZB_NOISE>(js[i], ps, win / 2, c.sms, total_s);
        if (items < 0) return fail(FY_ECUDA, "%s: volume %d: tensor map", what, i);
        total_s += items;
        fyzb::Params pg{};
        pg.nz = q.nz; pg.ny = q.ny; pg.nx = q.nx;
        pg.f0 = mv; pg.guide = d.dst; pg.o0 = q.out; pg.out_mode = 0; pg.eps = 0.f;
        pg.eps_ptr = fy_noise_eps_ptr(ctlp[i]);
        items = fyzb::make_job<fyzb::ZB_GUIDED_OUT_MV>(jg[i], pg, radius, c.sms, total_g);
        if (items < 0) return fail(FY_ECUDA, "%s: volume %d: tensor map", what, i);
        total_g += items;
    }
    fy_noise_batch_pack(guard.nb, H + off_packs);
    if ((e = cudaMemcpyAsync(D, H, up_bytes, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaEventRecord(c.batch_done, st)) != cudaSuccess)
        return fail_cuda(e, what);
    c.batch_pending = true;
    // ---- 1. deconvolutions on the batch streams
    if ((e = cudaEventRecord(c.bfork, st)) != cudaSuccess) return fail_cuda(e, what);
    for (int k = 0; k < K; ++k)
        if ((e = cudaStreamWaitEvent(c.bst[k], c.bfork, 0)) != cudaSuccess) return fail_cuda(e, what);
    for (int i = 0; i < n && e == cudaSuccess; ++i) e = fy_launch_deconv(dl[i], c.bst[i % K]);
    for (int k = 0; k < K && e == cudaSuccess; ++k)
        if ((e = cudaEventRecord(c.bev[k], c.bst[k])) == cudaSuccess) e = cudaStreamWaitEvent(st, c.bev[k], 0);
    // ---- 2. noise statistics, 3. selection, 4. guided output
    unsigned long long* next = reinterpret_cast<unsigned long long*>(D + off_next);
    if (e == cudaSuccess)
        e = fyzb::launch_queue<fyzb::ZB_NOISE>(reinterpret_cast<const fyzb::BoxJob*>(D + off_jobs_s), n, total_s,
                                               next, win / 2, c.sms, st);
    if (e == cudaSuccess) e = fy_noise_batch_launch(guard.nb, D + off_packs, st);
    if (e == cudaSuccess)
        e = fyzb::launch_queue<fyzb::ZB_GUIDED_OUT_MV>(reinterpret_cast<const fyzb::BoxJob*>(D + off_jobs_g), n,
                                                       total_g, next + 1, radius, c.sms, st);
    if (e != cudaSuccess) return fail_cuda(e, what);
    fy::count_launch(5 * n + 2 + fy_noise_batch_steps(guard.nb));
    fy::ws_release(st);
    return FY_OK;
}
