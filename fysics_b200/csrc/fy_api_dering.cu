// fy_api_dering.cu -- C-ABI ring removal (dering.c) and the fy_gpu_dering device handle.
//
// fy_dering keeps the reference's host layout (fysics.h:406-415): callers read ring[] and
// have_rings directly and may fwrite the struct's arrays. Bookkeeping on those small host
// arrays (init, tile copies, merge) stays on the host exactly as in dering.c:31-73,119-123;
// the per-voxel work (accumulate, apply) and the vote run on the GPU.
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <vector>

#include "fy_context.h"

using fy::ctx;
using fy::fail;
using fy::fail_cuda;

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

namespace {

// (y,x) -> sector*nr + radius of the ss-subsampled grid, -1 out of range (dering.c:86-99).
// Host double math with the same expressions as the reference, so sectors on exact
// boundaries (diagonals) resolve identically; sqrt argument contracted to one FMA as the
// reference's FMA-enabled build does.
std::vector<int> build_map(double cy, double cx, long y0, long x0, long dy, long dx, int ss, int ns, int nr) {
    const long sy = (dy + ss - 1) / ss, sx = (dx + ss - 1) / ss;
    std::vector<int> m((size_t)sy * sx);
    const double inv_sect = ns / (2.0 * M_PI);
    for (long yi = 0; yi < sy; yi++) {
        const double gy = (double)(y0 + yi * ss) - cy, gy2 = gy * gy;
        for (long xi = 0; xi < sx; xi++) {
            const double gx = (double)(x0 + xi * ss) - cx;
            const int ri = (int)(sqrt(fma(gx, gx, gy2)) + 0.5);
            if (ri >= nr) { m[(size_t)yi * sx + xi] = -1; continue; }
            int q = (int)((atan2(gy, gx) + M_PI) * inv_sect);
            if (q >= ns) q = ns - 1;
            m[(size_t)yi * sx + xi] = q * nr + ri;
        }
    }
    return m;
}

struct MapCache {
    double cy = 0, cx = 0;
    long y0 = 0, x0 = 0, dy = 0, dx = 0;
    int ss = 0, ns = 0, nr = 0;
    bool valid = false;
    fy::DevBuf buf;
    bool same(double a, double b, long c, long d, long e, long f, int g, int h, int i) const {
        return valid && cy == a && cx == b && y0 == c && x0 == d && dy == e && dx == f && ss == g && ns == h && nr == i;
    }
};
thread_local MapCache t_map;

int ensure_map(double cy, double cx, long y0, long x0, long dy, long dx, int ss, int ns, int nr,
               cudaStream_t st, const int** out) {
    MapCache& mc = t_map;
    if (!mc.same(cy, cx, y0, x0, dy, dx, ss, ns, nr)) {
        std::vector<int> m = build_map(cy, cx, y0, x0, dy, dx, ss, ns, nr);
        cudaError_t e = mc.buf.ensure(m.size() * sizeof(int));
        if (e != cudaSuccess) return fail_cuda(e, "dering map");
        if ((e = cudaMemcpyAsync(mc.buf.p, m.data(), m.size() * sizeof(int), cudaMemcpyHostToDevice, st)) != cudaSuccess)
            return fail_cuda(e, "dering map upload");
        mc.cy = cy; mc.cx = cx; mc.y0 = y0; mc.x0 = x0; mc.dy = dy; mc.dx = dx;
        mc.ss = ss; mc.ns = ns; mc.nr = nr; mc.valid = true;
    }
    *out = mc.buf.as<int>();
    return FY_OK;
}

void finalize_defaults(int& hp_win, double& min_amp, double& max_amp) {
    if (hp_win < 3) hp_win = 15;                       // dering.c:138-140
    if (min_amp <= 0) min_amp = 0.5;
    if (max_amp <= 0) max_amp = 6.0;
}
}  // namespace

// ---------------------------------------------------------------- host-struct API
extern "C" int fy_dering_init(fy_dering* d, long Z, long Y, long X, double cy, double cx, int slab_z, int ns) {
    fy::enter();
    memset(d, 0, sizeof(*d));                          // dering.c:31-49
    d->Z = Z; d->Y = Y; d->X = X;
    d->cy = cy >= 0 ? cy : (Y - 1) / 2.0;
    d->cx = cx >= 0 ? cx : (X - 1) / 2.0;
    d->slab_z = slab_z > 0 ? slab_z : 512;
    d->nslab = (int)((Z + d->slab_z - 1) / d->slab_z);
    d->ns = ns > 0 ? ns : 8;
    if (d->ns > 64) return fail(FY_EUNSUPPORTED, "fy_dering_init: ns %d > 64", d->ns);
    const double ry = d->cy > Y - 1 - d->cy ? d->cy : Y - 1 - d->cy;
    const double rx = d->cx > X - 1 - d->cx ? d->cx : X - 1 - d->cx;
    d->nr = (int)(sqrt(ry * ry + rx * rx)) + 2;
    const size_t nb = (size_t)d->nslab * d->ns * d->nr;
    d->sum = (float*)calloc(nb, sizeof(float));
    d->cnt = (unsigned int*)calloc(nb, sizeof(unsigned int));
    d->ring = (float*)calloc((size_t)d->nslab * d->nr, sizeof(float));
    if (!d->sum || !d->cnt || !d->ring) {
        free(d->sum); free(d->cnt); free(d->ring);
        d->sum = nullptr; d->cnt = nullptr; d->ring = nullptr;
        return fail(FY_ENOMEM, "fy_dering_init: allocation failed");
    }
    return FY_OK;
}

extern "C" void fy_dering_free(fy_dering* d) {
    free(d->sum); free(d->cnt); free(d->ring);
    d->sum = nullptr; d->cnt = nullptr; d->ring = nullptr;
}

extern "C" int fy_dering_tile_init(fy_dering* t, const fy_dering* d) {
    fy::enter();
    *t = *d;                                           // dering.c:58-67
    t->nslab = 1;
    const size_t nb = (size_t)t->ns * t->nr;
    t->sum = (float*)calloc(nb, sizeof(float));
    t->cnt = (unsigned int*)calloc(nb, sizeof(unsigned int));
    t->ring = nullptr;
    if (!t->sum || !t->cnt) {
        free(t->sum); free(t->cnt);
        return fail(FY_ENOMEM, "fy_dering_tile_init: allocation failed");
    }
    return FY_OK;
}

extern "C" void fy_dering_tile_reset(fy_dering* t) {
    const size_t nb = (size_t)t->ns * t->nr;
    memset(t->sum, 0, nb * sizeof(float));
    memset(t->cnt, 0, nb * sizeof(unsigned int));
}

extern "C" void fy_dering_merge_tile(fy_dering* d, int slab, const fy_dering* t) {
    if (slab < 0 || slab >= d->nslab) return;          // dering.c:119-123
    const size_t nb = (size_t)d->ns * d->nr, off = (size_t)slab * nb;
    for (size_t i = 0; i < nb; i++) { d->sum[off + i] += t->sum[i]; d->cnt[off + i] += t->cnt[i]; }
}

// GPU accumulate of one u8 region into the single-slab state t (dering.c:78-116). The
// exact integer bin totals are added to t's float sums: identical to the reference's
// one-sample-at-a-time float accumulation while a bin stays below 2^24.
extern "C" void fy_dering_accumulate_u8(fy_dering* t, const unsigned char* buf, long y0, long x0, long dz,
                                        long dy, long dx, int ss) {
    fy::enter();
    const char* what = "fy_dering_accumulate_u8";
    if (ss < 1) ss = 1;
    if (!t || !buf || !t->sum || !t->cnt) { fail(FY_EINVAL, "%s: null pointer", what); return; }
    if (dz <= 0 || dy <= 0 || dx <= 0) return;
    if (fy::ensure_ctx()) return;
    fy::ThreadCtx& c = ctx();
    cudaStream_t st = c.st;
    const int nbins = t->ns * t->nr;
    const size_t nbytes = (size_t)dz * dy * dx;
    fy::ws_acquire(st);
    cudaError_t e;
    const int* map = nullptr;
    if (ensure_map(t->cy, t->cx, y0, x0, dy, dx, ss, t->ns, t->nr, st, &map)) return;
    if ((e = c.vin.ensure(nbytes)) != cudaSuccess) { fail_cuda(e, what); return; }
    const size_t acc_bytes = (size_t)nbins * (sizeof(unsigned long long) + sizeof(unsigned int));
    if ((e = c.small.ensure(acc_bytes)) != cudaSuccess) { fail_cuda(e, what); return; }
    if ((e = c.pin.ensure(acc_bytes)) != cudaSuccess) { fail_cuda(e, what); return; }
    unsigned long long* dsum = c.small.as<unsigned long long>();
    unsigned int* dcnt = (unsigned int*)(dsum + nbins);
    if ((e = cudaMemsetAsync(dsum, 0, acc_bytes, st)) != cudaSuccess) { fail_cuda(e, what); return; }
    if ((e = cudaMemcpyAsync(c.vin.p, buf, nbytes, cudaMemcpyHostToDevice, st)) != cudaSuccess) { fail_cuda(e, what); return; }
    if ((e = fy_launch_dering_accum(c.vin.as<uint8_t>(), map, dsum, dcnt, nbins, dz, dy, dx, ss, c.sms, st)) != cudaSuccess) {
        fail_cuda(e, what); return;
    }
    fy::count_launch();
    if ((e = cudaMemcpyAsync(c.pin.p, dsum, acc_bytes, cudaMemcpyDeviceToHost, st)) != cudaSuccess) { fail_cuda(e, what); return; }
    fy::ws_release(st);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) { fail_cuda(e, what); return; }
    const unsigned long long* hs = (const unsigned long long*)c.pin.p;
    const unsigned int* hc = (const unsigned int*)(hs + nbins);
    for (int b = 0; b < nbins; ++b) {
        if (hc[b]) { t->sum[b] += (float)hs[b]; t->cnt[b] += hc[b]; }
    }
}

extern "C" long fy_dering_finalize(fy_dering* d, int hp_win, unsigned int min_cnt, double min_amp,
                                   double max_amp) {
    fy::enter();
    const char* what = "fy_dering_finalize";
    finalize_defaults(hp_win, min_amp, max_amp);
    if (!d || !d->sum || !d->cnt || !d->ring) { fail(FY_EINVAL, "%s: uninitialised state", what); return 0; }
    if (fy::ensure_ctx()) return 0;
    fy::ThreadCtx& c = ctx();
    cudaStream_t st = c.st;
    const size_t nb = (size_t)d->nslab * d->ns * d->nr, nring = (size_t)d->nslab * d->nr;
    fy::ws_acquire(st);
    cudaError_t e;
    // device layout: sum_f | cnt | ring | detected(u64) | have(int) | scratch
    const size_t off_cnt = nb * 4, off_ring = off_cnt + nb * 4, off_det = ((off_ring + nring * 4 + 15) / 16) * 16;
    const size_t off_scr = off_det + 16, total = off_scr + fy_dering_finalize_scratch(d->nslab, d->ns, d->nr);
    if ((e = c.aux.ensure(total)) != cudaSuccess) { fail_cuda(e, what); return 0; }
    char* base = (char*)c.aux.p;
    if ((e = cudaMemcpyAsync(base, d->sum, nb * 4, cudaMemcpyHostToDevice, st)) != cudaSuccess) { fail_cuda(e, what); return 0; }
    if ((e = cudaMemcpyAsync(base + off_cnt, d->cnt, nb * 4, cudaMemcpyHostToDevice, st)) != cudaSuccess) { fail_cuda(e, what); return 0; }
    if ((e = fy_launch_dering_finalize((const float*)base, (const unsigned int*)(base + off_cnt), (float*)(base + off_ring),
                                       base + off_scr, (unsigned long long*)(base + off_det), (int*)(base + off_det + 8),
                                       d->nslab, d->ns, d->nr, hp_win, min_cnt, min_amp, max_amp, st)) != cudaSuccess) {
        fail_cuda(e, what); return 0;
    }
    fy::count_launch(3);
    if ((e = c.pin.ensure(16)) != cudaSuccess) { fail_cuda(e, what); return 0; }
    if ((e = cudaMemcpyAsync(d->ring, base + off_ring, nring * 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess) { fail_cuda(e, what); return 0; }
    if ((e = cudaMemcpyAsync(c.pin.p, base + off_det, 16, cudaMemcpyDeviceToHost, st)) != cudaSuccess) { fail_cuda(e, what); return 0; }
    fy::ws_release(st);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) { fail_cuda(e, what); return 0; }
    const long det = (long)*(const unsigned long long*)c.pin.p;
    d->have_rings = det >= 2;
    return det;
}

extern "C" void fy_dering_apply(const fy_dering* d, float* f, long z0, long y0, long x0, long dz, long dy, long dx,
                                double scale) {
    fy::enter();
    const char* what = "fy_dering_apply";
    if (!d || !d->have_rings) return;                  // dering.c:202
    if (!f || !d->ring) { fail(FY_EINVAL, "%s: null pointer", what); return; }
    if (dz <= 0 || dy <= 0 || dx <= 0) return;
    if (dy > 65535) { fail(FY_EUNSUPPORTED, "%s: dy %ld > 65535", what, dy); return; }
    if (fy::ensure_ctx()) return;
    fy::ThreadCtx& c = ctx();
    cudaStream_t st = c.st;
    const size_t n = (size_t)dz * dy * dx, nring = (size_t)d->nslab * d->nr;
    fy::ws_acquire(st);
    cudaError_t e;
    if ((e = c.vin.ensure(n * 4)) != cudaSuccess) { fail_cuda(e, what); return; }
    if ((e = c.small.ensure(nring * 4)) != cudaSuccess) { fail_cuda(e, what); return; }
    if ((e = cudaMemcpyAsync(c.vin.p, f, n * 4, cudaMemcpyHostToDevice, st)) != cudaSuccess) { fail_cuda(e, what); return; }
    if ((e = cudaMemcpyAsync(c.small.p, d->ring, nring * 4, cudaMemcpyHostToDevice, st)) != cudaSuccess) { fail_cuda(e, what); return; }
    if ((e = fy_launch_dering_apply(c.vin.as<float>(), c.small.as<float>(), nullptr, d->nslab, d->nr, d->slab_z, d->cy,
                                    d->cx, z0, y0, x0, dz, dy, dx, scale, st)) != cudaSuccess) { fail_cuda(e, what); return; }
    fy::count_launch();
    if ((e = cudaMemcpyAsync(f, c.vin.p, n * 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess) { fail_cuda(e, what); return; }
    fy::ws_release(st);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) fail_cuda(e, what);
}

// ---------------------------------------------------------------- device handle
struct fy_gpu_dering {
    fy_dering geo;                  // geometry (sum/cnt/ring unused on the host side)
    int dev;
    unsigned long long* dsum;       // [nslab][ns][nr] exact sums
    unsigned int* dcnt;
    float* dsumf;                   // float view for the finalize (exact < 2^24)
    float* dring;                   // [nslab][nr]
    unsigned long long* ddet;
    int* dhave;
    void* dscr;
};

namespace {
__global__ void k_u64_to_f32(const unsigned long long* s, float* f, size_t n) {
    fy_pdl_wait();
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        f[i] = (float)s[i];
}
}  // namespace

extern "C" int fy_gpu_dering_create(fy_gpu_dering** out, long Z, long Y, long X, double cy, double cx, int slab_z,
                                    int ns) {
    fy::enter();
    if (!out) return fail(FY_EINVAL, "fy_gpu_dering_create: null handle");
    int rc = fy::ensure_ctx();
    if (rc) return rc;
    fy_gpu_dering* h = (fy_gpu_dering*)calloc(1, sizeof(fy_gpu_dering));
    if (!h) return fail(FY_ENOMEM, "fy_gpu_dering_create");
    if ((rc = fy_dering_init(&h->geo, Z, Y, X, cy, cx, slab_z, ns))) { free(h); return rc; }
    fy_dering_free(&h->geo);                          // geometry only on the host
    h->dev = ctx().dev;
    const size_t nb = (size_t)h->geo.nslab * h->geo.ns * h->geo.nr, nring = (size_t)h->geo.nslab * h->geo.nr;
    cudaError_t e = cudaSuccess;
    if ((e = cudaMalloc(&h->dsum, nb * 8)) || (e = cudaMalloc(&h->dcnt, nb * 4)) || (e = cudaMalloc(&h->dsumf, nb * 4)) ||
        (e = cudaMalloc(&h->dring, nring * 4)) || (e = cudaMalloc(&h->ddet, 16)) ||
        (e = cudaMalloc(&h->dscr, fy_dering_finalize_scratch(h->geo.nslab, h->geo.ns, h->geo.nr)))) {
        cudaFree(h->dsum); cudaFree(h->dcnt); cudaFree(h->dsumf); cudaFree(h->dring); cudaFree(h->ddet); cudaFree(h->dscr);
        free(h);
        return fail_cuda(e, "fy_gpu_dering_create");
    }
    h->dhave = (int*)(h->ddet + 1);
    cudaMemset(h->dsum, 0, nb * 8);
    cudaMemset(h->dcnt, 0, nb * 4);
    cudaMemset(h->dring, 0, nring * 4);
    cudaMemset(h->ddet, 0, 16);
    if ((e = cudaDeviceSynchronize()) != cudaSuccess) return fail_cuda(e, "fy_gpu_dering_create");
    *out = h;
    return FY_OK;
}

extern "C" void fy_gpu_dering_destroy(fy_gpu_dering* h) {
    if (!h) return;
    cudaFree(h->dsum); cudaFree(h->dcnt); cudaFree(h->dsumf); cudaFree(h->dring); cudaFree(h->ddet); cudaFree(h->dscr);
    free(h);
}

extern "C" int fy_gpu_dering_reset(fy_gpu_dering* h, void* stream) {
    fy::enter();
    if (!h) return fail(FY_EINVAL, "fy_gpu_dering_reset: null handle");
    const size_t nb = (size_t)h->geo.nslab * h->geo.ns * h->geo.nr;
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e;
    if ((e = cudaMemsetAsync(h->dsum, 0, nb * 8, st)) || (e = cudaMemsetAsync(h->dcnt, 0, nb * 4, st)) ||
        (e = cudaMemsetAsync(h->ddet, 0, 16, st)))
        return fail_cuda(e, "fy_gpu_dering_reset");
    return FY_OK;
}

// Accumulate a device u8 region at global (z0,y0,x0) into slab z0/slab_z (the pipeline's
// accumulate + merge, pipeline.c:680-685, fused).
extern "C" int fy_gpu_dering_accumulate_u8(fy_gpu_dering* h, const unsigned char* d_buf, long z0, long y0, long x0,
                                           long dz, long dy, long dx, int ss, void* stream) {
    fy::enter();
    const char* what = "fy_gpu_dering_accumulate_u8";
    if (!h || !d_buf) return fail(FY_EINVAL, "%s: null pointer", what);
    if (ss < 1) ss = 1;
    int rc = fy::ensure_ctx();
    if (rc) return rc;
    long slab = z0 / h->geo.slab_z;
    if (slab < 0 || slab >= h->geo.nslab) return fail(FY_EINVAL, "%s: z0 %ld outside the volume", what, z0);
    cudaStream_t st = (cudaStream_t)stream;
    const int* map = nullptr;
    if ((rc = ensure_map(h->geo.cy, h->geo.cx, y0, x0, dy, dx, ss, h->geo.ns, h->geo.nr, st, &map))) return rc;
    const size_t nb = (size_t)h->geo.ns * h->geo.nr;
    cudaError_t e = fy_launch_dering_accum(d_buf, map, h->dsum + slab * nb, h->dcnt + slab * nb, (int)nb, dz, dy, dx,
                                           ss, ctx().sms, st);
    if (e != cudaSuccess) return fail_cuda(e, what);
    fy::count_launch();
    return FY_OK;
}

extern "C" int fy_gpu_dering_finalize(fy_gpu_dering* h, int hp_win, unsigned int min_cnt, double min_amp,
                                      double max_amp, void* stream) {
    fy::enter();
    if (!h) return fail(FY_EINVAL, "fy_gpu_dering_finalize: null handle");
    finalize_defaults(hp_win, min_amp, max_amp);
    cudaStream_t st = (cudaStream_t)stream;
    const size_t nb = (size_t)h->geo.nslab * h->geo.ns * h->geo.nr;
    cudaError_t e = fy_launch_pdl(k_u64_to_f32, dim3((unsigned)((nb + 255) / 256 < 1024 ? (nb + 255) / 256 : 1024)),
                                  dim3(256), 0, st, (const unsigned long long*)h->dsum, h->dsumf, nb);
    if (e != cudaSuccess) return fail_cuda(e, "fy_gpu_dering_finalize");
    e = fy_launch_dering_finalize(h->dsumf, h->dcnt, h->dring, h->dscr, h->ddet, h->dhave, h->geo.nslab,
                                              h->geo.ns, h->geo.nr, hp_win, min_cnt, min_amp, max_amp, st);
    if (e != cudaSuccess) return fail_cuda(e, "fy_gpu_dering_finalize");
    fy::count_launch(4);
    return FY_OK;
}

void fy_dering_ring_args(const fy_gpu_dering* h, long z0, long y0, long x0, double scale, RingApply* ra) {
    ra->ring = h->dring;
    ra->have = h->dhave;
    ra->nslab = h->geo.nslab;
    ra->nr = h->geo.nr;
    ra->slab_z = h->geo.slab_z;
    ra->cy = h->geo.cy;
    ra->cx = h->geo.cx;
    ra->z0 = z0; ra->y0 = y0; ra->x0 = x0;
    ra->sc = (float)scale;
}

extern "C" int fy_gpu_dering_apply(const fy_gpu_dering* h, float* d_f, long z0, long y0, long x0, long dz, long dy,
                                   long dx, double scale, void* stream) {
    fy::enter();
    if (!h || !d_f) return fail(FY_EINVAL, "fy_gpu_dering_apply: null pointer");
    if (dy > 65535) return fail(FY_EUNSUPPORTED, "fy_gpu_dering_apply: dy > 65535");
    cudaError_t e = fy_launch_dering_apply(d_f, h->dring, h->dhave, h->geo.nslab, h->geo.nr, h->geo.slab_z, h->geo.cy,
                                           h->geo.cx, z0, y0, x0, dz, dy, dx, scale, (cudaStream_t)stream);
    if (e != cudaSuccess) return fail_cuda(e, "fy_gpu_dering_apply");
    fy::count_launch();
    return FY_OK;
}

// Copy the device state into a host fy_dering initialised with the same geometry
// (sum as float, cnt, ring, have_rings); returns the detected count through *detected.
extern "C" int fy_gpu_dering_download(const fy_gpu_dering* h, fy_dering* d, long* detected, void* stream) {
    fy::enter();
    if (!h || !d || !d->sum || !d->cnt || !d->ring) return fail(FY_EINVAL, "fy_gpu_dering_download: null pointer");
    if (d->nslab != h->geo.nslab || d->ns != h->geo.ns || d->nr != h->geo.nr)
        return fail(FY_EINVAL, "fy_gpu_dering_download: geometry mismatch");
    cudaStream_t st = (cudaStream_t)stream;
    const size_t nb = (size_t)h->geo.nslab * h->geo.ns * h->geo.nr, nring = (size_t)h->geo.nslab * h->geo.nr;
    std::vector<unsigned long long> s(nb);
    unsigned long long det[2] = {0, 0};
    cudaError_t e;
    if ((e = cudaMemcpyAsync(s.data(), h->dsum, nb * 8, cudaMemcpyDeviceToHost, st)) ||
        (e = cudaMemcpyAsync(d->cnt, h->dcnt, nb * 4, cudaMemcpyDeviceToHost, st)) ||
        (e = cudaMemcpyAsync(d->ring, h->dring, nring * 4, cudaMemcpyDeviceToHost, st)) ||
        (e = cudaMemcpyAsync(det, h->ddet, 16, cudaMemcpyDeviceToHost, st)) || (e = cudaStreamSynchronize(st)))
        return fail_cuda(e, "fy_gpu_dering_download");
    for (size_t i = 0; i < nb; ++i) d->sum[i] = (float)s[i];
    d->have_rings = (int)(det[1] & 0xffffffffu);
    if (detected) *detected = (long)det[0];
    return FY_OK;
}
