// fy_calib.cu -- pass-1 calibration statistics on the GPU: the u8 histogram
// (fy_hist_accumulate_u8, stream.c:76-86), the flat-region noise floor (fy_flat_noise,
// stream.c:174-200) and the noise-correlation anisotropy (fy_noise_aniso, noise.c:210-269).
//
//   k_hist_u8       16-byte loads; each warp counts into 4 shared sub-histograms picked by
//                   lane (neighbouring lanes rarely hit the same copy), summed per CTA into
//                   256 global 64-bit counters. Integer counts: identical to the reference.
//   k_block_stats   one warp per block of blk^3 (flat noise) or 8^3 (anisotropy) voxels:
//                   FP64 sums of the values and of their squares, the squares taken in the
//                   reference's precision (a float product for the noise floor, a double
//                   one for the anisotropy); per block an orderable 64-bit key of the
//                   statistic whose order statistic is wanted, or ~0 when the block is out.
//   k_select        one CTA: the k-th smallest key (k from the device count of valid keys)
//                   by eight 8-bit radix passes; every thread counts its keys in a private
//                   column of counters, so no atomics are needed.
//   k_aniso_lags    one warp per flat block: residuals (float, as the reference's in-place
//                   subtraction), their squares and the lag-1 products along z, y, x (FP64);
//                   per-block partial sums.
//   k_aniso_final   one CTA: the partial sums in a fixed order, the ratios and the status.
// The reference's FP64 sums run in its own (vectorised, -Ofast) order; these run as warp
// trees. They agree to a few ulp, and the order statistics pick the same block unless two
// block values are that close.
#include <algorithm>
#include <cstring>

#include "fy_context.h"

using fy::ctx;
using fy::fail;
using fy::fail_cuda;

namespace {

constexpr unsigned long long kOut = ~0ull;    // key of a block that does not take part

FY_D unsigned long long fkey64(float f) {     // orderable key of a float in the low 32 bits
    const uint32_t u = __float_as_uint(f);
    return u ^ ((uint32_t)((int32_t)u >> 31) | 0x80000000u);
}
FY_HD float funkey64(unsigned long long k) {
    const uint32_t kk = (uint32_t)k;
    const uint32_t u = (kk & 0x80000000u) ? (kk & 0x7FFFFFFFu) : ~kk;
    float f;
    memcpy(&f, &u, 4);
    return f;
}

// ---------------------------------------------------------------- histogram
constexpr int kHistThreads = 256, kHistCopies = 4;
__global__ void __launch_bounds__(kHistThreads) k_hist_u8(const uint8_t* __restrict__ d, size_t n,
                                                          unsigned long long* __restrict__ hist) {
    __shared__ unsigned int h[kHistThreads / 32][kHistCopies][256];
    for (int i = threadIdx.x; i < (kHistThreads / 32) * kHistCopies * 256; i += blockDim.x) (&h[0][0][0])[i] = 0;
    __syncthreads();
    unsigned int* mine = h[threadIdx.x >> 5][threadIdx.x & (kHistCopies - 1)];
    const size_t head = ((16 - ((uintptr_t)d & 15)) & 15) < n ? ((16 - ((uintptr_t)d & 15)) & 15) : n;
    const size_t body = (n - head) / 16;
    const size_t gtid = (size_t)blockIdx.x * blockDim.x + threadIdx.x, gstride = (size_t)gridDim.x * blockDim.x;
    if (gtid < head) atomicAdd(&mine[d[gtid]], 1u);
    const uint4* v = reinterpret_cast<const uint4*>(d + head);
    for (size_t q = gtid; q < body; q += gstride) {
        const uint4 w = __ldg(v + q);
        const uint32_t ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            atomicAdd(&mine[ws[j] & 255u], 1u);
            atomicAdd(&mine[(ws[j] >> 8) & 255u], 1u);
            atomicAdd(&mine[(ws[j] >> 16) & 255u], 1u);
            atomicAdd(&mine[ws[j] >> 24], 1u);
        }
    }
    for (size_t i = head + body * 16 + gtid; i < n; i += gstride) atomicAdd(&mine[d[i]], 1u);
    __syncthreads();
    for (int b = threadIdx.x; b < 256; b += blockDim.x) {
        unsigned long long s = 0;
        for (int w = 0; w < kHistThreads / 32; ++w)
            for (int c = 0; c < kHistCopies; ++c) s += h[w][c][b];
        if (s) atomicAdd(&hist[b], s);
    }
}

// ---------------------------------------------------------------- block statistics
FY_D double warp_sum(double v) {
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    return v;
}

// MODE 0 (noise floor): key = bits of sqrt(max(var, 0)) for blocks with mean > 0.1
// (stream.c:181-195). MODE 1 (anisotropy): blocks whose voxels are all > 0 keep their mean
// and variance, key = the variance as a float (noise.c:220-230).
template <int MODE>
__global__ void __launch_bounds__(256) k_block_stats(const float* __restrict__ v, int ny, int nx, int blk,
                                                     int bz, int by, int bx, unsigned long long* __restrict__ key,
                                                     double* __restrict__ bmean, double* __restrict__ bvar,
                                                     unsigned long long* __restrict__ nvalid) {
    const long nb = (long)bz * by * bx;
    const long b = (long)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    if (b >= nb) return;
    const int lane = threadIdx.x & 31;
    const long z0 = (b / ((long)by * bx)) * blk, y0 = ((b / bx) % by) * blk, x0 = (b % bx) * blk;
    const int b3 = blk * blk * blk;
    double s = 0, s2 = 0;
    bool positive = true;
    for (int k = lane; k < b3; k += 32) {
        const int dz = k / (blk * blk), dy = (k / blk) % blk, dx = k % blk;
        const float t = __ldg(v + ((size_t)(z0 + dz) * ny + (y0 + dy)) * nx + (x0 + dx));
        s += t;
        if (MODE == 0) {
            const float t2 = __fmul_rn(t, t);           // the reference's float val*val
            s2 += t2;
        } else {
            s2 += (double)t * t;
            if (t <= 0.f) positive = false;              // noise.c:224 (a NaN voxel does not exclude)
        }
    }
    s = warp_sum(s);
    s2 = warp_sum(s2);
    positive = __all_sync(0xffffffffu, positive);
    if (lane) return;
    const double c = (double)b3, mean = s / c, var = s2 / c - mean * mean;
    unsigned long long k = kOut;
    if (MODE == 0) {
        if (mean > 0.1) k = (unsigned long long)__double_as_longlong(sqrt(var > 0 ? var : 0));
    } else {
        bmean[b] = mean;
        bvar[b] = var;
        if (positive) k = fkey64((float)var);
    }
    key[b] = k;
    if (k != kOut) atomicAdd(nvalid, 1ull);
}

// ---------------------------------------------------------------- k-th smallest key
// One CTA of kSelThreads threads over n keys; k = nvalid / div (the reference's index m/10
// or nv/5). Keys equal to kOut sort last and are never selected (k < nvalid). Dynamic
// shared memory: 256 digits x kSelThreads private 32-bit counters.
constexpr int kSelThreads = 128;
__global__ void __launch_bounds__(kSelThreads) k_select(const unsigned long long* __restrict__ key, long n,
                                                        const unsigned long long* __restrict__ nvalid, int div,
                                                        unsigned long long* __restrict__ out) {
    extern __shared__ unsigned int cnt[];              // [digit][thread]
    __shared__ unsigned long long part[256];
    __shared__ unsigned long long s_sel[2];
    const int t = threadIdx.x;
    const unsigned long long m = *nvalid;
    if (m == 0) {
        if (t == 0) *out = kOut;
        return;
    }
    unsigned long long rank = m / div, prefix = 0, pmask = 0;
    for (int sh = 56; sh >= 0; sh -= 8) {
        for (int i = t; i < 256 * kSelThreads; i += kSelThreads) cnt[i] = 0;
        __syncthreads();
        for (long i = t; i < n; i += kSelThreads) {
            const unsigned long long k = key[i];
            if ((k & pmask) == prefix) ++cnt[((k >> sh) & 255u) * kSelThreads + t];
        }
        __syncthreads();
        for (int d = t; d < 256; d += kSelThreads) {
            unsigned long long s = 0;
            for (int j = 0; j < kSelThreads; ++j) s += cnt[d * kSelThreads + ((j + d) & (kSelThreads - 1))];
            part[d] = s;
        }
        __syncthreads();
        if (t == 0) {                                    // 256 digits: a short serial scan
            unsigned long long acc = 0;
            for (int d = 0; d < 256; ++d) {
                if (rank < acc + part[d]) { s_sel[0] = (unsigned long long)d; s_sel[1] = rank - acc; break; }
                acc += part[d];
            }
        }
        __syncthreads();
        prefix |= s_sel[0] << sh;
        pmask |= 255ull << sh;
        rank = s_sel[1];
        __syncthreads();
    }
    if (t == 0) *out = prefix;
}

__global__ void k_floor_out(const unsigned long long* __restrict__ sel, double* __restrict__ out) {
    *out = *sel == kOut ? 0.0 : __longlong_as_double((long long)*sel);      // 0 without bright blocks
}

// ---------------------------------------------------------------- anisotropy lag sums
// One warp per 8^3 block; lane l owns rows (dz, dy) = l and l + 32 of the block (8 voxels
// each), staged in shared memory for the neighbours' products.
__global__ void __launch_bounds__(256) k_aniso_lags(const float* __restrict__ v, int ny, int nx, int bz, int by,
                                                    int bx, const unsigned long long* __restrict__ key,
                                                    const double* __restrict__ bvar,
                                                    const double* __restrict__ bmean,
                                                    const unsigned long long* __restrict__ thresh_key,
                                                    double4* __restrict__ part, int* __restrict__ used) {
    __shared__ float r[256 / 32][512];
    const long nb = (long)bz * by * bx;
    const long b = (long)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    if (b >= nb) return;
    const int lane = threadIdx.x & 31;
    const float thresh = funkey64(*thresh_key);
    // noise.c:245: only blocks whose voxels are all > 0 and whose variance <= threshold
    const bool flat = key[b] != kOut && !(bvar[b] > (double)thresh);
    if (!flat) {
        if (lane == 0) { part[b] = make_double4(0, 0, 0, 0); used[b] = 0; }
        return;
    }
    float* rb = r[threadIdx.x >> 5];
    const float fm = (float)bmean[b];
    const long z0 = (b / ((long)by * bx)) * 8, y0 = ((b / bx) % by) * 8, x0 = (b % bx) * 8;
    for (int q = 0; q < 2; ++q) {
        const int row = lane + 32 * q, dz = row >> 3, dy = row & 7;
        const float* src = v + ((size_t)(z0 + dz) * ny + (y0 + dy)) * nx + x0;
#pragma unroll
        for (int dx = 0; dx < 8; ++dx) rb[row * 8 + dx] = __fsub_rn(__ldg(src + dx), fm);
    }
    __syncwarp();
    double den = 0, lz = 0, ly = 0, lx = 0;
    for (int q = 0; q < 2; ++q) {
        const int row = lane + 32 * q, dz = row >> 3, dy = row & 7;
#pragma unroll
        for (int dx = 0; dx < 8; ++dx) {
            const int i = row * 8 + dx;
            const double c = rb[i];
            den += c * c;
            if (dz + 1 < 8) lz += c * (double)rb[i + 64];
            if (dy + 1 < 8) ly += c * (double)rb[i + 8];
            if (dx + 1 < 8) lx += c * (double)rb[i + 1];
        }
    }
    den = warp_sum(den);
    lz = warp_sum(lz);
    ly = warp_sum(ly);
    lx = warp_sum(lx);
    if (lane == 0) { part[b] = make_double4(den, lz, ly, lx); used[b] = 1; }
}

// One CTA: the block partials summed in a fixed order (each thread a contiguous run, then
// a fixed tree), rho = 8/7 * lag / den (noise.c:262-268), status 1 for too few non-zero or
// flat blocks or a zero denominator.
struct AnisoOut { double rho_z, rho_xy; int status; };
__global__ void __launch_bounds__(256) k_aniso_final(const double4* __restrict__ part, const int* __restrict__ used,
                                                     long nb, const unsigned long long* __restrict__ nvalid,
                                                     AnisoOut* __restrict__ out) {
    __shared__ double sd[4][256];
    __shared__ long long su[256];
    const int t = threadIdx.x;
    const long per = (nb + 255) / 256, i0 = t * per, i1 = i0 + per < nb ? i0 + per : nb;
    double a0 = 0, a1 = 0, a2 = 0, a3 = 0;
    long long u = 0;
    for (long i = i0; i < i1; ++i) {
        if (!used[i]) continue;
        const double4 p = part[i];
        a0 += p.x; a1 += p.y; a2 += p.z; a3 += p.w;
        ++u;
    }
    sd[0][t] = a0; sd[1][t] = a1; sd[2][t] = a2; sd[3][t] = a3; su[t] = u;
    __syncthreads();
    for (int off = 128; off > 0; off >>= 1) {
        if (t < off) {
            for (int j = 0; j < 4; ++j) sd[j][t] += sd[j][t + off];
            su[t] += su[t + off];
        }
        __syncthreads();
    }
    if (t == 0) {
        const double den = sd[0][0];
        AnisoOut o{0.0, 0.0, 1};
        if (*nvalid >= 64 && su[0] >= 32 && den > 0) {
            const double corr = 8.0 / 7.0;
            o.rho_z = corr * sd[1][0] / den;
            o.rho_xy = corr * 0.5 * (sd[2][0] + sd[3][0]) / den;
            o.status = 0;
        }
        *out = o;
    }
}

unsigned blocks_for(long nwarps) { return (unsigned)((nwarps + 7) / 8); }
size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// Scratch layout: valid count and selected key (256 B), keys, block means, variances, lag
// partials, used flags.
struct CalibLayout {
    size_t keys, mean, var, part, used, total;
};
CalibLayout calib_layout(long nb) {
    CalibLayout L;
    L.keys = 256;
    L.mean = L.keys + align256(nb * sizeof(unsigned long long));
    L.var = L.mean + align256(nb * sizeof(double));
    L.part = L.var + align256(nb * sizeof(double));
    L.used = L.part + align256(nb * sizeof(double4));
    L.total = L.used + align256(nb * sizeof(int));
    return L;
}
long nblocks(int nz, int ny, int nx, int blk) { return (long)(nz / blk) * (ny / blk) * (nx / blk); }

// Enqueue the noise floor of d_v (blk >= 4) into d_out (one double).
cudaError_t launch_flat_noise(const float* d_v, int nz, int ny, int nx, int blk, double* d_out, void* scratch,
                              cudaStream_t st, int& launches) {
    const long nb = nblocks(nz, ny, nx, blk);
    if (nb <= 0) return cudaMemsetAsync(d_out, 0, sizeof(double), st);      // stream.c:176: 0.0
    char* base = (char*)scratch;
    unsigned long long* nvalid = (unsigned long long*)base;
    unsigned long long* sel = nvalid + 1;
    const CalibLayout L = calib_layout(nb);
    unsigned long long* key = (unsigned long long*)(base + L.keys);
    cudaError_t e = cudaMemsetAsync(nvalid, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
    k_block_stats<0><<<blocks_for(nb), 256, 0, st>>>(d_v, ny, nx, blk, nz / blk, ny / blk, nx / blk, key, nullptr,
                                                     nullptr, nvalid);
    const size_t smem = 256 * kSelThreads * sizeof(unsigned int);
    if ((e = fy_smem_optin(k_select, smem)) != cudaSuccess) return e;
    k_select<<<1, kSelThreads, smem, st>>>(key, nb, nvalid, 10, sel);           // stds[m/10]
    k_floor_out<<<1, 1, 0, st>>>(sel, d_out);
    launches += 3;
    return cudaGetLastError();
}

// Enqueue the anisotropy of d_v into d_out (AnisoOut); nb >= 64 checked by the caller.
cudaError_t launch_aniso(const float* d_v, int nz, int ny, int nx, AnisoOut* d_out, void* scratch, cudaStream_t st,
                         int& launches) {
    const int bz = nz / 8, by = ny / 8, bx = nx / 8;
    const long nb = (long)bz * by * bx;
    char* base = (char*)scratch;
    unsigned long long* nvalid = (unsigned long long*)base;
    unsigned long long* sel = nvalid + 1;
    const CalibLayout L = calib_layout(nb);
    unsigned long long* key = (unsigned long long*)(base + L.keys);
    double* bmean = (double*)(base + L.mean);
    double* bvar = (double*)(base + L.var);
    double4* part = (double4*)(base + L.part);
    int* used = (int*)(base + L.used);
    cudaError_t e = cudaMemsetAsync(nvalid, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
    k_block_stats<1><<<blocks_for(nb), 256, 0, st>>>(d_v, ny, nx, 8, bz, by, bx, key, bmean, bvar, nvalid);
    const size_t smem = 256 * kSelThreads * sizeof(unsigned int);
    if ((e = fy_smem_optin(k_select, smem)) != cudaSuccess) return e;
    k_select<<<1, kSelThreads, smem, st>>>(key, nb, nvalid, 5, sel);            // bvar[nv/5]
    k_aniso_lags<<<blocks_for(nb), 256, 0, st>>>(d_v, ny, nx, bz, by, bx, key, bvar, bmean, sel, part, used);
    k_aniso_final<<<1, 256, 0, st>>>(part, used, nb, nvalid, d_out);
    launches += 4;
    return cudaGetLastError();
}

}  // namespace

// ---------------------------------------------------------------- C-ABI: host histogram state
// The 256-bin bookkeeping is O(256) host work on caller-visible arrays (fy_hist_state is
// part of the ABI); the per-voxel counting runs on the GPU.
extern "C" void fy_hist_init(fy_hist_state* s) {
    if (!s) return;
    memset(s->hist, 0, sizeof(s->hist));
    s->total = 0;
}

extern "C" void fy_hist_merge(fy_hist_state* dst, const fy_hist_state* src) {
    if (!dst || !src) return;
    for (int i = 0; i < 256; ++i) dst->hist[i] += src->hist[i];
    dst->total += src->total;
}

// stream.c:99-104: the first bin whose running count reaches (long)(pct/100 * total).
extern "C" int fy_hist_percentile_u8(const fy_hist_state* s, double pct) {
    if (!s) return 255;
    const long target = (long)(pct / 100.0 * (double)s->total);
    long acc = 0;
    for (int i = 0; i < 256; ++i) {
        acc += s->hist[i];
        if (acc >= target) return i;
    }
    return 255;
}

// stream.c:108-116: the same over bins 1..254 (masked 0 and clipped 255 left out).
extern "C" int fy_hist_percentile_u8_inner(const fy_hist_state* s, double pct) {
    if (!s) return 0;
    long total = 0;
    for (int i = 1; i <= 254; ++i) total += s->hist[i];
    if (total <= 0) return 0;
    const long target = (long)(pct / 100.0 * (double)total);
    long acc = 0;
    for (int i = 1; i <= 254; ++i) {
        acc += s->hist[i];
        if (acc >= target) return i;
    }
    return 254;
}

// Host chunk: copied to the device, counted there, the 256 counts added to s.
extern "C" void fy_hist_accumulate_u8(fy_hist_state* s, const unsigned char* chunk, size_t n) {
    fy::enter();
    const char* what = "fy_hist_accumulate_u8";
    if (!s || (!chunk && n)) { fail(FY_EINVAL, "%s: null pointer", what); return; }
    if (n == 0) return;
    if (fy::ensure_ctx()) return;
    fy::ThreadCtx& c = ctx();
    cudaStream_t st = c.st;
    fy::ws_acquire(st);
    cudaError_t e;
    if ((e = c.vin.ensure(n)) != cudaSuccess) { fail_cuda(e, what); return; }
    if ((e = c.small.ensure(256 * sizeof(unsigned long long))) != cudaSuccess) { fail_cuda(e, what); return; }
    if ((e = c.pin.ensure(256 * sizeof(unsigned long long))) != cudaSuccess) { fail_cuda(e, what); return; }
    unsigned long long* dh = c.small.as<unsigned long long>();
    if ((e = cudaMemsetAsync(dh, 0, 256 * sizeof(unsigned long long), st)) != cudaSuccess) { fail_cuda(e, what); return; }
    if ((e = cudaMemcpyAsync(c.vin.p, chunk, n, cudaMemcpyHostToDevice, st)) != cudaSuccess) { fail_cuda(e, what); return; }
    const size_t q = n / 16 + 1;
    const unsigned g = (unsigned)std::min<size_t>((q + kHistThreads - 1) / kHistThreads, (size_t)c.sms * 4);
    k_hist_u8<<<g, kHistThreads, 0, st>>>(c.vin.as<uint8_t>(), n, dh);
    fy::count_launch();
    if ((e = cudaGetLastError()) != cudaSuccess) { fail_cuda(e, what); return; }
    if ((e = cudaMemcpyAsync(c.pin.p, dh, 256 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st)) != cudaSuccess) {
        fail_cuda(e, what);
        return;
    }
    fy::ws_release(st);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) { fail_cuda(e, what); return; }
    const unsigned long long* hh = (const unsigned long long*)c.pin.p;
    for (int i = 0; i < 256; ++i) s->hist[i] += (long)hh[i];
    s->total += (long)n;
}

// Returns the noise floor; NaN (with the reason in fy_gpu_last_error) when it cannot run.
extern "C" double fy_flat_noise(const float* v, int nz, int ny, int nx, int blk) {
    fy::enter();
    const char* what = "fy_flat_noise";
    const double nan = __builtin_nan("");
    if (blk < 4) blk = 8;                                             // stream.c:175
    if (nz < 0 || ny < 0 || nx < 0) { fail(FY_EINVAL, "%s: bad dims", what); return nan; }
    const long nb = nblocks(nz, ny, nx, blk);
    if (nb <= 0) return 0;                                            // stream.c:176
    if (!v) { fail(FY_EINVAL, "%s: null input", what); return nan; }
    if (fy::ensure_ctx()) return nan;
    fy::ThreadCtx& c = ctx();
    cudaStream_t st = c.st;
    const size_t n = (size_t)nz * ny * nx;
    fy::ws_acquire(st);
    cudaError_t e;
    if ((e = c.vin.ensure(n * sizeof(float))) != cudaSuccess) { fail_cuda(e, what); return nan; }
    if ((e = c.aux.ensure(calib_layout(nb).total)) != cudaSuccess) { fail_cuda(e, what); return nan; }
    if ((e = c.small.ensure(256)) != cudaSuccess) { fail_cuda(e, what); return nan; }
    if ((e = c.pin.ensure(sizeof(double))) != cudaSuccess) { fail_cuda(e, what); return nan; }
    if ((e = cudaMemcpyAsync(c.vin.p, v, n * sizeof(float), cudaMemcpyHostToDevice, st)) != cudaSuccess) {
        fail_cuda(e, what);
        return nan;
    }
    int launches = 0;
    double* d_out = c.small.as<double>();
    if ((e = launch_flat_noise(c.vin.as<float>(), nz, ny, nx, blk, d_out, c.aux.p, st, launches)) != cudaSuccess) {
        fail_cuda(e, what);
        return nan;
    }
    fy::count_launch(launches);
    if ((e = cudaMemcpyAsync(c.pin.p, d_out, sizeof(double), cudaMemcpyDeviceToHost, st)) != cudaSuccess) {
        fail_cuda(e, what);
        return nan;
    }
    fy::ws_release(st);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) { fail_cuda(e, what); return nan; }
    return *(const double*)c.pin.p;
}

// 0 with rho_z, rho_xy written; 1 (the reference's failure) for too few blocks; an FY_E*
// code above 1 when it cannot run.
extern "C" int fy_noise_aniso(const float* v, int nz, int ny, int nx, double* rho_z, double* rho_xy) {
    fy::enter();
    const char* what = "fy_noise_aniso";
    if (nz < 0 || ny < 0 || nx < 0) return fail(FY_EINVAL, "%s: bad dims", what);
    const long nb = nblocks(nz, ny, nx, 8);
    if (nb < 64) return 1;                                            // noise.c:217
    if (!v || !rho_z || !rho_xy) return fail(FY_EINVAL, "%s: null pointer", what);
    int rc = fy::ensure_ctx();
    if (rc) return rc;
    fy::ThreadCtx& c = ctx();
    cudaStream_t st = c.st;
    const size_t n = (size_t)nz * ny * nx;
    fy::ws_acquire(st);
    cudaError_t e;
    if ((e = c.vin.ensure(n * sizeof(float))) != cudaSuccess) return fail_cuda(e, what);
    if ((e = c.aux.ensure(calib_layout(nb).total)) != cudaSuccess) return fail_cuda(e, what);
    if ((e = c.small.ensure(256)) != cudaSuccess) return fail_cuda(e, what);
    if ((e = c.pin.ensure(sizeof(AnisoOut))) != cudaSuccess) return fail_cuda(e, what);
    if ((e = cudaMemcpyAsync(c.vin.p, v, n * sizeof(float), cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return fail_cuda(e, what);
    int launches = 0;
    AnisoOut* d_out = c.small.as<AnisoOut>();
    if ((e = launch_aniso(c.vin.as<float>(), nz, ny, nx, d_out, c.aux.p, st, launches)) != cudaSuccess)
        return fail_cuda(e, what);
    fy::count_launch(launches);
    if ((e = cudaMemcpyAsync(c.pin.p, d_out, sizeof(AnisoOut), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return fail_cuda(e, what);
    fy::ws_release(st);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return fail_cuda(e, what);
    const AnisoOut o = *(const AnisoOut*)c.pin.p;
    if (o.status) return 1;
    *rho_z = o.rho_z;
    *rho_xy = o.rho_xy;
    return 0;
}

// ---------------------------------------------------------------- C-ABI: device forms
extern "C" int fy_gpu_hist_accumulate_u8(const unsigned char* d_chunk, size_t n, unsigned long long* d_hist,
                                         void* stream) {
    fy::enter();
    const char* what = "fy_gpu_hist_accumulate_u8";
    if ((!d_chunk && n) || !d_hist) return fail(FY_EINVAL, "%s: null pointer", what);
    if (n == 0) return FY_OK;
    int rc = fy::ensure_ctx();
    if (rc) return rc;
    const size_t q = n / 16 + 1;
    const unsigned g = (unsigned)std::min<size_t>((q + kHistThreads - 1) / kHistThreads, (size_t)ctx().sms * 4);
    k_hist_u8<<<g, kHistThreads, 0, (cudaStream_t)stream>>>(d_chunk, n, d_hist);
    fy::count_launch();
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? FY_OK : fail_cuda(e, what);
}

extern "C" size_t fy_gpu_calib_scratch_bytes(int nz, int ny, int nx, int blk) {
    if (blk < 4) blk = 8;
    long nb = nblocks(nz, ny, nx, blk);
    const long nb8 = nblocks(nz, ny, nx, 8);
    if (nb8 > nb) nb = nb8;
    return calib_layout(nb > 0 ? nb : 1).total;
}

extern "C" int fy_gpu_flat_noise(const float* d_v, int nz, int ny, int nx, int blk, double* d_floor,
                                 void* d_scratch, void* stream) {
    fy::enter();
    const char* what = "fy_gpu_flat_noise";
    if (!d_v || !d_floor || !d_scratch) return fail(FY_EINVAL, "%s: null pointer", what);
    if (nz < 0 || ny < 0 || nx < 0) return fail(FY_EINVAL, "%s: bad dims", what);
    if (blk < 4) blk = 8;
    int rc = fy::ensure_ctx();
    if (rc) return rc;
    int launches = 0;
    const cudaError_t e = launch_flat_noise(d_v, nz, ny, nx, blk, d_floor, d_scratch, (cudaStream_t)stream, launches);
    fy::count_launch(launches);
    return e == cudaSuccess ? FY_OK : fail_cuda(e, what);
}

extern "C" int fy_gpu_noise_aniso(const float* d_v, int nz, int ny, int nx, fy_aniso_result* d_out, void* d_scratch,
                                  void* stream) {
    fy::enter();
    const char* what = "fy_gpu_noise_aniso";
    static_assert(sizeof(fy_aniso_result) == sizeof(AnisoOut), "fy_aniso_result layout");
    if (!d_v || !d_out || !d_scratch) return fail(FY_EINVAL, "%s: null pointer", what);
    if (nz < 0 || ny < 0 || nx < 0) return fail(FY_EINVAL, "%s: bad dims", what);
    int rc = fy::ensure_ctx();
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    if (nblocks(nz, ny, nx, 8) < 64) {                                // noise.c:217: status 1
        const AnisoOut o{0.0, 0.0, 1};
        const cudaError_t e = cudaMemcpyAsync(d_out, &o, sizeof o, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) cudaStreamSynchronize(st);            // `o` lives on this stack
        return e == cudaSuccess ? FY_OK : fail_cuda(e, what);
    }
    int launches = 0;
    const cudaError_t e = launch_aniso(d_v, nz, ny, nx, (AnisoOut*)d_out, d_scratch, st, launches);
    fy::count_launch(launches);
    return e == cudaSuccess ? FY_OK : fail_cuda(e, what);
}
