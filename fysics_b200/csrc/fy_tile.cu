// fy_tile.cu -- the export tool's per-tile chain (fy_process_buffer, pipeline.c:252-510) on
// the GPU: one haloed u8 tile in, the inner tile as u8 out.
//
//   k_tile_any      all-air test (pipeline.c:472-476): an empty buffer skips the chain
//   k_tile_prep     u8/255 (pipeline.c:46-48), ring subtraction at scale 1/255
//                   (dering.c:200-248), z drift (zdrift.c:64-71); writes orig and the working
//                   field, windowed to physical units when the deconvolution runs (:271-272)
//   deconvolution   fy_gpu_deconvolve_ex in place: plain auto-reg, or matched (:273-275)
//   k_tile_unwin    re-window, dec-range rescale, clamp to [0, 1] (:277-288)
//   guided filter   fy_gpu_guided, r = 2, subsampled coefficients by default (:290-297)
//   air zero        k_box_line_smem x3 over the 2x-decimated orig (the sliding sums of
//                   guided.c:34-98; the last pass also bins the means), k_air_cut (stream.c:138-168 and
//                   pipeline.c:330-364), k_air_apply (the texture split, :355-399), which
//                   also writes the despeckle's x-run labels
//   despeckle       union-find over 6-connected material (:223-250, :400-405): k_cc_union,
//                   k_cc_count (roots, sizes, face contact); the zeroing of small interior
//                   components is applied by the quantiser
//   k_tile_quant    recenter (:407-421) and the dithered quantiser (:53-65, :501-506) over
//                   the inner tile
//
// Arithmetic follows the reference source operation for operation, with its a*b+c forms
// fused and its divisions by constants taken as multiplications by the rounded reciprocal,
// as its build (-Ofast, FMA target) compiles them. The box smooth's 1/count is IEEE: the
// reference build's vectorised reciprocals depend on the host CPU in their last bit. With
// the deconvolution and guided filter off, the output equals the oracle restatement bit for
// bit.
#include "fy_context.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <algorithm>

using fy::ctx;
using fy::fail;
using fy::fail_cuda;

extern "C" int fy_gpu_deconvolve_ex(const void* d_in, int src_u8, double f32_min, double f32_max, float* d_out,
                                    int nz, int ny, int nx, const fy_physics* p, double param, int kind,
                                    double fz2_scale, void* stream);
extern "C" int fy_gpu_guided(const float* d_in, float* d_out, int nz, int ny, int nx, int radius, double eps, int s,
                             void* stream);

namespace {

constexpr int kUfMaxIter = 1 << 22;      // bound on every union-find walk (never reached in practice)
constexpr unsigned kEdge = 0x80000000u;  // component touches a face of the buffer
constexpr int kTpb = 128;

struct TileCtl {
    int any;                  // the buffer has a nonzero voxel
    int err;                  // a union-find walk hit kUfMaxIter
    unsigned hist[256];       // scratch-smooth histogram
    int cuts[3];              // value cut, uniform cut, textured cut (u8 levels)
    float cutf_uni, cutf_tex;
};

// stream.c:138-168
__host__ __device__ double valley_depth_hd(const long* hist, int* dark_out, int* light_out, int* valley_out) {
    double hf[256];
    for (int i = 0; i < 256; i++) {
        long s = 0;
        int cnt = 0;
        for (int j = i - 2; j <= i + 2; j++)
            if (j >= 0 && j < 256) { s += hist[j]; cnt++; }
        hf[i] = (double)s / cnt;
    }
    hf[0] = 0; hf[254] = 0; hf[255] = 0;
    double mx = 0;
    for (int i = 0; i < 256; i++) mx = hf[i] > mx ? hf[i] : mx;
    if (mx <= 0) return -1;
    int pk[256], np = 0;
    for (int u = 3; u < 253; u++) {
        if (!(hf[u] >= hf[u - 1] && hf[u] >= hf[u + 1] && hf[u] > 0.05 * mx)) continue;
        if (np > 0 && u - pk[np - 1] <= 10) {
            if (hf[u] > hf[pk[np - 1]]) pk[np - 1] = u;
        } else {
            pk[np++] = u;
        }
    }
    if (np < 2) return -1;
    int p1 = pk[0], p2 = pk[1];
    for (int i = 0; i < np; i++) {
        const int u = pk[i];
        if (hf[u] > hf[p1]) { p2 = p1; p1 = u; }
        else if (hf[u] > hf[p2] && u != p1) p2 = u;
    }
    const int a = p1 < p2 ? p1 : p2, b = p1 < p2 ? p2 : p1;
    int v = a;
    double vmin = hf[a];
    for (int u = a; u <= b; u++)
        if (hf[u] < vmin) { vmin = hf[u]; v = u; }
    if (dark_out) *dark_out = a;
    if (light_out) *light_out = b;
    if (valley_out) *valley_out = v;
    const double mn = hf[a] < hf[b] ? hf[a] : hf[b];
    return 1.0 - vmin / (mn + 1e-12);
}

// pipeline.c:53-58
__device__ __forceinline__ float dither01(long z, long y, long x) {
    unsigned h = (unsigned)z * 73856093u ^ (unsigned)y * 19349663u ^ (unsigned)x * 83492791u;
    h ^= h >> 16;
    h *= 0x7feb352du;
    h ^= h >> 15;
    h *= 0x846ca68bu;
    h ^= h >> 16;
    return __fmul_rn((float)(h >> 8), 1.0f / 16777216.0f);
}

// ---------------------------------------------------------------- all-air test
__global__ void __launch_bounds__(256) k_tile_any(const uint8_t* __restrict__ u8, size_t n, TileCtl* ctl) {
    const size_t mis = (size_t)((16 - ((uintptr_t)u8 & 15)) & 15);
    const size_t head = mis < n ? mis : n;
    const size_t nw = (n - head) / 16, tail = head + nw * 16;
    const uint4* w = reinterpret_cast<const uint4*>(u8 + head);
    const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x, nth = (size_t)gridDim.x * blockDim.x;
    unsigned found = 0;
    for (size_t i = tid; i < nw; i += nth) {
        const uint4 v = __ldg(w + i);
        found |= v.x | v.y | v.z | v.w;
    }
    for (size_t i = tid; i < head; i += nth) found |= u8[i];
    for (size_t i = tail + tid; i < n; i += nth) found |= u8[i];
    if (__syncthreads_or(found != 0) && threadIdx.x == 0) ctl->any = 1;
}

// ---------------------------------------------------------------- prep
struct PrepArgs {
    const uint8_t* u8;
    float* orig;
    float* work;              // the deconvolution's input (windowed), or nullptr
    long hz, hy, hx;
    // rings: rows [s0, s0 + rows) of the [nslab][nr] table, or ring == nullptr
    const float* ring;
    long s0, nslab, slab_z;
    int nr;
    double cy, cx;
    long rz0, ry0, rx0;
    float sc;
    const float* zdrift;      // hz factors from global z = rz0, or nullptr
    int windowed;
    float wlo, wspan;
};

// Four consecutive voxels per thread (one 4-byte load, 16-byte stores when aligned).
// Coordinates are derived only when rings or z drift need them.
__device__ __forceinline__ float prep_one(const PrepArgs& a, unsigned u, size_t i, unsigned plane) {
    float f = __fmul_rn((float)u, 1.0f / 255.0f);
    if (a.ring || a.zdrift) {
        const unsigned ii = (unsigned)i;            // hz*hy*hx < 2^31
        const unsigned z = ii / plane, rem = ii - z * plane;
        if (a.ring && f > 0.0f) {
            const unsigned y = rem / (unsigned)a.hx, x = rem - y * (unsigned)a.hx;
            const double gy = (double)(a.ry0 + y) - a.cy, gx = (double)(a.rx0 + x) - a.cx;
            const int r = (int)(sqrt(gy * gy + gx * gx) + 0.5);
            if (r < a.nr) {
                long s = (a.rz0 + (long)z) / a.slab_z;
                s = s < 0 ? 0 : (s >= a.nslab ? a.nslab - 1 : s);
                const float w = __fmaf_rn(-a.sc, __ldg(a.ring + (size_t)(s - a.s0) * a.nr + r), f);
                f = w > 0.0f ? w : 0.0f;
            }
        }
        if (a.zdrift) f = __fmul_rn(f, __ldg(a.zdrift + z));
    }
    return f;
}

__global__ void __launch_bounds__(256) k_tile_prep(PrepArgs a) {
    const size_t n = (size_t)a.hz * a.hy * a.hx;
    const unsigned plane = (unsigned)(a.hy * a.hx);
    const bool vec = ((uintptr_t)a.u8 & 3) == 0;
    for (size_t q = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) * 4; q < n;
         q += (size_t)gridDim.x * blockDim.x * 4) {
        unsigned u[4] = {0, 0, 0, 0};
        if (vec && q + 4 <= n) {
            const uchar4 v = *reinterpret_cast<const uchar4*>(a.u8 + q);
            u[0] = v.x; u[1] = v.y; u[2] = v.z; u[3] = v.w;
        } else {
            for (int k = 0; k < 4 && q + k < n; k++) u[k] = a.u8[q + k];
        }
        float f[4], w[4];
        for (int k = 0; k < 4; k++) {
            f[k] = prep_one(a, u[k], q + k, plane);
            w[k] = a.windowed ? __fmaf_rn(f[k], a.wspan, a.wlo) : f[k];
        }
        if (q + 4 <= n) {                           // orig and work are 256-byte aligned, q % 4 == 0
            *reinterpret_cast<float4*>(a.orig + q) = make_float4(f[0], f[1], f[2], f[3]);
            if (a.work) *reinterpret_cast<float4*>(a.work + q) = make_float4(w[0], w[1], w[2], w[3]);
        } else {
            for (int k = 0; q + k < n; k++) {
                a.orig[q + k] = f[k];
                if (a.work) a.work[q + k] = w[k];
            }
        }
    }
}

// ---------------------------------------------------------------- after the deconvolution
__global__ void __launch_bounds__(256) k_tile_unwin(float* __restrict__ f, size_t n, int windowed, float wlo,
                                                    float inv, int rescale, float lo, float dinv) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        float v = f[i];
        if (windowed) v = __fmul_rn(__fsub_rn(v, wlo), inv);
        if (rescale) v = __fmul_rn(__fsub_rn(v, lo), dinv);
        f[i] = v < 0.0f ? 0.0f : (v > 1.0f ? 1.0f : v);
    }
}

// ---------------------------------------------------------------- scratch smooth
// One thread per line: prime the sum with samples [0, r], then per sample emit sum/count and
// slide (add the entering sample, then subtract the leaving one), as guided.c:56-95.
struct LineArgs {
    const float* in;
    float* out;
    int L, r;
    long A, B;                // lines = A x B
    long ia, ib, il;          // input strides: outer, inner, along the line
    long oa, ob, ol;
    unsigned* hist;           // staged kernel only: histogram of the means (the air cut's bins)
};

__global__ void __launch_bounds__(kTpb) k_box_line(LineArgs a) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.A * a.B) return;
    const long ai = t / a.B, bi = t - ai * a.B;
    const float* in = a.in + ai * a.ia + bi * a.ib;
    float* out = a.out + ai * a.oa + bi * a.ob;
    float s = 0.0f;
    for (int i = 0; i <= a.r && i < a.L; ++i) s = __fadd_rn(s, in[i * a.il]);
    for (int i = 0; i < a.L; ++i) {
        const int lo = i - a.r < 0 ? 0 : i - a.r, hi = i + a.r > a.L - 1 ? a.L - 1 : i + a.r;
        out[i * a.ol] = __fmul_rn(s, __frcp_rn((float)(hi - lo + 1)));
        if (i + a.r + 1 < a.L) s = __fadd_rn(s, in[(i + a.r + 1) * a.il]);
        if (i - a.r >= 0) s = __fsub_rn(s, in[(i - a.r) * a.il]);
    }
}

// The same sliding sums with the lines staged through shared memory: a CTA takes kLines
// consecutive lines, loads them with coalesced requests (along the line when it is
// contiguous, across lines otherwise), walks its line in shared memory and stores the
// means back the same way. Shared memory: 2 * L * (kLines + 1) floats.
constexpr int kLines = 32;               // lines per CTA: ~5000 lines per pass at 144^3 -> 160 CTAs
constexpr int kLineThreads = 128;        // the load and store phases use four warps
constexpr int kLp = kLines + 1;
__global__ void __launch_bounds__(kLineThreads) k_box_line_smem(LineArgs a, int along) {
    extern __shared__ float sl[];
    float* so = sl + (size_t)a.L * kLp;
    __shared__ long ibase[kLines], obase[kLines];
    __shared__ unsigned shist[256];
    if (a.hist)
        for (int k = threadIdx.x; k < 256; k += kLineThreads) shist[k] = 0;
    const long lines = a.A * a.B, t0 = (long)blockIdx.x * kLines;
    const int tid = threadIdx.x;
    const int nl = (int)(lines - t0 < kLines ? lines - t0 : kLines);
    if (tid < nl) {
        const long t = t0 + tid, ai = t / a.B, bi = t - ai * a.B;
        ibase[tid] = ai * a.ia + bi * a.ib;
        obase[tid] = ai * a.oa + bi * a.ob;
    }
    __syncthreads();
    // contiguous lines: consecutive threads walk along a line (k = j*L + e); otherwise they
    // walk across lines (k = e*kLines + j), skipping the missing lines of the last CTA
    const unsigned L = (unsigned)a.L, total = along ? (unsigned)nl * L : (unsigned)kLines * L;
#pragma unroll 4
    for (unsigned k = tid; k < total; k += kLineThreads) {
        const unsigned j = along ? k / L : k % kLines, e = along ? k - (k / L) * L : k / kLines;
        if ((int)j < nl) sl[e * kLp + j] = a.in[ibase[j] + (long)e * a.il];
    }
    __syncthreads();
    if (tid < nl) {
        const float* in = sl + tid;
        float* out = so + tid;
        const float rin = __frcp_rn((float)(2 * a.r + 1));
        float s = 0.0f;
        for (int i = 0; i <= a.r && i < a.L; ++i) s = __fadd_rn(s, in[i * kLp]);
        for (int i = 0; i < a.L; ++i) {
            const int lo = i - a.r < 0 ? 0 : i - a.r, hi = i + a.r > a.L - 1 ? a.L - 1 : i + a.r;
            const int cnt = hi - lo + 1;
            out[i * kLp] = __fmul_rn(s, cnt == 2 * a.r + 1 ? rin : __frcp_rn((float)cnt));
            if (i + a.r + 1 < a.L) s = __fadd_rn(s, in[(i + a.r + 1) * kLp]);
            if (i - a.r >= 0) s = __fsub_rn(s, in[(i - a.r) * kLp]);
        }
    }
    __syncthreads();
#pragma unroll 4
    for (unsigned k = tid; k < total; k += kLineThreads) {
        const unsigned j = along ? k / L : k % kLines, e = along ? k - (k / L) * L : k / kLines;
        if ((int)j < nl) {
            const float v = so[e * kLp + j];
            a.out[obase[j] + (long)e * a.ol] = v;
            if (a.hist) {                   // pipeline.c:318-321: (int)(v*255 + 0.5), clamped
                int bin = (int)__fmaf_rn(v, 255.0f, 0.5f);
                bin = bin < 0 ? 0 : (bin > 255 ? 255 : bin);
                atomicAdd(&shist[bin], 1u);
            }
        }
    }
    if (a.hist) {
        __syncthreads();
        for (int k = threadIdx.x; k < 256; k += kLineThreads)
            if (shist[k]) atomicAdd(&a.hist[k], shist[k]);
    }
}

__global__ void __launch_bounds__(256) k_air_hist(const float* __restrict__ sm, size_t n, TileCtl* ctl) {
    __shared__ unsigned h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        int b = (int)__fmaf_rn(sm[i], 255.0f, 0.5f);
        b = b < 0 ? 0 : (b > 255 ? 255 : b);
        atomicAdd(&h[b], 1u);
    }
    __syncthreads();
    if (h[threadIdx.x]) atomicAdd(&ctl->hist[threadIdx.x], h[threadIdx.x]);
}

// The valley (stream.c:138-168) and the value cut with its texture split (pipeline.c:330-378),
// one CTA of 256 threads, a thread per bin: smoothed counts, their maximum, the local-maximum
// candidates and the valley's first minimum in parallel; the peak merge, which is sequential
// by definition, walks the candidate bits on one thread. Same arithmetic as valley_depth_hd.
__global__ void __launch_bounds__(256) k_air_cut(TileCtl* ctl, int air_cut_u8, int air_cut_band, double air_thresh,
                                                 double air_cut_aggr) {
    __shared__ double hf[256];
    __shared__ double wmax[8];
    __shared__ unsigned cand[8];
    __shared__ int s_ab[3];
    __shared__ double wmin[8];
    __shared__ int wmini[8];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    long sum = 0;
    int cnt = 0;
    for (int j = t - 2; j <= t + 2; j++)
        if (j >= 0 && j < 256) { sum += ctl->hist[j]; cnt++; }
    double h = (double)sum / cnt;
    if (t == 0 || t == 254 || t == 255) h = 0;
    hf[t] = h;
    double m = h;
    for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0) wmax[warp] = m;
    __syncthreads();
    double mx = wmax[0];
    for (int k = 1; k < 8; k++) mx = fmax(mx, wmax[k]);
    const bool c = t >= 3 && t < 253 && hf[t] >= hf[t - 1] && hf[t] >= hf[t + 1] && hf[t] > 0.05 * mx;
    const unsigned bal = __ballot_sync(0xffffffffu, c);
    if (lane == 0) cand[warp] = bal;
    __syncthreads();
    if (t == 0) {
        int ok = 0, a = 0, b = 0;
        if (mx > 0) {
            int pk[32], np = 0;           // kept peaks are > 10 bins apart: at most 23 in [3, 253)
            for (int w = 0; w < 8; w++)
                for (unsigned bits = cand[w]; bits; bits &= bits - 1) {
                    const int u = w * 32 + __ffs(bits) - 1;
                    if (np > 0 && u - pk[np - 1] <= 10) {
                        if (hf[u] > hf[pk[np - 1]]) pk[np - 1] = u;
                    } else if (np < 32) {
                        pk[np++] = u;
                    }
                }
            if (np >= 2) {
                int p1 = pk[0], p2 = pk[1];
                for (int i = 0; i < np; i++) {
                    const int u = pk[i];
                    if (hf[u] > hf[p1]) { p2 = p1; p1 = u; }
                    else if (hf[u] > hf[p2] && u != p1) p2 = u;
                }
                a = p1 < p2 ? p1 : p2;
                b = p1 < p2 ? p2 : p1;
                ok = 1;
            }
        }
        s_ab[0] = a; s_ab[1] = b; s_ab[2] = ok;
    }
    __syncthreads();
    const int a = s_ab[0], b = s_ab[1], ok = s_ab[2];
    // first minimum over [a, b] (strict <, so the lowest bin among equal minima)
    double vm = (ok && t >= a && t <= b) ? hf[t] : INFINITY;
    int vi = (ok && t >= a && t <= b) ? t : 1 << 30;
    for (int o = 16; o; o >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, vm, o);
        const int oi = __shfl_xor_sync(0xffffffffu, vi, o);
        if (ov < vm || (ov == vm && oi < vi)) { vm = ov; vi = oi; }
    }
    if (lane == 0) { wmin[warp] = vm; wmini[warp] = vi; }
    __syncthreads();
    if (t != 0) return;
    int dark = 0, light = 0, valley = 0;
    double d = -1;
    if (ok) {
        double vmin = wmin[0];
        int v = wmini[0];
        for (int k = 1; k < 8; k++)
            if (wmin[k] < vmin || (wmin[k] == vmin && wmini[k] < v)) { vmin = wmin[k]; v = wmini[k]; }
        dark = a; light = b; valley = v;
        const double mn = hf[a] < hf[b] ? hf[a] : hf[b];
        d = 1.0 - vmin / (mn + 1e-12);
    }
    const int pf = air_thresh > 0 ? (int)__fma_rn(air_thresh, 255.0, 0.5) : 39;
    int cut;
    if (air_cut_u8 >= 0) {
        const int gg = air_cut_u8, band = air_cut_band;
        if (d >= 0) {
            double g = air_cut_aggr;
            g = g < 0 ? 0 : (g > 2 ? 2 : g);
            int local;
            if (valley <= pf) local = pf;
            else if (g <= 1.0) local = (int)__dadd_rn(__fma_rn(g, (double)(valley - pf), (double)pf), 0.5);
            else
                local = (int)__dadd_rn(
                    __fma_rn(__dsub_rn(g, 1.0), (double)(light > valley ? light - valley : 0), (double)valley), 0.5);
            cut = local < gg - band ? gg - band : (local > gg + band ? gg + band : local);
        } else {
            cut = gg;
        }
    } else if (d >= 0) {
        const int mid = (dark + valley) / 2;
        cut = dark + 8 < mid ? dark + 8 : mid;
    } else {
        cut = (int)__dmul_rn(air_thresh > 0 ? air_thresh : 0.05, 255.0);
    }
    const int spread = valley > pf ? (valley - pf) / 2 : 8;
    int cu = cut + spread;
    if (valley > cut && cu > valley) cu = valley;
    int ct = cut - spread;
    if (ct < pf) ct = pf;
    ctl->cuts[0] = cut;
    ctl->cuts[1] = cu;
    ctl->cuts[2] = ct;
    ctl->cutf_uni = __fmul_rn((float)cu, 1.0f / 255.0f);
    ctl->cutf_tex = __fmul_rn((float)ct, 1.0f / 255.0f);
}

// The x of the first voxel of this voxel's material run within the CTA's row segment
// (threads = consecutive x, whole warps): the warp's own ballot, then the earlier warps'
// ballots in shared memory. Every thread of the CTA must call it (two barriers).
__device__ __forceinline__ int run_head(bool mat, unsigned* wbits) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned bits = __ballot_sync(0xffffffffu, mat);
    if (lane == 0) wbits[warp] = bits;
    __syncthreads();
    int head = 0;
    const unsigned gaps = ~bits & ((1u << lane) - 1u);
    if (gaps) {
        head = warp * 32 + 32 - __clz(gaps);
    } else {
        for (int w = warp - 1; w >= 0; --w) {
            const unsigned g = ~wbits[w];
            if (g) { head = w * 32 + 32 - __clz(g); break; }
        }
    }
    __syncthreads();                         // wbits is rewritten by the next row
    return head;
}

struct AirArgs {
    float* f;                 // may alias orig: each voxel reads orig and writes f at itself
    const float* orig;
    const float* sm;
    const TileCtl* ctl;
    long nz, ny, nx, lz, ly, lx;
    int lowres;
    int* lab;                 // despeckle on: x-run labels of the material (f > 0) written here
    unsigned* info;
};

__device__ __forceinline__ float blend4(const float* s, size_t r00, size_t r01, size_t r10, size_t r11, long k,
                                        float w00, float w01, float w10, float w11) {
    return __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(w00, s[r00 + k]), __fmul_rn(w01, s[r01 + k])),
                               __fmul_rn(w10, s[r10 + k])),
                     __fmul_rn(w11, s[r11 + k]));
}

// zero f where the scratch smooth (trilinear from the decimated grid) is below the cut,
// the cut chosen by the local texture |orig - smooth| (pipeline.c:355-399)
__global__ void __launch_bounds__(1024) k_air_apply(AirArgs a) {
    __shared__ unsigned wbits[32];
    const long x = (long)blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    const bool in = x < a.nx;
    const float cu = a.ctl->cutf_uni, ct = a.ctl->cutf_tex;
    for (long z = blockIdx.z; z < a.nz; z += gridDim.z) {
        const size_t i = ((size_t)z * a.ny + y) * a.nx + x;
        float fv = 0.0f;
        if (in) {
            float v;
            if (a.lowres) {
                long z0 = z >> 1, y0 = y >> 1, x0 = x >> 1;
                if (z0 > a.lz - 2) z0 = a.lz - 2;
                if (y0 > a.ly - 2) y0 = a.ly - 2;
                if (x0 > a.lx - 2) x0 = a.lx - 2;
                float zf = __fsub_rn(__fmul_rn(0.5f, (float)z), (float)z0);
                float yf = __fsub_rn(__fmul_rn(0.5f, (float)y), (float)y0);
                float fx = __fsub_rn(__fmul_rn(0.5f, (float)x), (float)x0);
                zf = zf > 1.0f ? 1.0f : zf;
                yf = yf > 1.0f ? 1.0f : yf;
                fx = fx > 1.0f ? 1.0f : fx;
                const float w00 = __fmul_rn(1.0f - zf, 1.0f - yf), w01 = __fmul_rn(1.0f - zf, yf);
                const float w10 = __fmul_rn(zf, 1.0f - yf), w11 = __fmul_rn(zf, yf);
                const size_t r00 = ((size_t)z0 * a.ly + y0) * a.lx, r01 = r00 + a.lx;
                const size_t r10 = r00 + (size_t)a.ly * a.lx, r11 = r10 + a.lx;
                const float a0 = blend4(a.sm, r00, r01, r10, r11, x0, w00, w01, w10, w11);
                const float a1 = blend4(a.sm, r00, r01, r10, r11, x0 + 1, w00, w01, w10, w11);
                v = __fmaf_rn(__fsub_rn(a1, a0), fx, a0);
            } else {
                v = a.sm[i];
            }
            const float o = a.orig[i];
            const float tex = fabsf(__fsub_rn(o, v));
            fv = a.f[i];
            if (v < (tex < 0.03f ? cu : ct)) { fv = 0.0f; a.f[i] = 0.0f; }
        }
        if (a.lab) {               // despeckle on: each material voxel points at its x-run's first voxel
            const bool mat = in && fv > 0.0f;
            const int head = run_head(mat, wbits);
            if (in) {
                const int t = (int)threadIdx.x;
                a.lab[i] = mat ? (int)(i - (size_t)(t - head)) : -1;
                if (mat && t == head) a.info[i] = 0u;       // run heads are the only possible roots
            }
        }
    }
}

// ---------------------------------------------------------------- connected components
__device__ __forceinline__ int uf_find(int* L, int i, int* err) {
    for (int it = 0; it < kUfMaxIter; ++it) {
        const int p = __ldcg(L + i);     // L2 reads: links made by other threads are seen
        if (p == i) return i;
        const int g = __ldcg(L + p);
        if (g != p) L[i] = g;            // path halving: g is an ancestor of i
        i = g;
    }
    *err = 1;
    return i;
}

// Read-only walk to the root: the flatten pass uses it, so that no store of another walk can
// land on a label after its final root was written.
__device__ __forceinline__ int uf_root(const int* L, int i, int* err) {
    for (int it = 0; it < kUfMaxIter; ++it) {
        const int p = __ldcg(L + i);
        if (p == i) return i;
        i = p;
    }
    *err = 1;
    return i;
}

__device__ __forceinline__ void uf_union(int* L, int a, int b, int* err) {
    for (int it = 0; it < kUfMaxIter; ++it) {
        a = uf_find(L, a, err);
        b = uf_find(L, b, err);
        if (a == b) return;
        if (a < b) { const int t = a; a = b; b = t; }   // link the larger root under the smaller
        const int old = atomicMin(&L[a], b);
        if (old == a) return;
        a = old;
    }
    *err = 1;
}

struct CcArgs {
    float* f;
    int* lab;
    unsigned* info;
    int* err;
    long nz, ny, nx;
    int min_size;
};

// Join runs: across a row-segment (CTA) boundary in x, and to the -y and -z neighbours where
// a run overlap starts (if the left neighbours are both material, they already joined the
// runs). Launched with the air pass's CTA width, so the segments are the same.
__global__ void __launch_bounds__(1024) k_cc_union(CcArgs a) {
    const long x = (long)blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= a.nx) return;
    const int nx = (int)a.nx, plane = (int)(a.ny * a.nx);
    for (long z = blockIdx.z; z < a.nz; z += gridDim.z) {
        const int i = (int)(((size_t)z * a.ny + y) * a.nx + x);
        // Only the signs (material or not) are read here, and those never change; issuing
        // all six loads before any test keeps them to one memory round trip.
        const int c = a.lab[i];
        const int l = x > 0 ? a.lab[i - 1] : -1;
        const int u = y > 0 ? a.lab[i - nx] : -1;
        const int ul = (x > 0 && y > 0) ? a.lab[i - 1 - nx] : -1;
        const int d = z > 0 ? a.lab[i - plane] : -1;
        const int dl = (x > 0 && z > 0) ? a.lab[i - 1 - plane] : -1;
        if (c < 0) continue;
        const bool left = l >= 0;
        if (left && x % blockDim.x == 0) uf_union(a.lab, i, i - 1, a.err);   // across row segments
        if (u >= 0 && !(left && ul >= 0)) uf_union(a.lab, i, i - nx, a.err);
        if (d >= 0 && !(left && dl >= 0)) uf_union(a.lab, i, i - plane, a.err);
    }
}

// Roots by read-only walks from the x-run heads (a run's voxels share its head's root;
// each thread then stores its voxel's root for the zero pass), component sizes and face
// contact with one atomic per run of equal roots in a warp. A count stops growing once it
// reaches min_size and a face-touching root takes no count: both leave the zero test
// (no face contact and fewer than min_size voxels) unchanged.
__global__ void __launch_bounds__(1024) k_cc_count(CcArgs a) {
    __shared__ unsigned wbits[32];
    __shared__ int sroot[1024];
    const long x = (long)blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    const int lane = threadIdx.x & 31;
    const bool in = x < a.nx;
    for (long z = blockIdx.z; z < a.nz; z += gridDim.z) {
        const size_t i = ((size_t)z * a.ny + y) * a.nx + x;
        const int l = in ? __ldcg(a.lab + i) : -1;
        // the voxel's x-run (within the CTA's row segment) shares one root: the head walks
        const int head = run_head(l >= 0, wbits);
        const int t = (int)threadIdx.x;
        if (l >= 0 && t == head) sroot[t] = uf_root(a.lab, l, a.err);
        __syncthreads();
        const int root = l >= 0 ? sroot[head] : -1;
        __syncthreads();                     // sroot is rewritten by the next row
        if (root >= 0) a.lab[i] = root;
        const bool edge = root >= 0 && (z == 0 || z == a.nz - 1 || y == 0 || y == a.ny - 1 || x == 0 || x == a.nx - 1);
        const int prev = __shfl_up_sync(0xffffffffu, root, 1);
        const unsigned heads = __ballot_sync(0xffffffffu, lane == 0 || prev != root);
        const unsigned edges = __ballot_sync(0xffffffffu, edge);
        if (root >= 0 && (lane == 0 || prev != root)) {
            const unsigned after = heads & ~((2u << lane) - 1u);      // run heads above this lane
            const int end = after ? __ffs(after) - 1 : 32;
            const unsigned seg = (end == 32 ? 0xffffffffu : (1u << end) - 1u) & ~((1u << lane) - 1u);
            // Only "touches a face" and "has at least min_size voxels" decide the zero pass, so
            // a root already known to be either takes no more atomics (the giant components
            // would otherwise serialise on one address).
            const unsigned v = __ldcg(a.info + root);
            if (!(v & kEdge)) {
                if (edges & seg) atomicOr(&a.info[root], kEdge);
                else if ((long)(v & ~kEdge) < a.min_size) atomicAdd(&a.info[root], (unsigned)(end - lane));
            }
        }
    }
}

// ---------------------------------------------------------------- recenter + quantise
struct QuantArgs {
    const float* f;
    uint8_t* out;
    long hy, hx;
    long iz0, iy0, ix0;       // inner tile origin inside the buffer
    long tz, ty, tx;
    long gz0, gy0, gx0;       // inner tile origin in the volume
    int no_dither, norm;
    float midf, k;
    const int* lab;           // despeckle on: voxel -> component root (k_cc_count), else nullptr
    const unsigned* info;
    int min_size;
};

__global__ void __launch_bounds__(1024) k_tile_quant(QuantArgs a) {
    const long x = (long)blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= a.tx) return;
    for (long z = blockIdx.z; z < a.tz; z += gridDim.z) {
        const size_t j = ((size_t)(a.iz0 + z) * a.hy + (a.iy0 + y)) * a.hx + (a.ix0 + x);
        float v = a.f[j];
        if (a.lab) {                        // the despeckle's zeroing, for the voxels kept
            const int root = a.lab[j];
            if (root >= 0) {
                const unsigned c = a.info[root];
                if (!(c & kEdge) && (long)(c & ~kEdge) < a.min_size) v = 0.0f;
            }
        }
        if (a.norm) {
            if (v <= 0.0f) {
                v = 0.0f;
            } else {
                const float w = __fadd_rn(0.5f, __fmul_rn(__fsub_rn(v, a.midf), a.k));   // not fused, as the reference build
                v = w < 0.0f ? 0.0f : (w > 1.0f ? 1.0f : w);
            }
        }
        const float t = __fmaf_rn(v, 255.0f, a.no_dither ? 0.5f : dither01(a.gz0 + z, a.gy0 + y, a.gx0 + x));
        uint8_t q = 0;
        if (t > 0.0f) {
            const int qi = (int)t;
            q = qi > 255 ? 255 : (uint8_t)qi;
        }
        a.out[((size_t)z * a.ty + y) * a.tx + x] = q;
    }
}

// ---------------------------------------------------------------- host side
struct TileWs {
    fy::DevBuf u8, orig, work, alt, t1, t2, sm, lab, info, tab, ctl, out;
    fy::HostBuf pin, hin, hout;   // control and tables; host-API staging of the u8 tile in/out
    bool have_state = false;
    long hist[256];
    int cuts[3];
};
thread_local TileWs tws;

unsigned grid1(size_t n, int tpb, int sms) {
    size_t g = (n + tpb - 1) / tpb, cap = (size_t)sms * 8;
    return (unsigned)std::max<size_t>(1, std::min(g, cap));
}

// Row kernels: a CTA spans a row (x) in whole warps, up to 1024 threads; grid (x, y, z).
// Warp lanes stay aligned with x % 32, which the run labels rely on.
int row_threads(long nx) { return (int)std::min<long>(1024, (nx + 31) / 32 * 32); }
dim3 grid_rows(long nx, long ny, long nz) {
    const long t = row_threads(nx);
    return dim3((unsigned)((nx + t - 1) / t), (unsigned)ny, (unsigned)std::min<long>(nz, 65535));
}

// eps_for_tile, pipeline.c:447-456
double tile_eps(const fy_pipeline_cfg* c, double ecy, double ecx, long y0, long x0, long ty, long tx) {
    if (!c->have_eps_r || c->guided_eps <= 0 || c->eps_fn_med <= 0) return 0.0;
    const double ry = y0 + ty / 2.0 - ecy, rx = x0 + tx / 2.0 - ecx;
    const double fn = c->eps_fn_a + c->eps_fn_b * sqrt(ry * ry + rx * rx);
    const double s = fn / c->eps_fn_med;
    double s2 = s * s;
    if (s2 < 0.4) s2 = 0.4;
    if (s2 > 8.0) s2 = 8.0;
    return c->guided_eps * s2;
}

// One pass of line sums; with ctl set (the last pass) the histogram of the means is added
// to ctl->hist as they are stored (or by k_air_hist after the unstaged kernel).
cudaError_t box_pass(const float* in, float* out, int L, int r, long A, long B, long ia, long ib, long il, long oa,
                     long ob, long ol, cudaStream_t st, TileCtl* ctl = nullptr, int sms = 148) {
    LineArgs a{in, out, L, r, A, B, ia, ib, il, oa, ob, ol, nullptr};
    const long lines = A * B;
    const size_t smem = (size_t)2 * L * kLp * sizeof(float);
    if (smem <= 200 * 1024) {
        cudaError_t e = fy_smem_optin(k_box_line_smem, smem);
        if (e != cudaSuccess) return e;
        a.hist = ctl ? ctl->hist : nullptr;
        k_box_line_smem<<<(unsigned)((lines + kLines - 1) / kLines), kLineThreads, smem, st>>>(a, ib != 1 ? 1 : 0);
    } else {
        k_box_line<<<(unsigned)((lines + kTpb - 1) / kTpb), kTpb, 0, st>>>(a);
        if (ctl) {
            const size_t m = (size_t)A * B * L;
            k_air_hist<<<grid1(m, 256, sms), 256, 0, st>>>(out, m, ctl);
        }
    }
    return cudaGetLastError();
}

#define TRY(call)                                           \
    do {                                                    \
        cudaError_t e_ = (call);                            \
        if (e_ != cudaSuccess) return fail_cuda(e_, what);  \
    } while (0)

int tile_chain(const fy_pipeline_cfg* c, const uint8_t* d_u8, long rz0, long ry0, long rx0, long hz, long hy,
               long hx, long z0, long y0, long x0, long tz, long ty, long tx, long vol_y, long vol_x, uint8_t* d_out,
               int* all_air, cudaStream_t st, const char* what) {
    fy::ThreadCtx& cx = ctx();
    TileWs& w = tws;
    w.have_state = false;
    const size_t hn = (size_t)hz * hy * hx, tn = (size_t)tz * ty * tx;
    TRY(w.ctl.ensure(sizeof(TileCtl)));
    TRY(w.pin.ensure(sizeof(TileCtl)));
    TileCtl* ctl = w.ctl.as<TileCtl>();
    TileCtl* hctl = (TileCtl*)w.pin.p;
    TRY(cudaMemsetAsync(ctl, 0, sizeof(TileCtl), st));
    k_tile_any<<<grid1(hn / 16 + 1, 256, cx.sms), 256, 0, st>>>(d_u8, hn, ctl);
    TRY(cudaGetLastError());
    TRY(cudaMemcpyAsync(hctl, ctl, sizeof(int) * 2, cudaMemcpyDeviceToHost, st));
    TRY(cudaStreamSynchronize(st));
    int launches = 1;
    if (!hctl->any) {
        if (tn) TRY(cudaMemsetAsync(d_out, 0, tn, st));
        TRY(cudaStreamSynchronize(st));
        fy::count_launch(launches);
        if (all_air) *all_air = 1;
        return FY_OK;
    }
    if (c->do_musica) return fail(FY_EUNSUPPORTED, "%s: MUSICA is not on the GPU path", what);

    // ring rows and z-drift factors of this buffer, staged through pinned memory
    const fy_dering* dr = c->have_dering ? c->dering : nullptr;
    const bool rings = dr && dr->have_rings && dr->ring && dr->nr > 0 && dr->nslab > 0 && dr->slab_z > 0;
    const bool zdrift = c->have_zdrift && c->zdrift_factor;
    long s0 = 0, s1 = -1;
    if (rings) {
        auto slab = [&](long z) { long s = z / dr->slab_z; return s < 0 ? 0L : (s >= dr->nslab ? (long)dr->nslab - 1 : s); };
        s0 = slab(rz0);
        s1 = slab(rz0 + hz - 1);
    }
    const size_t ring_floats = rings ? (size_t)(s1 - s0 + 1) * dr->nr : 0, zd_floats = zdrift ? (size_t)hz : 0;
    const size_t ctl_bytes = (sizeof(TileCtl) + 255) & ~(size_t)255;
    const size_t tab_bytes = (ring_floats + zd_floats) * sizeof(float);
    const float* d_ring = nullptr;
    const float* d_zd = nullptr;
    if (tab_bytes) {
        TRY(w.pin.ensure(ctl_bytes + tab_bytes));
        hctl = (TileCtl*)w.pin.p;
        float* h = (float*)((char*)w.pin.p + ctl_bytes);
        if (rings) memcpy(h, dr->ring + (size_t)s0 * dr->nr, ring_floats * sizeof(float));
        if (zdrift) memcpy(h + ring_floats, c->zdrift_factor + rz0, zd_floats * sizeof(float));
        TRY(w.tab.ensure(tab_bytes));
        TRY(cudaMemcpyAsync(w.tab.p, h, tab_bytes, cudaMemcpyHostToDevice, st));
        if (rings) d_ring = w.tab.as<float>();
        if (zdrift) d_zd = w.tab.as<float>() + ring_floats;
    }

    // Buffers: orig (the pre-deconvolution copy) always; the working field is orig itself
    // until a stage writes a new one (deconvolution in place on `work`, guided into `alt`),
    // since the air cut reads orig and writes f one voxel at a time.
    TRY(w.orig.ensure(hn * sizeof(float)));
    float* orig = w.orig.as<float>();
    float* f = orig;
    if (c->do_deconv) {
        TRY(w.work.ensure(hn * sizeof(float)));
        f = w.work.as<float>();
    }
    const bool windowed = c->window_hi > c->window_lo;
    const float wlo = (float)c->window_lo, wspan = (float)(c->window_hi - c->window_lo);
    {
        PrepArgs a{};
        a.u8 = d_u8; a.orig = orig; a.work = c->do_deconv ? f : nullptr;
        a.hz = hz; a.hy = hy; a.hx = hx;
        a.ring = d_ring;
        if (rings) {
            a.s0 = s0; a.nslab = dr->nslab; a.slab_z = dr->slab_z; a.nr = dr->nr; a.cy = dr->cy; a.cx = dr->cx;
        } else {
            a.slab_z = 1; a.nslab = 1;
        }
        a.rz0 = rz0; a.ry0 = ry0; a.rx0 = rx0;
        a.sc = (float)(1.0 / 255.0);
        a.zdrift = d_zd;
        a.windowed = c->do_deconv && windowed;
        a.wlo = wlo; a.wspan = wspan;
        k_tile_prep<<<grid1((hn + 3) / 4, 256, cx.sms), 256, 0, st>>>(a);
        TRY(cudaGetLastError());
        launches++;
        fy_prof_mark(st, "tile.prep");
    }

    int rc;
    if (c->do_deconv) {                                           // pipeline.c:260-288
        fy_physics ph{c->delta_beta, c->energy_kev, c->distance_mm, c->pixel_um, c->unsharp_sigma, c->unsharp_coeff,
                      c->psf_sigma_vox,
                      (c->psf_z_ratio > 1.0 && c->psf_sigma_vox > 0) ? c->psf_z_ratio * c->psf_sigma_vox : 0.0};
        ph.delta_beta *= fy_auto_deltabeta_scale(&ph);
        const bool matched = c->use_matched_deconv && c->psf_sigma_vox > 0;
        if ((rc = fy_gpu_deconvolve_ex(f, 0, 0.0, 0.0, f, (int)hz, (int)hy, (int)hx, &ph,
                                       matched ? c->deconv_tikhonov : -1.0, matched ? 1 : 0, 1.0, st)))
            return rc;
        const bool rescale = c->have_dec_range && c->dec_hi - c->dec_lo > 1e-6;
        k_tile_unwin<<<grid1(hn, 256, cx.sms), 256, 0, st>>>(f, hn, windowed, wlo, windowed ? 1.0f / wspan : 1.0f,
                                                             rescale, (float)c->dec_lo,
                                                             rescale ? 1.0f / (float)(c->dec_hi - c->dec_lo) : 1.0f);
        TRY(cudaGetLastError());
        launches++;
        fy_prof_mark(st, "tile.unwin");
    }

    const double ecy = c->dering_cy > 0 ? c->dering_cy : (vol_y - 1) / 2.0;
    const double ecx = c->dering_cx > 0 ? c->dering_cx : (vol_x - 1) / 2.0;
    const double teps = tile_eps(c, ecy, ecx, y0, x0, ty, tx);
    if (c->guided_eps > 0 || teps > 0) {                          // pipeline.c:290-297
        const double eps = teps > 0 ? teps : c->guided_eps;
        const int gs = c->guided_subsample == 0 ? 2 : c->guided_subsample;
        TRY(w.alt.ensure(hn * sizeof(float)));
        float* g = w.alt.as<float>();
        if ((rc = fy_gpu_guided(f, g, (int)hz, (int)hy, (int)hx, 2, eps, gs, st))) return rc;
        f = g;
        fy_prof_mark(st, "tile.guided");
    }

    if (c->do_air_zero) {                                         // pipeline.c:299-405
        const int sr = c->scratch_passes > 0 ? c->scratch_passes : 5;
        const long lz = (hz + 1) / 2, ly = (hy + 1) / 2, lx = (hx + 1) / 2;
        const bool lowres = lz >= 2 && ly >= 2 && lx >= 2;
        const long mz = lowres ? lz : hz, my = lowres ? ly : hy, mx = lowres ? lx : hx;
        const size_t m = (size_t)mz * my * mx;
        const int r = lowres ? std::max(1, (sr + 1) / 2) : sr;
        const long d = lowres ? 2 : 1;
        TRY(w.t1.ensure(m * sizeof(float)));
        TRY(w.t2.ensure(m * sizeof(float)));
        TRY(w.sm.ensure(m * sizeof(float)));
        float *t1 = w.t1.as<float>(), *t2 = w.t2.as<float>(), *sm = w.sm.as<float>();
        const long mp = my * mx;
        // x lines (decimated read of orig), then y lines, then z lines
        TRY(box_pass(orig, t1, (int)mx, r, mz, my, d * hy * hx, d * hx, d, mp, mx, 1, st));
        TRY(box_pass(t1, t2, (int)my, r, mz, mx, mp, 1, mx, mp, 1, mx, st));
        TRY(box_pass(t2, sm, (int)mz, r, my, mx, mx, 1, mp, mx, 1, mp, st, ctl, cx.sms));   // + histogram
        fy_prof_mark(st, "tile.scratch_box");
        k_air_cut<<<1, 256, 0, st>>>(ctl, c->air_cut_u8, c->air_cut_band, c->air_thresh, c->air_cut_aggr);
        TRY(cudaGetLastError());
        fy_prof_mark(st, "tile.air_cut");
        const bool cc = c->air_min_component > 0;
        if (cc) {
            TRY(w.lab.ensure(hn * sizeof(int)));
            TRY(w.info.ensure(hn * sizeof(unsigned)));
        }
        AirArgs aa{f, orig, sm, ctl, hz, hy, hx, lz, ly, lx, lowres ? 1 : 0, cc ? w.lab.as<int>() : nullptr,
                   cc ? w.info.as<unsigned>() : nullptr};
        k_air_apply<<<grid_rows(hx, hy, hz), row_threads(hx), 0, st>>>(aa);
        TRY(cudaGetLastError());
        launches += 5;
        fy_prof_mark(st, "tile.air_apply");
        if (cc) {
            CcArgs ca{f, w.lab.as<int>(), w.info.as<unsigned>(), &ctl->err, hz, hy, hx, c->air_min_component};
            k_cc_union<<<grid_rows(hx, hy, hz), row_threads(hx), 0, st>>>(ca);
            fy_prof_mark(st, "tile.cc_union");
            k_cc_count<<<grid_rows(hx, hy, hz), row_threads(hx), 0, st>>>(ca);
            TRY(cudaGetLastError());
            launches += 2;
            fy_prof_mark(st, "tile.cc_count");
            // the zeroing of small interior components happens in the quantiser, which
            // reads the inner tile only
        }
    }

    {                                                             // pipeline.c:407-421, 500-506
        QuantArgs q{};
        q.f = f; q.out = d_out; q.hy = hy; q.hx = hx;
        q.iz0 = z0 - rz0; q.iy0 = y0 - ry0; q.ix0 = x0 - rx0;
        q.tz = tz; q.ty = ty; q.tx = tx;
        q.gz0 = z0; q.gy0 = y0; q.gx0 = x0;
        q.no_dither = c->no_dither;
        q.norm = c->have_norm && c->norm_hi > c->norm_lo;
        q.midf = 0.5f * (float)(c->norm_lo + c->norm_hi) * (1.0f / 255.0f);
        q.k = q.norm ? (2.0f * 0.375f) * 255.0f / (float)(c->norm_hi - c->norm_lo) : 0.0f;
        const bool cc = c->do_air_zero && c->air_min_component > 0;
        q.lab = cc ? w.lab.as<int>() : nullptr;
        q.info = cc ? w.info.as<unsigned>() : nullptr;
        q.min_size = c->air_min_component;
        if (tn) {
            k_tile_quant<<<grid_rows(tx, ty, tz), row_threads(tx), 0, st>>>(q);
            TRY(cudaGetLastError());
            launches++;
        }
        fy_prof_mark(st, "tile.quant");
    }
    TRY(cudaMemcpyAsync(hctl, ctl, sizeof(TileCtl), cudaMemcpyDeviceToHost, st));
    TRY(cudaStreamSynchronize(st));
    fy::count_launch(launches);
    if (hctl->err) return fail(FY_ETIMEDOUT, "%s: connected-component walk exceeded %d steps", what, kUfMaxIter);
    if (c->do_air_zero) {
        for (int i = 0; i < 256; i++) w.hist[i] = hctl->hist[i];
        for (int i = 0; i < 3; i++) w.cuts[i] = hctl->cuts[i];
        w.have_state = true;
    }
    if (all_air) *all_air = 0;
    return FY_OK;
}

int check_geometry(const fy_pipeline_cfg* c, const void* in, const void* out, long rz0, long ry0, long rx0, long hz,
                   long hy, long hx, long z0, long y0, long x0, long tz, long ty, long tx, const char* what) {
    if (!c || !in || !out) return fail(FY_EINVAL, "%s: null pointer", what);
    if (hz < 1 || hy < 1 || hx < 1 || tz < 0 || ty < 0 || tx < 0)
        return fail(FY_EINVAL, "%s: bad dims %ldx%ldx%ld / %ldx%ldx%ld", what, hz, hy, hx, tz, ty, tx);
    if (z0 < rz0 || y0 < ry0 || x0 < rx0 || z0 + tz > rz0 + hz || y0 + ty > ry0 + hy || x0 + tx > rx0 + hx)
        return fail(FY_EINVAL, "%s: inner tile outside the buffer", what);
    if ((double)hz * hy * hx >= 2147483647.0 || hy > 65535 || ty > 65535)
        return fail(FY_EUNSUPPORTED, "%s: buffer %ldx%ldx%ld too large for one tile", what, hz, hy, hx);
    if (c->do_deconv && (hz > INT32_MAX || hy > INT32_MAX || hx > INT32_MAX))
        return fail(FY_EUNSUPPORTED, "%s: dims", what);
    return FY_OK;
}

}  // namespace

extern "C" double fy_valley_depth(const long hist[256], int* dark_out, int* light_out, int* valley_out) {
    return valley_depth_hd(hist, dark_out, light_out, valley_out);
}

extern "C" int fy_gpu_process_buffer(const fy_pipeline_cfg* cfg, const unsigned char* d_u8, long rz0, long ry0,
                                     long rx0, long hz, long hy, long hx, long z0, long y0, long x0, long tz, long ty,
                                     long tx, long vol_y, long vol_x, unsigned char* d_out, int* all_air,
                                     void* stream) {
    fy::enter();
    const char* what = "fy_gpu_process_buffer";
    int rc = check_geometry(cfg, d_u8, d_out, rz0, ry0, rx0, hz, hy, hx, z0, y0, x0, tz, ty, tx, what);
    if (rc) return rc;
    if ((rc = fy::ensure_ctx())) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    fy::ws_acquire(st);
    rc = tile_chain(cfg, d_u8, rz0, ry0, rx0, hz, hy, hx, z0, y0, x0, tz, ty, tx, vol_y, vol_x, d_out, all_air, st,
                    what);
    fy::ws_release(st);
    return rc;
}

extern "C" int fy_process_buffer(const fy_pipeline_cfg* cfg, const unsigned char* u8buf, long rz0, long ry0,
                                 long rx0, long hz, long hy, long hx, long z0, long y0, long x0, long tz, long ty,
                                 long tx, long vol_y, long vol_x, unsigned char* out, int* all_air) {
    fy::enter();
    const char* what = "fy_process_buffer";
    int rc = check_geometry(cfg, u8buf, out, rz0, ry0, rx0, hz, hy, hx, z0, y0, x0, tz, ty, tx, what);
    if (rc) return rc;
    if ((rc = fy::ensure_ctx())) return rc;
    fy::ThreadCtx& c = ctx();
    cudaStream_t st = c.st;
    TileWs& w = tws;
    const size_t hn = (size_t)hz * hy * hx, tn = (size_t)tz * ty * tx;
    fy::ws_acquire(st);
    cudaError_t e;
    if ((e = w.u8.ensure(hn)) != cudaSuccess || (e = w.out.ensure(tn ? tn : 1)) != cudaSuccess)
        return fail_cuda(e, what);
    // Pageable host buffers go through this thread's pinned staging, so that the copies are
    // plain DMA and the threads of a worker pool do not serialise on the driver's staging.
    const bool pin_in = fy::is_pinned(u8buf), pin_out = fy::is_pinned(out);
    const void* src = u8buf;
    if (!pin_in) {
        if ((e = w.hin.ensure(hn)) != cudaSuccess) return fail_cuda(e, what);
        memcpy(w.hin.p, u8buf, hn);
        src = w.hin.p;
    }
    if ((e = cudaMemcpyAsync(w.u8.p, src, hn, cudaMemcpyHostToDevice, st)) != cudaSuccess) return fail_cuda(e, what);
    rc = tile_chain(cfg, w.u8.as<uint8_t>(), rz0, ry0, rx0, hz, hy, hx, z0, y0, x0, tz, ty, tx, vol_y, vol_x,
                    w.out.as<uint8_t>(), all_air, st, what);
    if (rc) return rc;
    if (tn) {
        void* dst = out;
        if (!pin_out) {
            if ((e = w.hout.ensure(tn)) != cudaSuccess) return fail_cuda(e, what);
            dst = w.hout.p;
        }
        if ((e = cudaMemcpyAsync(dst, w.out.p, tn, cudaMemcpyDeviceToHost, st)) != cudaSuccess) return fail_cuda(e, what);
        if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return fail_cuda(e, what);
        if (!pin_out) memcpy(out, w.hout.p, tn);
    }
    fy::ws_release(st);
    return FY_OK;
}

void fy_tile_release() {
    TileWs& w = tws;
    for (fy::DevBuf* b : {&w.u8, &w.orig, &w.work, &w.alt, &w.t1, &w.t2, &w.sm, &w.lab, &w.info, &w.tab, &w.ctl, &w.out})
        b->release();
    w.pin.release();
    w.hin.release();
    w.hout.release();
    w.have_state = false;
}

extern "C" int fy_process_buffer_air_state(long hist[256], int cuts[3]) {
    const TileWs& w = tws;
    if (!w.have_state) return 1;
    if (hist) memcpy(hist, w.hist, sizeof w.hist);
    if (cuts) memcpy(cuts, w.cuts, sizeof w.cuts);
    return 0;
}
