#pragma once
// fy_deconv.cuh -- fused half-spectrum Wiener deconvolution (fy_deconvolve /
// fy_deconvolve_matched, paganin.c:152-342) as five HBM passes:
//
//   P1 X  : gather rows (u8 dewindow or f32) with reflect padding in x, two rows per
//           complex FFT, untangle -> half-spectrum rows         (paganin.c:165-194)
//   P2 Y  : forward over py for each stored z plane, reflect/zero rows gathered on load
//   P3 Z  : forward over pz (reflected planes gathered on load), radial weight from the
//           4096-entry LUT over u = f^2 with linear interpolation (paganin.c:212-244),
//           inverse over pz, store only the z < nz planes that survive the crop
//   P4 Y  : inverse for z < nz, store only rows y < ny          (paganin.c:254-260)
//   P5 X  : two-for-one C2R of surviving rows, x 1/(pz*py*px), crop (paganin.c:262-289)
//
// Algorithmic traffic at p = n (no padding): P1 4+4 (1+4 from u8), P2 8, P3 8, P4 8,
// P5 4+4 bytes per voxel.
//
// Kernels take N > 0 for a compile-time FFT plan of length N on their axis (instantiated
// for the common padded sizes in fy_deconv_ct_*.cu, compiled in parallel), or N = 0 for the
// runtime plan (fy_deconv.cu). fy_deconv_pass<N> enqueues one of the five passes.
#include "fy_internal.h"

namespace {
// Line transform with a compile-time plan when N > 0 (n == N, pitch PS), else the
// runtime plan `pl` with pitch ps.
constexpr int ct_pitch(int n) { return n > 0 ? ct_tile_lines(n) : 0; }
constexpr int ct_e(int n) { return n % 3 == 0 ? (n >= 24 ? 24 : n) : (n >= 16 ? 16 : n); }
template <int N, int E, int PS, int SIGN, class LD, class ST>
FY_D void fft_line(float2* __restrict__ sline, int ps, int tl, const FftPlan& pl, const float2* __restrict__ tw,
                   LD ld, ST st) {
    if constexpr (N > 0) line_fft_ct<N, E, PS, SIGN>(sline, tl, tw, ld, st);
    else line_fft<E>(sline, ps, tl, pl, tw, (float)SIGN, ld, st);
}
// A column pass's transform whose first pass reads global memory: with a compile-time plan
// the first pass's loads are issued before `prologue` fills the tile's shared tables, so the
// two latencies overlap and one barrier covers both (the runtime plan: prologue, barrier,
// transform, as before).
template <int N, int E, int PS, int SIGN, class LD, class PRO, class ST>
FY_D void fft_line_pre(float2* __restrict__ sline, int ps, int tl, const FftPlan& pl, const float2* __restrict__ tw,
                       LD ld, PRO prologue, ST st) {
    if constexpr (N > 0) {
        float2 v[E];
        ct_load<N, E, ct_radix(N, 0), PS>(v, tl, ld);
        prologue();
        __syncthreads();
        ct_passes<N, E, PS, SIGN, 0>(v, sline, tl, tw, st);
    } else {
        prologue();
        __syncthreads();
        line_fft<E>(sline, ps, tl, pl, tw, (float)SIGN, ld, st);
    }
}
// Threads per CTA never exceed W*n/E: 512 for 2^k lines (E=16), 256 for 3*2^k (E=24).
template <int E> struct KB { static constexpr int nt = (E % 3 == 0) ? 256 : 512; };
// Lines per tile of a column pass with a compile-time length N: the FFT core's tile
// (ct_tile_lines; N = 0: the runtime plan's, fy_tile_shape), or with NARROW 8 lines of 512
// points (256 threads, four CTAs per SM), so one CTA's loads overlap three others' transforms.
// Measured at 512^3: the forward Y pass 266 -> 253 us narrow; the inverse Y pass unchanged;
// the Z pass 426 -> 466 us (its transform pair per tile keeps the SM busy either way).
template <int N, int E, bool NARROW> struct YZ {
    static constexpr bool on = NARROW && N == 512;
    static constexpr int lines = on ? 8 : ct_pitch(N);
    static constexpr int nt = on ? 256 : KB<E>::nt;
    static constexpr int minb = on ? 4 : 2;
};
template <int N, bool NARROW> TileShape yz_tile_shape(int n) {
    if constexpr (YZ<N, 16, NARROW>::on) {
        TileShape t;
        t.W = YZ<N, 16, NARROW>::lines;
        t.wlog = fy_log2i(t.W);
        t.E = 16;
        t.NT = t.W * N / t.E;
        return t;
    } else {
        return fy_tile_shape(n);
    }
}


// Thread -> (line l, thread-in-line tl) with the line index fastest.
struct Lane {
    int l, tl;
    FY_D Lane(int wlog) : l(threadIdx.x & ((1 << wlog) - 1)), tl(threadIdx.x >> wlog) {}
};

// ---------------------------------------------------------------- P1
// Rows q = z*ny + y (z < nz, y < ny) paired (2m, 2m+1) into one complex line; a CTA owns W
// lines, staged line-major in shared memory (pitch px+1, odd: conflict-free for the FFT's
// line-strided accesses). Each thread loads the same VEC-wide chunk of both rows of a line
// pair, so it writes VEC consecutive complex values; reflect padding is filled from the
// staged line afterwards.
// Half-spectrum row offsets of the 2W rows (two per line) of a row tile, computed once per
// CTA: row q = z*ny + y sits at (z*py + y)*hxp; -1 past the last row.
FY_D void row_offsets(long long* off, long q0, int W, long Q, const SpecGeom& g) {
    for (int i = threadIdx.x; i < 2 * W; i += blockDim.x) {
        const long q = q0 + i;
        const int qi = (int)q;                          // nz*ny < 2^31 (each padded axis <= 4096)
        off[i] = q < Q ? ((long long)(qi / g.ny) * g.py + (qi % g.ny)) * g.hxp : -1;
    }
}

template <class T, int VEC> struct VecLoad;
template <> struct VecLoad<float, 4> {
    static FY_D void run(const float* p, float* v) {
        const float4 x = __ldg(reinterpret_cast<const float4*>(p));
        v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
    }
};
template <> struct VecLoad<uint8_t, 4> {
    static FY_D void run(const uint8_t* p, float* v) {
        const uchar4 x = __ldg(reinterpret_cast<const uchar4*>(p));
        v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
    }
};
template <class T> struct VecLoad<T, 1> {
    static FY_D void run(const T* p, float* v) { v[0] = (float)__ldg(p); }
};

// ---- bulk staging of P1's u8 rows: one thread copies the CTA's rows (one contiguous run,
// 16-byte aligned) with cp.async.bulk onto an mbarrier; every thread waits on it, bounded. A
// wait that gives up raises dc_timeout (reported by fy_gpu_kernel_timeouts), waits once more
// (bounded) for the copy in flight and leaves the CTA's lines unwritten.
static __device__ int dc_timeout;      // set when a bounded wait expires (never expected)
constexpr int kDcWaitSpins = 1 << 20;
FY_D unsigned dc_smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
FY_D bool dc_wait(unsigned long long* bar, unsigned parity) {
    for (int i = 0; i < kDcWaitSpins; ++i) {
        unsigned ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(dc_smem_u32(bar)), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}
FY_D void dc_bulk_rows(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(dc_smem_u32(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(dc_smem_u32(bar)), "r"(bytes)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n"
                 ::"r"(dc_smem_u32(dst)), "l"(src), "r"(bytes), "r"(dc_smem_u32(bar))
                 : "memory");
}
// Host: this unit's expired bulk waits (0 expected; -1 when unreadable).
inline int dc_timeouts() {
    int v = 0;
    if (cudaMemcpyFromSymbol(&v, dc_timeout, sizeof v) != cudaSuccess) { cudaGetLastError(); return -1; }
    return v;
}
// Host: whether P1 stages its u8 rows in bulk, and the extra shared memory it then needs.
inline bool dc_bulk_u8(const DeconvLaunch& d) {
    return d.src_u8 && d.g.nx % 16 == 0 && ((uintptr_t)d.src & 15) == 0;
}

template <int N, int E, class T, int VEC>
__global__ void __launch_bounds__(KB<E>::nt, 2) k_x_fwd(const T* __restrict__ src, float lo, float scale, int is_u8,
                                                        float2* __restrict__ spec, SpecGeom g,
                                                        const __grid_constant__ FftPlan pl,
                                                        const float2* __restrict__ tw, int wlog, FastDiv dchunk,
                                                        FastDiv dhx, FastDiv dpad) {
    fy_pdl_wait();
    extern __shared__ float4 smem4[];
    const int W = 1 << wlog, LPX = g.px + 1;
    float2* s = reinterpret_cast<float2*>(smem4);
    float2* stw = s + W * LPX;
    __shared__ long long soff[2 * 16];
    const long Q = (long)g.nz * g.ny;
    const long q0 = (long)blockIdx.x * 2 * W;
    // u8 rows in bulk (dc_bulk_u8 on the host decides the same and sizes the staging area)
    const bool bulk = sizeof(T) == 1 && VEC == 4 && is_u8 && (g.nx & 15) == 0 && ((uintptr_t)src & 15) == 0;
    __shared__ __align__(8) unsigned long long xbar;
    const unsigned char* su8 =
        reinterpret_cast<const unsigned char*>((reinterpret_cast<uintptr_t>(stw + pl.n) + 15) & ~(uintptr_t)15);
    if (bulk && threadIdx.x == 0) {
        const long nrows = Q - q0 < 2 * W ? Q - q0 : 2 * W;
        dc_bulk_rows(const_cast<unsigned char*>(su8), src + q0 * g.nx, (unsigned)(nrows * g.nx), &xbar);
    }
    load_twiddles(stw, tw, pl.n);
    row_offsets(soff, q0, W, Q, g);
    if (bulk) {
        __syncthreads();                               // the barrier is initialised
        if (__syncthreads_or(!dc_wait(&xbar, 0u))) {
            if (threadIdx.x == 0) {
                atomicExch(&dc_timeout, 1);
                dc_wait(&xbar, 0u);                    // the copy in flight, bounded
            }
            __syncthreads();
            return;
        }
    }
    const int nch = g.nx / VEC;
    for (int it = threadIdx.x; it < W * nch; it += blockDim.x) {
        const int l = dchunk.div(it), x = (it - l * nch) * VEC;
        const long qa = q0 + 2 * l, qb = qa + 1;
        float va[VEC], vb[VEC];
#pragma unroll
        for (int j = 0; j < VEC; ++j) va[j] = vb[j] = 0.f;
        if (bulk) {                                    // rows 2l and 2l+1 of the staged run
            if (qa < Q) {
                const uchar4 u = *reinterpret_cast<const uchar4*>(su8 + (size_t)(2 * l) * g.nx + x);
                va[0] = u.x; va[1] = u.y; va[2 % VEC] = u.z; va[3 % VEC] = u.w;
            }
            if (qb < Q) {
                const uchar4 u = *reinterpret_cast<const uchar4*>(su8 + (size_t)(2 * l + 1) * g.nx + x);
                vb[0] = u.x; vb[1] = u.y; vb[2 % VEC] = u.z; vb[3 % VEC] = u.w;
            }
        } else {
            if (qa < Q) VecLoad<T, VEC>::run(src + qa * g.nx + x, va);
            if (qb < Q) VecLoad<T, VEC>::run(src + qb * g.nx + x, vb);
        }
        float2* dst = s + l * LPX + x;
#pragma unroll
        for (int j = 0; j < VEC; ++j) {
            float a = va[j], b = vb[j];
            if (is_u8) {                                   // fy_u8_to_phys, FMA as the reference build
                a = qa < Q ? __fmaf_rn(a, scale, lo) : 0.f;
                b = qb < Q ? __fmaf_rn(b, scale, lo) : 0.f;
            }
            dst[j] = make_float2(a, b);
        }
    }
    const int npad = g.px - g.nx;
    if (npad > 0) {
        __syncthreads();
        for (int it = threadIdx.x; it < W * npad; it += blockDim.x) {
            const int l = dpad.div(it), x = g.nx + (it - l * npad);
            s[l * LPX + x] = g.zero_pad ? make_float2(0.f, 0.f) : s[l * LPX + reflect_idx(x, g.nx)];
        }
    }
    __syncthreads();
    const Lane ln(wlog);
    float2* line = s + ln.l * LPX;
    fft_line<N, E, 1, -1>(line, 1, ln.tl, pl, stw,
                [&](int i) { return line[i]; },
                [&](int i, float2 v) { line[i] = v; });
    __syncthreads();
    for (int idx = threadIdx.x; idx < W * g.hx; idx += blockDim.x) {
        const int l = dhx.div(idx), k = idx - l * g.hx;
        const long long oa = soff[2 * l], ob = soff[2 * l + 1];
        if (oa < 0) continue;
        const int mk = k == 0 ? 0 : g.px - k;
        float2 A, B;
        untangle(s[l * LPX + k], s[l * LPX + mk], A, B);
        spec[oa + k] = A;
        if (ob >= 0) spec[ob + k] = B;
    }
}

// ---------------------------------------------------------------- P2
// CTA = (column tile of W half-spectrum columns, stored plane z). Pass-0 inputs come
// straight from global memory (W consecutive columns = one 8W-byte run per point);
// rows >= ny are the reflected (or zero) rows.
template <int N, int E>
__global__ void __launch_bounds__(YZ<N, E, true>::nt, YZ<N, E, true>::minb) k_y_fwd(float2* __restrict__ spec, SpecGeom g, const __grid_constant__ FftPlan pl,
                                                 const float2* __restrict__ tw, int wlog) {
    fy_pdl_wait();
    extern __shared__ float4 smem4[];
    const int W = 1 << wlog;
    float2* s = reinterpret_cast<float2*>(smem4);
    float2* stw = s + pl.n * W;
    const Lane ln(wlog);
    float2* col = spec + (size_t)blockIdx.y * g.py * g.hxp + blockIdx.x * W + ln.l;
    fft_line_pre<N, E, YZ<N, E, true>::lines, -1>(s + ln.l, W, ln.tl, pl, stw,
                [&](int i) {
                    const int ys = i < g.ny ? i : (g.zero_pad ? -1 : reflect_idx(i, g.ny));
                    return ys < 0 ? make_float2(0.f, 0.f) : col[(size_t)ys * g.hxp];
                },
                [&]() { load_twiddles(stw, tw, pl.n); },
                [&](int i, float2 v) { col[(size_t)i * g.hxp] = v; });
}

// ---------------------------------------------------------------- P3
// CTA = (column tile, row y). Forward over z (reflected planes gathered on load), radial
// LUT weight over the tile in shared memory, inverse over z, store z < nz.
template <int N, int E>
__global__ void __launch_bounds__(KB<E>::nt, 2) k_z_weight(float2* __restrict__ spec, SpecGeom g,
                                                       const __grid_constant__ FftPlan pl,
                                                       const float2* __restrict__ tw,
                                                       const float* __restrict__ lut,
                                                       const double* __restrict__ fz2,
                                                       const double* __restrict__ fy2,
                                                       const double* __restrict__ fx2, double us, int wlog) {
    fy_pdl_wait();
    extern __shared__ float4 smem4[];
    const int W = 1 << wlog;
    float2* s = reinterpret_cast<float2*>(smem4);
    float2* stw = s + pl.n * W;
    double* sfz = reinterpret_cast<double*>(stw + pl.n);
    double2* syx = reinterpret_cast<double2*>(sfz + pl.n);    // per column (fy^2, fx^2)
    const Lane ln(wlog);
    const int c0 = blockIdx.x * W;
    const size_t zstride = (size_t)g.py * g.hxp;
    float2* col = spec + (size_t)blockIdx.y * g.hxp + c0 + ln.l;
    // (issuing the first loads before these tables, as the Y passes do, measured 424 -> 434 us)
    load_twiddles(stw, tw, pl.n);
    for (int i = threadIdx.x; i < pl.n; i += blockDim.x) sfz[i] = fz2[i];
    for (int i = threadIdx.x; i < W; i += blockDim.x) {
        const bool in = c0 + i < g.hx;
        syx[i] = make_double2(in ? fy2[blockIdx.y] : 0.0, in ? __ldg(fx2 + c0 + i) : 0.0);
    }
    __syncthreads();
    fft_line<N, E, ct_pitch(N), -1>(s + ln.l, W, ln.tl, pl, stw,
                [&](int i) {
                    const int zs = i < g.nz ? i : (g.zero_pad ? -1 : reflect_idx(i, g.nz));
                    return zs < 0 ? make_float2(0.f, 0.f) : col[(size_t)zs * zstride];
                },
                [&](int z, float2 v) { s[z * W + ln.l] = v; });
    __syncthreads();
    // the weight of each point is applied as the inverse transform's first pass reads it (the
    // thread's own column, every point once), so the weighted tile needs no separate pass
    fft_line<N, E, ct_pitch(N), +1>(s + ln.l, W, ln.tl, pl, stw,
                [&](int i) {
                    const float2 v = s[i * W + ln.l];
                    const double2 yx = syx[ln.l];
                    const double t = ((sfz[i] + yx.x) + yx.y) * us;  // paganin.c:234-236
                    int ti = (int)t;
                    if (ti >= FY_LUT_N) ti = FY_LUT_N - 1;
                    // the table (16 KB, read-only) through L1 rather than copied per tile
                    const float l0 = __ldg(lut + ti), l1 = __ldg(lut + ti + 1);
                    const float w = l0 + (l1 - l0) * (float)(t - ti);
                    return make_float2(v.x * w, v.y * w);
                },
                [&](int z, float2 v) { if (z < g.nz) col[(size_t)z * zstride] = v; });
}

// ---------------------------------------------------------------- P4
template <int N, int E>
__global__ void __launch_bounds__(KB<E>::nt, 2) k_y_inv(float2* __restrict__ spec, SpecGeom g, const __grid_constant__ FftPlan pl,
                                                 const float2* __restrict__ tw, int keep_rows, int wlog) {
    fy_pdl_wait();
    extern __shared__ float4 smem4[];
    const int W = 1 << wlog;
    float2* s = reinterpret_cast<float2*>(smem4);
    float2* stw = s + pl.n * W;
    const Lane ln(wlog);
    float2* col = spec + (size_t)blockIdx.y * g.py * g.hxp + blockIdx.x * W + ln.l;
    fft_line_pre<N, E, ct_pitch(N), +1>(s + ln.l, W, ln.tl, pl, stw,
                [&](int i) { return col[(size_t)i * g.hxp]; },
                [&]() { load_twiddles(stw, tw, pl.n); },
                [&](int i, float2 v) { if (i < keep_rows) col[(size_t)i * g.hxp] = v; });
}

// ---------------------------------------------------------------- P5
// Line-major like P1; the two output rows of a line are written VEC floats at a time.
template <int N, int E, int VEC>
__global__ void __launch_bounds__(KB<E>::nt, 2) k_x_inv(const float2* __restrict__ spec, float* __restrict__ dst,
                                                        SpecGeom g, const __grid_constant__ FftPlan pl,
                                                        const float2* __restrict__ tw, float invN, int wlog,
                                                        FastDiv dchunk, FastDiv dhx) {
    fy_pdl_wait();
    extern __shared__ float4 smem4[];
    const int W = 1 << wlog, LPX = g.px + 1;
    float2* s = reinterpret_cast<float2*>(smem4);
    float2* stw = s + W * LPX;
    __shared__ long long soff[2 * 16];
    const long Q = (long)g.nz * g.ny;
    const long q0 = (long)blockIdx.x * 2 * W;
    load_twiddles(stw, tw, pl.n);
    row_offsets(soff, q0, W, Q, g);
    __syncthreads();
    const int hi_max = g.px - g.hx;                 // m in [1, px-hx] mirrors to px-m
    // kU rows' elements per thread are loaded before any is stored, so that many loads are in
    // flight per thread while the CTA waits for its tile
    constexpr int kU = 8;
    const int total = W * g.hx, step = blockDim.x;
    for (int base = threadIdx.x; base < total; base += kU * step) {
        float2 A[kU], B[kU];
        int L[kU], K[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const int idx = base + u * step;
            A[u] = B[u] = make_float2(0.f, 0.f);
            L[u] = -1;
            K[u] = 0;
            if (idx < total) {
                const int l = dhx.div(idx), k = idx - l * g.hx;
                const long long oa = soff[2 * l], ob = soff[2 * l + 1];
                L[u] = l;
                K[u] = k;
                if (oa >= 0) A[u] = __ldg(spec + oa + k);
                if (ob >= 0) B[u] = __ldg(spec + ob + k);
            }
        }
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            if (L[u] < 0) continue;
            const int l = L[u], k = K[u];
            s[l * LPX + k] = pack_lo(A[u], B[u]);
            if (k >= 1 && k <= hi_max) s[l * LPX + g.px - k] = pack_hi(A[u], B[u]);
        }
    }
    __syncthreads();
    const Lane ln(wlog);
    float2* line = s + ln.l * LPX;
    fft_line<N, E, 1, +1>(line, 1, ln.tl, pl, stw,
                [&](int i) { return line[i]; },
                [&](int i, float2 v) { line[i] = v; });
    __syncthreads();
    const int nch = g.nx / VEC;
    for (int it = threadIdx.x; it < W * nch; it += blockDim.x) {
        const int l = dchunk.div(it), x = (it - l * nch) * VEC;
        const long qa = q0 + 2 * l, qb = qa + 1;
        if (qa >= Q) continue;
        const float2* v = s + l * LPX + x;
        if (VEC == 4) {
            *reinterpret_cast<float4*>(dst + qa * g.nx + x) =
                make_float4(v[0].x * invN, v[1].x * invN, v[2].x * invN, v[3].x * invN);
            if (qb < Q)
                *reinterpret_cast<float4*>(dst + qb * g.nx + x) =
                    make_float4(v[0].y * invN, v[1].y * invN, v[2].y * invN, v[3].y * invN);
        } else {
            dst[qa * g.nx + x] = v[0].x * invN;
            if (qb < Q) dst[qb * g.nx + x] = v[0].y * invN;
        }
    }
}


// Enqueue pass `pass` (1..5) with the compile-time plan of length N (N > 0, that pass's axis
// length) or the runtime plans (N = 0).
template <int N>
cudaError_t fy_deconv_pass(int pass, const DeconvLaunch& d, cudaStream_t st) {
    const SpecGeom& g = d.g;
    const long Q = (long)g.nz * g.ny;
    auto with_e = [&](int n, auto&& body) -> cudaError_t {
        if constexpr (N > 0) return body(std::integral_constant<int, ct_e(N)>{});
        else return fy_with_e(fy_fft_e(n), body);
    };
    switch (pass) {
    case 1: {   // X forward, rows paired two per line (line-major staging)
        const TileShape t = fy_x_tile_shape(1, g.px);
        const size_t smem = (size_t)t.W * (g.px + 1) * sizeof(float2) + (size_t)g.px * sizeof(float2) +
                            (dc_bulk_u8(d) ? (size_t)2 * t.W * g.nx + 16 : 0);
        const unsigned grid = (unsigned)((Q + 2 * t.W - 1) / (2 * t.W));
        const int esz = d.src_u8 ? 1 : 4;
        const bool vec = g.nx % 4 == 0 && ((uintptr_t)d.src % (4 * esz)) == 0;
        const int pad = g.px - g.nx > 0 ? g.px - g.nx : 1;
        return with_e(g.px, [&](auto ec) -> cudaError_t {
            constexpr int E = decltype(ec)::value;
            cudaError_t e2 = cudaSuccess;
            const FastDiv dch(vec ? g.nx / 4 : g.nx), dhx(g.hx), dpad(pad);
#define FY_P1(T, V)                                                                                   \
            { auto k = k_x_fwd<N, E, T, V>;                                                           \
              if ((e2 = fy_smem_optin(k, smem)) != cudaSuccess) return e2;                            \
              if ((e2 = fy_launch_pdl(k, dim3(grid), dim3(t.NT), smem, st, (const T*)d.src, d.lo, d.scale,      \
                                      d.src_u8, d.spec, g, d.plx, d.twx, t.wlog, dch, dhx, dpad)) != cudaSuccess) \
                  return e2; }
            if (d.src_u8) { if (vec) FY_P1(uint8_t, 4) else FY_P1(uint8_t, 1) }
            else { if (vec) FY_P1(float, 4) else FY_P1(float, 1) }
#undef FY_P1
            return cudaGetLastError();
        });
    }
    case 2:     // Y forward over the stored planes
    case 4: {   // Y inverse, keep rows < ny
        const TileShape t = pass == 2 ? yz_tile_shape<N, true>(g.py) : yz_tile_shape<N, false>(g.py);
        const size_t smem = (size_t)g.py * t.W * sizeof(float2) + (size_t)g.py * sizeof(float2);
        dim3 grid(ceil_div_i(g.hx, t.W), g.nz);
        return with_e(g.py, [&](auto ec) -> cudaError_t {
            constexpr int E = decltype(ec)::value;
            if (pass == 2) {
                auto k = k_y_fwd<N, E>;
                cudaError_t e2 = fy_smem_optin(k, smem);
                if (e2 != cudaSuccess) return e2;
                if ((e2 = fy_launch_pdl(k, grid, dim3(t.NT), smem, st, d.spec, g, d.ply, d.twy, t.wlog)) != cudaSuccess)
                    return e2;
            } else {
                auto k = k_y_inv<N, E>;
                cudaError_t e2 = fy_smem_optin(k, smem);
                if (e2 != cudaSuccess) return e2;
                if ((e2 = fy_launch_pdl(k, grid, dim3(t.NT), smem, st, d.spec, g, d.ply, d.twy, g.ny, t.wlog)) !=
                    cudaSuccess)
                    return e2;
            }
            return cudaGetLastError();
        });
    }
    case 3: {   // Z forward, weight, Z inverse
        const TileShape t = fy_tile_shape(g.pz);
        const size_t smem = (size_t)g.pz * t.W * sizeof(float2) + (size_t)g.pz * sizeof(float2) +
                            (size_t)g.pz * sizeof(double) + (size_t)t.W * sizeof(double2);
        dim3 grid(ceil_div_i(g.hx, t.W), g.py);
        return with_e(g.pz, [&](auto ec) -> cudaError_t {
            constexpr int E = decltype(ec)::value;
            auto k = k_z_weight<N, E>;
            cudaError_t e2 = fy_smem_optin(k, smem);
            if (e2 != cudaSuccess) return e2;
            if ((e2 = fy_launch_pdl(k, grid, dim3(t.NT), smem, st, d.spec, g, d.plz, d.twz, d.lut, d.fz2, d.fy2, d.fx2,
                                    d.us, t.wlog)) != cudaSuccess)
                return e2;
            return cudaGetLastError();
        });
    }
    case 5: {   // X C2R, crop, 1/N (line-major staging, vector stores when rows are 16-byte aligned)
        const TileShape t = fy_x_tile_shape(5, g.px);
        const size_t smem = (size_t)t.W * (g.px + 1) * sizeof(float2) + (size_t)g.px * sizeof(float2);
        const unsigned grid = (unsigned)((Q + 2 * t.W - 1) / (2 * t.W));
        const float invN = 1.0f / ((float)g.pz * (float)g.py * (float)g.px);   // paganin.c:263
        const bool vec = g.nx % 4 == 0 && ((uintptr_t)d.dst % 16) == 0;
        return with_e(g.px, [&](auto ec) -> cudaError_t {
            constexpr int E = decltype(ec)::value;
            cudaError_t e2 = cudaSuccess;
            const FastDiv dch(vec ? g.nx / 4 : g.nx), dhx(g.hx);
            if (vec) {
                auto k = k_x_inv<N, E, 4>;
                if ((e2 = fy_smem_optin(k, smem)) != cudaSuccess) return e2;
                if ((e2 = fy_launch_pdl(k, dim3(grid), dim3(t.NT), smem, st, (const float2*)d.spec, d.dst, g, d.plx,
                                        d.twx, invN, t.wlog, dch, dhx)) != cudaSuccess)
                    return e2;
            } else {
                auto k = k_x_inv<N, E, 1>;
                if ((e2 = fy_smem_optin(k, smem)) != cudaSuccess) return e2;
                if ((e2 = fy_launch_pdl(k, dim3(grid), dim3(t.NT), smem, st, (const float2*)d.spec, d.dst, g, d.plx,
                                        d.twx, invN, t.wlog, dch, dhx)) != cudaSuccess)
                    return e2;
            }
            return cudaGetLastError();
        });
    }
    default:
        return cudaErrorInvalidValue;
    }
}

// One case of a compile-time dispatch switch over axis lengths.
#define FY_DECONV_CT_CASE(NN) case NN: return fy_deconv_pass<NN>(pass, d, st);

}  // namespace
