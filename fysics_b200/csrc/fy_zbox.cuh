// fy_zbox.cuh -- z-sliding 3-D box sums of two per-voxel quantities.
//
// Shared by the noise model's local statistics (noise.c:20-67) and the two passes of the
// guided filter (guided.c:113-141). A CTA owns a 64 x 16 column tile and a chunk of z
// planes. Per input plane zi:
//   stage   the plane's tile plus halo (x0-4 .. x0+68, y0-R .. y0+16+R) lands in a 4-deep
//           shared-memory ring, zero-filled outside the volume; planes zi+1 .. zi+3 are in
//           flight while zi is reduced. 16-byte-aligned rows: one thread issues a 3-D tensor
//           copy (TMA) per plane, completing on the slot's mbarrier. Other shapes: cp.async
//           by all threads.
//   X phase one item = 4 output columns of one staged row: the row's values, the window
//           sums of both quantities, two float4 stores; (TY + 2R) x TX/4 items (the halo
//           rows included), one or two per thread.
//   Y phase one thread = one output column x 4 output rows. Its (2R+1)-plane z ring of
//           XY sums stays in registers and gives the box of plane zi - R to the epilogue.
// With TMA staging a plane takes one CTA barrier, between the X and Y phases: the X sums
// alternate between two arrays, and each thread waits on the plane's mbarrier itself.
// cp.async staging adds a barrier before the X phase (the copies of other threads).
// The two quantities travel as one float2 through all three window sums, so each tap is
// one paired FP32 add (__fadd2_rn: two IEEE round-to-nearest adds, the same results as two
// scalar adds in the same order) and the XY sums are stored and read as pairs.
// Epilogues (KIND):
//   ZB_NOISE      u = I - c (zero outside the volume), fixed divisor win^3: local mean and
//                 variance as in noise.c:41-61, with the tile shift c removing the FP32
//                 cancellation of E[I^2] - E[I]^2.
//                 With o2 set it also writes the guided filter's (mean, var) pair of the
//                 same window (ZB_GUIDED_AB's formulas): a chain whose noise window equals
//                 the guided window then needs no ZB_GUIDED_AB pass.
//   ZB_GUIDED_AB  u = I - c, box MEANS over the in-bounds window: the window sum times
//                 the reciprocal in-bounds counts 1.0f/(float)count of the three axes
//                 (guided.c:22-28): var = max(corr - mean^2, 0), a = var/(var + eps),
//                 b = mean*(1 - a) (guided.c:121-132) -> interleaved (a, b) pairs, one 8-byte
//                 store per voxel.
//   ZB_GUIDED_OUT box means of the (a, b) pairs -> out = box(a)*I + box(b)
//                 (guided.c:136-140), or the two means themselves for the decimated variant
//                 (guided.c:181-182). The pairs are staged as one interleaved field.
//   ZB_GUIDED_OUT_MV  the same from staged (mean, var) pairs, turned into (a, b) as the X
//                 phase reads them, with ZB_GUIDED_AB's expressions, so the output equals the
//                 two-pass filter's bit for bit (eps > 0). (Converting each staged pair once,
//                 in place, a plane ahead measured 19% slower: the extra wait and conversion
//                 sit before the plane's barrier.)
// Window sums are direct (2R+1)-tap float sums in ascending order, started from the first
// tap, so no running-sum chain accumulates error. Each output voxel is written once by one
// thread, and ZB_GUIDED_OUT reads the guide only at the voxel it writes, so out may alias
// the guide. ZB_GUIDED_OUT can also subtract the ring profile from its output (the same
// arithmetic as fy_dering_apply), which saves the separate read-modify-write pass.
#pragma once
#include <cuda.h>
#include <mutex>
#include <type_traits>
#include "fy_internal.h"

namespace fyzb {

constexpr int TX = 64, TY = 16, NT = 256, NS = 4;
constexpr int SXW = TX + 8;                 // staged row: x0 - 4 .. x0 + TX + 4 (R <= 4)
enum { ZB_NOISE = 0, ZB_GUIDED_AB = 1, ZB_GUIDED_OUT = 2, ZB_GUIDED_OUT_MV = 3 };
__host__ __device__ constexpr bool out_kind(int k) { return k == ZB_GUIDED_OUT || k == ZB_GUIDED_OUT_MV; }
// Resident CTAs per SM (two: a third CTA of the noise statistics, which fits at R <= 2,
// measured 45% slower per pass).
__host__ __device__ constexpr int ctas_per_sm(int r, int kind) { return (void)r, (void)kind, 2; }

struct Params {
    const float* f0;       // I (NOISE, GUIDED_AB) or interleaved (a, b) | (mean, var) pairs (OUT kinds)
    const float* guide;    // I (OUT kinds, out_mode 0)
    float* o0;             // mean | (a, b) pairs | out (or box(a))
    float* o1;             // var  | -      | box(b) (out_mode 1)
    float* o2;             // NOISE: guided (mean, var) pairs, optional
    const float* eps_ptr;  // GUIDED_AB, GUIDED_OUT_MV: device eps (overrides eps when set)
    float eps;
    float inv_wc;          // NOISE: 1/win^3
    int wci;               // NOISE: win^3
    int out_mode;
    int nz, ny, nx, zchunk;
    RingApply ra;          // GUIDED_OUT, out_mode 0: ring subtraction on the output (optional)
};

// C = floats per staged voxel: 1 (I) or 2 (interleaved a, b).
template <int R, int C>
struct Geo {
    static constexpr int NR = 2 * R + 1;
    static constexpr int SY = TY + 2 * R;
    static constexpr int RW = C * SXW;                           // floats per staged row
    static constexpr int STAGE = (SY * RW + 31) / 32 * 32;      // floats per staged plane (128 B multiple)
    static constexpr int XS = SY * TX;                          // float2 per X-sum array
    static constexpr int GUIDE = C == 2 ? TX * TY : 0;           // floats per staged guide tile
    // the staged planes, the guide tiles (output passes), two X-sum arrays (alternate planes),
    // the reciprocal counts, 128 B for alignment
    static constexpr size_t bytes = (size_t)(NS * (STAGE + GUIDE) + 4 * XS + TX + TY) * sizeof(float) + 128;
};

FY_D float recip_count(int p, int L, int r) {
    const int lo = p - r < 0 ? 0 : p - r;
    const int hi = p + r > L - 1 ? L - 1 : p + r;
    return 1.0f / (float)(hi - lo + 1);                       // guided.c:26 (IEEE division)
}

FY_D float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
FY_D float2 mul2(float2 a, float f) { return __fmul2_rn(a, make_float2(f, f)); }

// Guided (mean, var) of a window from its shifted sums and the product of the three axes'
// reciprocal in-bounds counts (guided.c:121-128).
FY_D float2 guided_mv(float2 sums, float rxyz, float c) {
    const float2 e = mul2(sums, rxyz);                 // E[I-c], E[(I-c)^2]
    float var = e.y - e.x * e.x;
    if (var < 0.f) var = 0.f;
    return make_float2(e.x + c, var);
}
// (a, b) from (mean, var) (guided.c:129-131). a = var/(var + eps) uses the fast division
// (<= 2 ulp for the denominators here, var + eps in [eps, ~1]); the a/b pass and the
// output pass from (mean, var) share it, so both forms of the filter agree bit for bit.
FY_D float2 guided_ab(float2 mv, float eps) {
    const float a = __fdividef(mv.y, mv.y + eps);
    return make_float2(a, mv.x * (1.0f - a));
}

FY_D void cp16(float* sdst, const float* gsrc, bool valid) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gsrc), "r"(valid ? 16 : 0)
                 : "memory");
}
FY_D void cp4(float* sdst, const float* gsrc, bool valid) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gsrc), "r"(valid ? 4 : 0)
                 : "memory");
}
FY_D void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
FY_D void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// ---- TMA staging: one thread copies a plane's tile with cp.async.bulk.tensor, completion
// tracked by one mbarrier per ring slot. Waits are bounded: on expiry the kernel raises
// zb_timeout, waits (bounded) for its own copies in flight and returns.
struct TmaMaps {
    CUtensorMap m0;                    // the staged field; 64-byte aligned type
    CUtensorMap m1;                    // output passes: the guide I, one TX x TY tile per plane
    int guide;                         // m1 is valid: the guide is staged with the planes
};
// The maps a tile's copies use: the kernel parameter's (one volume per launch) or a job's in
// device memory (the work-queue kernel).
struct TmaRef {
    const CUtensorMap* m0;
    const CUtensorMap* m1;
    int guide;
};
static __device__ int zb_timeout;      // set when a bounded wait expires (never expected)
constexpr int kWaitSpins = 1 << 20;
// Polls allowed for each CTA's first wait on its staged plane. Always kWaitSpins, except
// when a failure-detection test sets it lower to make that wait expire on purpose (the drain
// that follows keeps the full bound, so every copy issued still lands before the CTA exits).
static __device__ int zb_first_wait_polls = kWaitSpins;

FY_D unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
FY_D void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
FY_D void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
FY_D bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
FY_D bool mbar_wait_bounded(unsigned long long* bar, unsigned parity, int polls = kWaitSpins) {
    for (int i = 0; i < polls; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
FY_D void tma_load_3d(float* dst, const CUtensorMap* map, int x, int y, int z, unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

// Issue plane zi into slot `dst` (thread 0 only). The innermost coordinate C*(x0 - 4) is a
// multiple of 4 floats (16 bytes) as the tensor copy requires; rows and planes outside the
// volume, negative ones included, are zero-filled by the copy.
// gdst, when not null, receives the guide tile of output plane zi - R (x0 a multiple of TX:
// 16-byte aligned), completing on the same barrier.
template <int R, int C>
FY_D void tma_stage(float* dst, float* gdst, const TmaRef& tm, unsigned long long* bar, int zi, int x0, int y0) {
    using G = Geo<R, C>;
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");   // prior generic reads of the slot
    mbar_expect_tx(bar, (unsigned)((G::SY * G::RW + (gdst ? TX * TY : 0)) * sizeof(float)));
    tma_load_3d(dst, tm.m0, C * (x0 - 4), y0 - R, zi, bar);
    if (gdst) tma_load_3d(gdst, tm.m1, x0, y0, zi - R, bar);
}

// Stage plane zi into dst with cp.async; zero fill outside the volume. VEC: 16-byte copies
// (nx % 4 == 0, so a copy never straddles the volume's x edge).
template <int R, int C, bool VEC>
FY_D void stage_plane(float* dst, const Params& p, int zi, int x0, int y0) {
    using G = Geo<R, C>;
    const bool zin = zi >= 0 && zi < p.nz;
    const size_t pbase = (size_t)(zin ? zi : 0) * p.ny * p.nx;
    if (VEC) {
        constexpr int Q = G::RW / 4;
        for (int k = threadIdx.x; k < G::SY * Q; k += NT) {
            const int yy = k / Q, q = k - yy * Q;
            const int gy = y0 - R + yy, gx = x0 - 4 + 4 * q / C;
            const bool ok = zin && gy >= 0 && gy < p.ny && gx >= 0 && gx < p.nx;
            cp16(dst + yy * G::RW + 4 * q, ok ? p.f0 + (pbase + (size_t)gy * p.nx + gx) * C : p.f0, ok);
        }
    } else {
        for (int k = threadIdx.x; k < G::SY * G::RW; k += NT) {
            const int yy = k / G::RW, e = k - yy * G::RW;
            const int gy = y0 - R + yy, gx = x0 - 4 + e / C;
            const bool ok = zin && gy >= 0 && gy < p.ny && gx >= 0 && gx < p.nx;
            cp4(dst + k, ok ? p.f0 + (pbase + (size_t)gy * p.nx + gx) * C + (e - (e / C) * C) : p.f0, ok);
        }
    }
}

// One CTA's tile (bx, by) and z chunk bz of a box pass. Returns false when a bounded wait gave
// up (the CTA then raised zb_timeout and drained its copies). With TMA it leaves the slot
// barriers invalidated, so the CTA can run another tile.
template <int R, int KIND, bool VEC, bool TMA>
FY_D bool zbox_tile(const Params& p, const TmaRef& tm, int bx, int by, int bz, unsigned long long* bars) {
    constexpr int C = out_kind(KIND) ? 2 : 1;
    using G = Geo<R, C>;
    constexpr int NR = G::NR;
    extern __shared__ float4 zb_smem4[];
    float* stage = reinterpret_cast<float*>((reinterpret_cast<uintptr_t>(zb_smem4) + 127) & ~(uintptr_t)127);
    float* sguide = stage + NS * G::STAGE;                         // NS guide tiles (output passes)
    float2* xs = reinterpret_cast<float2*>(sguide + NS * G::GUIDE);  // X sums of both quantities, 2 x [SY][TX]
    float* rx = reinterpret_cast<float*>(xs + 2 * G::XS);
    float* ry = rx + TX;
    const int t = threadIdx.x;
    const int nz = p.nz, ny = p.ny, nx = p.nx;
    const int x0 = bx * TX, y0 = by * TY;
    const int zs = bz * p.zchunk, ze = min(nz, zs + p.zchunk);
    const size_t plane = (size_t)ny * nx;
    // per-tile shift: one constant for every window this CTA forms
    const float c = out_kind(KIND) ? 0.f : __ldg(p.f0 + (size_t)zs * plane + (size_t)y0 * nx + x0);
    float eps = p.eps;
    if ((KIND == ZB_GUIDED_AB || KIND == ZB_GUIDED_OUT_MV) && p.eps_ptr) eps = *p.eps_ptr;   // device noise model
    if (t < TX) rx[t] = x0 + t < nx ? recip_count(x0 + t, nx, R) : 0.f;
    if (t < TY) ry[t] = y0 + t < ny ? recip_count(y0 + t, ny, R) : 0.f;
    const bool cols_in = x0 - 4 >= 0 && x0 + TX + 4 <= nx;       // no column of the staged rows is outside
    const int zfirst = zs - R, zend = ze + R;
    int zissued = min(zfirst + NS - 2, zend - 1);                // thread 0: last plane whose copy it issued
    const int first_polls = TMA ? zb_first_wait_polls : 0;
    // the guide tile of output plane zi - R rides with staged plane zi when that output plane
    // is this CTA's (TMA output passes with an aligned guide)
    const bool gstage = TMA && out_kind(KIND) && p.out_mode == 0 && tm.guide;
    auto guide_slot = [&](int slot, int zi) -> float* {
        return gstage && zi - R >= zs && zi - R < ze ? sguide + slot * G::GUIDE : nullptr;
    };
    if (TMA) {
        if (t == 0) {
            for (int s = 0; s < NS; ++s) mbar_init(&bars[s], 1);
            asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        }
        __syncthreads();
        if (t == 0)
            for (int s = 0; s < NS - 1; ++s)
                if (zfirst + s < zend)
                    tma_stage<R, C>(stage + s * G::STAGE, guide_slot(s, zfirst + s), tm, &bars[s], zfirst + s, x0, y0);
    } else {
#pragma unroll
        for (int s = 0; s < NS - 1; ++s) {
            if (zfirst + s < zend) stage_plane<R, C, VEC>(stage + s * G::STAGE, p, zfirst + s, x0, y0);
            cp_commit();
        }
    }
    // Y-phase role: output column xc, output rows 4*rg .. 4*rg+3
    const int xc = t & (TX - 1), rg = t >> 6;
    const int gx = x0 + xc;
    int cyx[4];                                                   // NOISE: in-bounds XY window size
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int gy = y0 + 4 * rg + k;
        cyx[k] = (min(gy + R, ny - 1) - max(gy - R, 0) + 1) * (min(gx + R, nx - 1) - max(gx - R, 0) + 1);
    }
    // GUIDED_OUT: ring radius of this thread's 4 output voxels (dering.c:200-248)
    bool rings = false;
    int ri[4] = {0, 0, 0, 0};
    float rv[4] = {0.f, 0.f, 0.f, 0.f};                           // ring values of the cached slab
    long rslab = -1;
    long rlo = 1, rhi = 0;                                        // global z range of the cached ring slab
    const float rz_in = recip_count(R, 2 * R + 1, R);             // 1/(2R+1): interior planes
    if (out_kind(KIND) && p.out_mode == 0 && p.ra.ring) {
        rings = p.ra.have ? (*p.ra.have != 0) : true;
        const double gxd = (double)(p.ra.x0 + gx) - p.ra.cx;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const double gyd = (double)(p.ra.y0 + y0 + 4 * rg + k) - p.ra.cy;
            ri[k] = (int)(sqrt(gyd * gyd + gxd * gxd) + 0.5);
        }
    }
    float2 rz2[NR][4];                                            // z ring of XY sums
#pragma unroll
    for (int q = 0; q < NR; ++q)
#pragma unroll
        for (int k = 0; k < 4; ++k) rz2[q][k] = make_float2(0.f, 0.f);

    // The plane loop is unrolled by NR so the z ring rotates by naming: plane zi lands in
    // ring slot ph = (zi - zfirst) mod NR, and the window of plane zi - R is slots ph+1 ..
    // ph+NR (mod NR) in ascending z.
    for (int zi0 = zfirst; zi0 < zend; zi0 += NR) {
#pragma unroll
        for (int ph = 0; ph < NR; ++ph) {
            const int zi = zi0 + ph;
            if (zi >= zend) break;
            const int slot = (zi - zfirst) & (NS - 1);
            // TMA: no barrier before the X phase. Every thread passed the previous plane's
            // barrier, so plane zi - 1's slot is read out (thread 0 refills it) and the X sums
            // of plane zi - 2, which share this plane's array, are read out.
            bool ok = true;
            float2* xcur = xs;
            if (TMA) {
                ok = mbar_wait_bounded(&bars[slot], (unsigned)(((zi - zfirst) / NS) & 1),
                                       zi == zfirst ? first_polls : kWaitSpins);
                xcur = xs + ((zi - zfirst) & 1) * G::XS;
            } else {
                cp_wait<NS - 2>();
                __syncthreads();             // plane zi landed for every thread; xs free again
                const int zn = zi + NS - 1;
                if (zn < zend) stage_plane<R, C, VEC>(stage + ((zn - zfirst) & (NS - 1)) * G::STAGE, p, zn, x0, y0);
                cp_commit();
            }
            const int zo = zi - R;
            const bool emit = zo >= zs && zo < ze && gx < nx;
            const size_t obase = (size_t)(emit ? zo : 0) * plane + (size_t)(y0 + 4 * rg) * nx + gx;
            float gv[4] = {0.f, 0.f, 0.f, 0.f};
            if (out_kind(KIND) && p.out_mode == 0 && emit && !gstage) {   // issued early, used after the Y phase
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    if (y0 + 4 * rg + k < ny) gv[k] = __ldg(p.guide + obase + (size_t)k * nx);
            }
            const float* sp = stage + slot * G::STAGE;
            const bool zin = zi >= 0 && zi < nz;
            // X phase, every staged row (the TY output rows and the 2R halo rows): an item is IW
            // output columns of one row starting at xs, P[j] = both quantities of staged column
            // x0 - 4 + xs + j. Each thread takes one 4-column item; the 2R halo rows' 4-column
            // items left over are split into 2-column halves spread over the first threads, so
            // the phase that gates the plane's barrier costs 1.5 item times instead of 2.
            // (One-column items for the halo rows cost (2R+1) taps' conversions per output
            // instead of (4+2R)/4; every split keeps the same taps in the same order.)
            auto xitem = [&](auto wc, int yy, int xs) {
                constexpr int IW = decltype(wc)::value;
                float2 P[12];
                if (C == 2) {                    // interleaved pairs: float4 = two columns
                    const float* row = sp + yy * G::RW + 2 * xs;
#pragma unroll
                    for (int j2 = (4 - R) / 2; j2 <= (IW + 3 + R) / 2; ++j2) {
                        const float4 v = *reinterpret_cast<const float4*>(row + 4 * j2);
                        P[2 * j2] = make_float2(v.x, v.y);
                        P[2 * j2 + 1] = make_float2(v.z, v.w);
                    }
                    if (KIND == ZB_GUIDED_OUT_MV) {          // (mean, var) -> (a, b)
#pragma unroll
                        for (int j = 4 - R; j < IW + 4 + R; ++j) P[j] = guided_ab(P[j], eps);
                    }
                } else {
                    const float* row = sp + yy * G::RW + xs;
                    float q1[12];
                    if (IW == 4) {                   // xs a multiple of 4: 16-byte loads
#pragma unroll
                        for (int j = 0; j < 3; ++j) {
                            const float4 v = *reinterpret_cast<const float4*>(row + 4 * j);
                            q1[4 * j] = v.x; q1[4 * j + 1] = v.y; q1[4 * j + 2] = v.z; q1[4 * j + 3] = v.w;
                        }
                    } else {                         // xs even: 8-byte loads
#pragma unroll
                        for (int j = (4 - R) & ~1; j < IW + 4 + R; j += 2) {
                            const float2 v = *reinterpret_cast<const float2*>(row + j);
                            q1[j] = v.x; q1[j + 1] = v.y;
                        }
                    }
                    const int gy = y0 - R + yy;
                    const bool rin = zin && gy >= 0 && gy < ny;
                    if (cols_in) {
                        const float cs = rin ? c : 0.f;           // outside rows were staged as 0
#pragma unroll
                        for (int j = 4 - R; j < IW + 4 + R; ++j) q1[j] = q1[j] - cs;
                    } else {
#pragma unroll
                        for (int j = 4 - R; j < IW + 4 + R; ++j) {
                            const int gxj = x0 - 4 + xs + j;
                            q1[j] = (rin && gxj >= 0 && gxj < nx) ? q1[j] - c : 0.f;
                        }
                    }
#pragma unroll
                    for (int j = 4 - R; j < IW + 4 + R; ++j) P[j] = make_float2(q1[j], q1[j] * q1[j]);
                }
                float2 o[IW];
#pragma unroll
                for (int k = 0; k < IW; ++k) {
                    float2 sm = P[4 + k - R];
#pragma unroll
                    for (int j = 5 + k - R; j <= 4 + k + R; ++j) sm = add2(sm, P[j]);
                    if (out_kind(KIND)) sm = mul2(sm, rx[xs + k]);
                    o[k] = sm;
                }
                float4* dst = reinterpret_cast<float4*>(xcur + yy * TX + xs);
#pragma unroll
                for (int k2 = 0; k2 < IW / 2; ++k2) dst[k2] = make_float4(o[2 * k2].x, o[2 * k2].y, o[2 * k2 + 1].x, o[2 * k2 + 1].y);
            };
            constexpr int NITEM = G::SY * (TX / 4), NHALF = 2 * (NITEM - NT);
            static_assert(NITEM >= NT && NHALF <= NT, "one full and at most one half item per thread");
            xitem(std::integral_constant<int, 4>{}, t >> 4, (t & 15) << 2);
            if (t < NHALF) {
                const int it = NT + (t >> 1);
                xitem(std::integral_constant<int, 2>{}, it >> 4, ((it & 15) << 2) + 2 * (t & 1));
            }
            if (TMA) {
                if (__syncthreads_or(!ok)) {      // plane zi never landed: flag, drain, return
                    if (t == 0) {
                        atomicExch(&zb_timeout, 1);
                        for (int zq = zi; zq <= zissued; ++zq)          // loads issued so far
                            mbar_wait_bounded(&bars[(zq - zfirst) & (NS - 1)], (unsigned)(((zq - zfirst) / NS) & 1));
                    }
                    __syncthreads();
                    return false;
                }
                // Refill the slot of plane zi - 1: past this barrier every thread has finished
                // plane zi - 1, its staged rows and its guide tile alike.
                const int zn = zi + NS - 1;
                if (t == 0 && zn < zend) {
                    const int sn = (zn - zfirst) & (NS - 1);
                    tma_stage<R, C>(stage + sn * G::STAGE, guide_slot(sn, zn), tm, &bars[sn], zn, x0, y0);
                    zissued = zn;
                }
            } else {
                __syncthreads();
            }
            // Y phase -> ring slot ph
            {
                float2 a[4 + 2 * R];
#pragma unroll
                for (int j = 0; j < 4 + 2 * R; ++j) a[j] = xcur[(4 * rg + j) * TX + xc];
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    float2 sm = a[k];
#pragma unroll
                    for (int j = 1; j <= 2 * R; ++j) sm = add2(sm, a[k + j]);
                    if (out_kind(KIND)) sm = mul2(sm, ry[4 * rg + k]);
                    rz2[ph][k] = sm;
                }
            }
            if (!emit) continue;
            if (out_kind(KIND) && rings) {                        // this plane's ring slab (dering.c:212-215)
                const long zg = p.ra.z0 + zo;
                if (!(zg >= rlo && zg < rhi)) {                   // left the cached slab's planes: divide once
                    const long q = zg / p.ra.slab_z;
                    rlo = q * p.ra.slab_z;
                    rhi = rlo + p.ra.slab_z;
                    long sl = q;
                    if (sl < 0) sl = 0;
                    if (sl >= p.ra.nslab) sl = p.ra.nslab - 1;
                    if (sl != rslab) {
                        rslab = sl;
#pragma unroll
                        for (int k = 0; k < 4; ++k)
                            rv[k] = ri[k] < p.ra.nr ? __ldg(p.ra.ring + (size_t)sl * p.ra.nr + ri[k]) : 0.f;
                    }
                }
            }
            const bool zint = zo >= R && zo + R <= nz - 1;        // the window's planes all inside
            const float rz = zint ? rz_in : recip_count(zo, nz, R);
            const int cz = zint ? 2 * R + 1 : min(zo + R, nz - 1) - max(zo - R, 0) + 1;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                if (y0 + 4 * rg + k >= ny) continue;
                float2 sm = rz2[(ph + 1) % NR][k];
#pragma unroll
                for (int q = 2; q <= NR; ++q) sm = add2(sm, rz2[(ph + q) % NR][k]);
                const float s1 = sm.x, s2 = sm.y;
                const size_t o = obase + (size_t)k * nx;
                if (KIND == ZB_NOISE) {
                    const int nini = cz * cyx[k];
                    const float nin = (float)nini;
                    // raw sums: S1 = S1' + nin*c, S2 = S2' + 2c*S1' + nin*c^2
                    const float m = (s1 + nin * c) * p.inv_wc;
                    float v;
                    if (nini == p.wci) {                           // interior: shifted, cancellation-free
                        const float e1 = s1 * p.inv_wc;
                        v = s2 * p.inv_wc - e1 * e1;
                    } else {
                        v = (s2 + 2.0f * c * s1 + nin * c * c) * p.inv_wc - m * m;
                    }
                    if (v < 0.f) v = 0.f;
                    p.o0[o] = m;
                    p.o1[o] = v;
                    if (p.o2)
                        reinterpret_cast<float2*>(p.o2)[o] = guided_mv(sm, rx[xc] * ry[4 * rg + k] * rz, c);
                } else if (KIND == ZB_GUIDED_AB) {
                    reinterpret_cast<float2*>(p.o0)[o] = guided_ab(guided_mv(sm, rx[xc] * ry[4 * rg + k] * rz, c), eps);
                } else {
                    const float2 mab = mul2(sm, rz);
                    if (p.out_mode == 0) {
                        const float g = gstage ? sguide[slot * G::GUIDE + (4 * rg + k) * TX + xc] : gv[k];
                        float w = mab.x * g + mab.y;
                        if (rings && w > 0.f && ri[k] < p.ra.nr) {     // masked voxels untouched
                            const float w2 = w - p.ra.sc * rv[k];
                            w = w2 > 0.f ? w2 : 0.f;
                        }
                        p.o0[o] = w;
                    } else {
                        p.o0[o] = mab.x; p.o1[o] = mab.y;
                    }
                }
            }
        }
    }
    if (!TMA) cp_wait<0>();
    if (TMA) {                 // every copy issued was waited for: the barriers can be retired
        __syncthreads();
        if (t == 0)
            for (int s = 0; s < NS; ++s)
                asm volatile("mbarrier.inval.shared::cta.b64 [%0];\n" ::"r"(smem_u32(&bars[s])) : "memory");
        __syncthreads();
    }
    return true;
}

template <int R, int KIND, bool VEC, bool TMA>
__global__ void __launch_bounds__(NT, ctas_per_sm(R, KIND)) k_zbox(const __grid_constant__ Params p, const __grid_constant__ TmaMaps tm) {
    fy_pdl_wait();
    __shared__ __align__(8) unsigned long long bars[NS];
    const TmaRef tr{&tm.m0, &tm.m1, tm.guide};
    zbox_tile<R, KIND, VEC, TMA>(p, tr, blockIdx.x, blockIdx.y, blockIdx.z, bars);
}

// A box pass over many volumes: one job per volume (its parameters, its tensor maps in device
// memory, its tile counts and the index of its first work item; jobs in item order). The
// work items are (volume, tile, z chunk) in one index space; persistent CTAs (ctas_per_sm per
// SM) take the next item from *next until none is left, so volumes of any size share one
// launch with no tail per volume. Each tile's arithmetic is the one-volume kernel's, so the
// results are bit-identical to it. TMA staging only (every volume's rows 16-byte aligned).
struct BoxJob {
    CUtensorMap m0, m1;                // 64-byte aligned
    Params p;
    int guide;                         // m1 valid
    int tx, ty;                        // tiles along x and y
    long long first;                   // first work item
};
template <int R, int KIND>
__global__ void __launch_bounds__(NT, ctas_per_sm(R, KIND)) k_zbox_queue(const BoxJob* __restrict__ jobs, int njobs,
                                                                        long long total,
                                                                        unsigned long long* __restrict__ next) {
    fy_pdl_wait();
    __shared__ __align__(8) unsigned long long bars[NS];
    __shared__ long long s_item;
    __shared__ __align__(16) Params s_p;
    for (;;) {
        if (threadIdx.x == 0) s_item = (long long)atomicAdd(next, 1ull);
        __syncthreads();
        const long long item = s_item;
        __syncthreads();                                  // read by every thread before the next ticket
        if (item >= total) return;
        int lo = 0, hi = njobs - 1;                       // the last job with first <= item
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (jobs[mid].first <= item) lo = mid; else hi = mid - 1;
        }
        const BoxJob& J = jobs[lo];
        const long long local = item - J.first;
        const int bx = (int)(local % J.tx), by = (int)((local / J.tx) % J.ty), bz = (int)(local / ((long long)J.tx * J.ty));
        if (threadIdx.x == 0) {          // the maps were written by a copy: acquire them for the tensor proxy
            asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;\n" ::"l"(&J.m0) : "memory");
            asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;\n" ::"l"(&J.m1) : "memory");
        }
        static_assert(sizeof(Params) % 4 == 0, "word copy");
        for (int i = threadIdx.x; i < (int)(sizeof(Params) / 4); i += blockDim.x)   // the job's parameters,
            reinterpret_cast<int*>(&s_p)[i] = reinterpret_cast<const int*>(&J.p)[i]; // read from shared memory
        __syncthreads();
        const TmaRef tr{&J.m0, &J.m1, J.guide};
        if (!zbox_tile<R, KIND, true, true>(s_p, tr, bx, by, bz, bars)) return;
    }
}

// Tiles and z chunks (fy_box_default_chunks, fy_internal.h). The chunk count is fixed by the
// shape, the kind's residency and the SM count alone: each chunk takes its variance shift
// from its first plane, so another chunking would round the sums differently.
inline dim3 grid_for(int kind, int nz, int ny, int nx, int r, int sms, int& zchunk) {
    const int tx = (nx + TX - 1) / TX, ty = (ny + TY - 1) / TY;
    const int nc = fy_box_default_chunks(nz, ny, nx, r, sms, ctas_per_sm(r, kind));
    zchunk = (nz + nc - 1) / nc;
    return dim3(tx, ty, (nz + zchunk - 1) / zchunk);
}

// Tensor map of one f32 volume field of c floats per voxel for the TMA staging: a box of
// bx voxels x by rows x 1 plane (the staged rows: SXW x SY; the guide: TX x TY), zero fill
// outside. The encoder comes from the
// driver through the runtime, so the library needs no link-time driver dependency. Returns
// false when unavailable.
inline bool make_tma_map(CUtensorMap* m, const float* base, int nz, int ny, int nx, int c, int bx, int by) {
    using EncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
    static EncodeFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeFn>(f);
        else
            cudaGetLastError();
    });
    if (!fn || ((uintptr_t)base & 15) || (nx % 4)) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)nx * c, (cuuint64_t)ny, (cuuint64_t)nz};
    const cuuint64_t strides[2] = {(cuuint64_t)nx * c * 4, (cuuint64_t)nx * ny * c * 4};
    const cuuint32_t box[3] = {(cuuint32_t)(bx * c), (cuuint32_t)by, 1};
    const cuuint32_t es[3] = {1, 1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims, strides, box, es,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int KIND, int R, bool VEC>
inline cudaError_t launch_r(const Params& p, dim3 grid, cudaStream_t st) {
    constexpr int C = out_kind(KIND) ? 2 : 1;
    const size_t smem = Geo<R, C>::bytes;
    TmaMaps tm;
    memset(&tm, 0, sizeof tm);
    const bool tma = VEC && make_tma_map(&tm.m0, p.f0, p.nz, p.ny, p.nx, C, SXW, Geo<R, C>::SY);
    if (tma && out_kind(KIND) && p.out_mode == 0 && p.guide)
        tm.guide = make_tma_map(&tm.m1, p.guide, p.nz, p.ny, p.nx, 1, TX, TY) ? 1 : 0;
    cudaError_t e;
    if (tma) {
        auto k = k_zbox<R, KIND, true, true>;
        if ((e = fy_smem_optin(k, smem)) != cudaSuccess) return e;
        return fy_launch_pdl(k, grid, dim3(NT), smem, st, p, tm);
    }
    auto k = k_zbox<R, KIND, VEC, false>;
    if ((e = fy_smem_optin(k, smem)) != cudaSuccess) return e;
    return fy_launch_pdl(k, grid, dim3(NT), smem, st, p, tm);
}

// The work-queue pass (k_zbox_queue). make_job fills one volume's job from its parameters
// (its z chunks as the one-volume launch picks them, so the results match it bit for bit) and
// returns its number of work items, or -1 when the volume cannot use TMA staging (rows not
// 16-byte aligned) or the encoder is unavailable.
template <int KIND, int R>
inline long long make_job_r(BoxJob& j, const Params& p, int sms, long long first) {
    constexpr int C = out_kind(KIND) ? 2 : 1;
    memset(&j, 0, sizeof j);
    j.p = p;
    const dim3 grid = grid_for(KIND, p.nz, p.ny, p.nx, R, sms, j.p.zchunk);
    if (p.nx % 4 || ((uintptr_t)p.f0 & 15)) return -1;
    if (!make_tma_map(&j.m0, p.f0, p.nz, p.ny, p.nx, C, SXW, Geo<R, C>::SY)) return -1;
    if (out_kind(KIND) && p.out_mode == 0 && p.guide)
        j.guide = make_tma_map(&j.m1, p.guide, p.nz, p.ny, p.nx, 1, TX, TY) ? 1 : 0;
    j.tx = (int)grid.x;
    j.ty = (int)grid.y;
    j.first = first;
    return (long long)grid.x * grid.y * grid.z;
}
template <int KIND>
inline long long make_job(BoxJob& j, const Params& p, int r, int sms, long long first) {
    switch (r) {
        case 1: return make_job_r<KIND, 1>(j, p, sms, first);
        case 2: return make_job_r<KIND, 2>(j, p, sms, first);
        case 3: return make_job_r<KIND, 3>(j, p, sms, first);
        case 4: return make_job_r<KIND, 4>(j, p, sms, first);
        default: return -1;
    }
}
// Launch the queue over njobs jobs in device memory (64-byte aligned) with `total` items;
// *next must hold 0 (stream order).
template <int KIND, int R>
inline cudaError_t launch_queue_r(const BoxJob* jobs, int njobs, long long total, unsigned long long* next, int sms,
                                  cudaStream_t st) {
    constexpr int C = out_kind(KIND) ? 2 : 1;
    const size_t smem = Geo<R, C>::bytes;
    auto k = k_zbox_queue<R, KIND>;
    cudaError_t e = fy_smem_optin(k, smem);
    if (e != cudaSuccess) return e;
    const long long want = (long long)sms * ctas_per_sm(R, KIND);
    const unsigned grid = (unsigned)(total < want ? (total > 0 ? total : 1) : want);
    return fy_launch_pdl(k, dim3(grid), dim3(NT), smem, st, jobs, njobs, total, next);
}
template <int KIND>
inline cudaError_t launch_queue(const BoxJob* jobs, int njobs, long long total, unsigned long long* next, int r,
                                int sms, cudaStream_t st) {
    switch (r) {
        case 1: return launch_queue_r<KIND, 1>(jobs, njobs, total, next, sms, st);
        case 2: return launch_queue_r<KIND, 2>(jobs, njobs, total, next, sms, st);
        case 3: return launch_queue_r<KIND, 3>(jobs, njobs, total, next, sms, st);
        case 4: return launch_queue_r<KIND, 4>(jobs, njobs, total, next, sms, st);
        default: return cudaErrorInvalidValue;
    }
}

// Number of bounded waits that expired in this translation unit's box passes (0 expected).
static inline int timeouts() {
    int v = 0;
    if (cudaMemcpyFromSymbol(&v, zb_timeout, sizeof v) != cudaSuccess) { cudaGetLastError(); return -1; }
    return v;
}

// Failure-detection tests: the polls allowed for each CTA's first wait (< 0: the normal
// bound); clears this translation unit's expiry flag. Synchronous.
static inline cudaError_t set_first_wait_polls(int polls) {
    const int v = polls < 0 ? kWaitSpins : polls, zero = 0;
    cudaError_t e = cudaMemcpyToSymbol(zb_first_wait_polls, &v, sizeof v);
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(zb_timeout, &zero, sizeof zero);
    return e;
}

// Enqueue one z-sliding box pass, radius r in [1, 4].
template <int KIND>
inline cudaError_t launch(Params p, int r, int sms, cudaStream_t st) {
    const dim3 grid = grid_for(KIND, p.nz, p.ny, p.nx, r, sms, p.zchunk);
    auto al = [](const void* q) { return ((uintptr_t)q & 15) == 0; };
    const bool vec = p.nx % 4 == 0 && al(p.f0);
    switch (r * 2 + (vec ? 1 : 0)) {
        case 2: return launch_r<KIND, 1, false>(p, grid, st);
        case 3: return launch_r<KIND, 1, true>(p, grid, st);
        case 4: return launch_r<KIND, 2, false>(p, grid, st);
        case 5: return launch_r<KIND, 2, true>(p, grid, st);
        case 6: return launch_r<KIND, 3, false>(p, grid, st);
        case 7: return launch_r<KIND, 3, true>(p, grid, st);
        case 8: return launch_r<KIND, 4, false>(p, grid, st);
        case 9: return launch_r<KIND, 4, true>(p, grid, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace fyzb
