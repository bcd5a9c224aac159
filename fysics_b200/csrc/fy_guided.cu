// fy_guided.cu -- 3-D self-guided filter (guided.c:113-241) and box mean (guided.c:19-106).
//
// Box semantics (guided.c:22-28, 35-98): the mean over the IN-BOUNDS part of a (2r+1)^3
// window, taken axis by axis, each axis dividing by its own clamped count with the
// reciprocal 1.0f/(float)count. Guided math per voxel (guided.c:121-135):
//   var = max(corr - mean^2, 0), a = var/(var + eps), b = mean*(1 - a),
//   out = box(a)*I + box(b).
//
// Fused path (r <= 4): one kernel per (16 x 32) output column tile that slides along z.
// Per input plane it stages I (+2r halo) in shared memory, forms the XY box means of
// (I - c) and (I - c)^2 over the a/b support, z-combines 2r+1 of those planes into
// mean/corr for the plane r behind, computes a,b there, XY-boxes them, and z-combines
// 2r+1 a/b planes into the output plane 2r behind. I is read from HBM once and out written
// once (8 B/voxel). The per-tile constant c (the tile's first in-volume sample) makes
// E[(I-c)^2] - E[I-c]^2 = E[I^2] - E[I]^2 exactly while removing most of the FP32
// cancellation that dominates the reference's error (guided.c:127); window sums are
// direct (2r+1)-tap float sums, so no long running-sum chain accumulates error.
//
// Generic path (any r, and fy_box_smooth): separable direct-sum box passes along x, y, z
// plus elementwise a/b and output kernels.
#include "fy_internal.h"

namespace {

FY_D float box_recip(int p, int L, int r) {
    const int lo = p - r < 0 ? 0 : p - r;
    const int hi = p + r > L - 1 ? L - 1 : p + r;
    return 1.0f / (float)(hi - lo + 1);                  // guided.c:26 (IEEE division)
}

// ---------------------------------------------------------------- generic separable path
template <int AXIS>
__global__ void __launch_bounds__(256) k_box_axis(const float* __restrict__ in, float* __restrict__ out,
                                                  int nz, int ny, int nx, int r) {
    const size_t n = (size_t)nz * ny * nx;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % nx);
        const size_t zy = i / nx;
        const int y = (int)(zy % ny), z = (int)(zy / ny);
        const int p = AXIS == 0 ? z : (AXIS == 1 ? y : x);
        const int L = AXIS == 0 ? nz : (AXIS == 1 ? ny : nx);
        const size_t st = AXIS == 0 ? (size_t)ny * nx : (AXIS == 1 ? (size_t)nx : 1);
        const int lo = p - r < 0 ? 0 : p - r, hi = p + r > L - 1 ? L - 1 : p + r;
        const float* b = in + i - (size_t)p * st;
        float s = 0.f;
        for (int j = lo; j <= hi; ++j) s += __ldg(b + (size_t)j * st);
        out[i] = s * box_recip(p, L, r);
    }
}

__global__ void k_square(const float* __restrict__ in, float* __restrict__ out, size_t n) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float v = in[i];
        out[i] = v * v;
    }
}

// a := var/(var+eps) into corr, b := mean*(1-a) into ab (guided.c:126-132)
__global__ void k_ab(const float* __restrict__ mean, float* __restrict__ corr_a, float* __restrict__ ab,
                     size_t n, float eps) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float m = mean[i];
        float var = ab[i] - m * m;
        if (var < 0.f) var = 0.f;
        const float a = var / (var + eps);
        corr_a[i] = a;
        ab[i] = m * (1.0f - a);
    }
}

__global__ void k_apply(const float* __restrict__ ma, const float* __restrict__ mb,
                        const float* __restrict__ in, float* __restrict__ out, size_t n) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = ma[i] * in[i] + mb[i];
}

unsigned grid_1d(size_t n) {
    size_t g = (n + 255) / 256;
    const size_t cap = 148 * 16;
    return (unsigned)(g < cap ? (g ? g : 1) : cap);
}

cudaError_t box3(const float* in, float* out, float* tmp, int nz, int ny, int nx, int r, cudaStream_t st,
                 int& launches) {
    const size_t n = (size_t)nz * ny * nx;
    k_box_axis<2><<<grid_1d(n), 256, 0, st>>>(in, out, nz, ny, nx, r);
    k_box_axis<1><<<grid_1d(n), 256, 0, st>>>(out, tmp, nz, ny, nx, r);
    k_box_axis<0><<<grid_1d(n), 256, 0, st>>>(tmp, out, nz, ny, nx, r);
    launches += 3;
    return cudaGetLastError();
}

// ---------------------------------------------------------------- fused z-sliding path
// CTA = 32 x 16 output columns sliding along z, 256 threads. Per input plane zi:
//   1. stage u = I - c over the tile + 2R halo (zeros outside the volume)
//   2. X means of u, u^2 over the a/b support columns (4 columns per thread)
//   3. Y means (4 rows per thread) pushed into a (2R+1)-plane z ring held in registers;
//      the ring gives mean/corr of plane zc = zi - R -> a, b over the support
//   4. X means of a, b over the output columns
//   5. Y means into a second register ring -> box(a), box(b) of plane zo = zi - 2R ->
//      out = box(a)*I + box(b)
// Widths are padded to multiples of 4 so every 4-wide segment stays inside its array.
constexpr int GTY = 16, GTX = 32, GNT = 256;

template <int R>
struct GuidedGeo {
    static constexpr int NR = 2 * R + 1;
    static constexpr int AY = GTY + 2 * R, AX = GTX + 2 * R;     // a/b support
    static constexpr int AYP = (AY + 3) & ~3, AXP = (AX + 3) & ~3;
    static constexpr int IYP = AYP + 2 * R, IXP = AXP + 2 * R;   // staged u region (padded)
};

template <int R>
struct GuidedSmem {
    using G = GuidedGeo<R>;
    float I[G::IYP][G::IXP];
    float xs1[G::IYP][G::AXP], xs2[G::IYP][G::AXP];
    float pa[G::AYP][G::AXP], pb[G::AYP][G::AXP];
    float xa[G::AYP][GTX], xb[G::AYP][GTX];
    float rx_s[G::AXP], ry_s[G::AYP];     // reciprocals of the support columns / rows
};

// MODE 0: out = box(a)*I + box(b). MODE 1: out = box(a), out_b = box(b) (the fast
// variant's low-resolution coefficient fields, guided.c:181-182).
template <int R, int MODE>
__global__ void __launch_bounds__(GNT, 2) k_guided_fused(const float* __restrict__ in, float* __restrict__ out,
                                                         float* __restrict__ out_b,
                                                         int nz, int ny, int nx, float eps,
                                                         const float* __restrict__ eps_ptr, int zchunk) {
    using G = GuidedGeo<R>;
    constexpr int NR = G::NR;
    __shared__ GuidedSmem<R> sm;
    if (eps_ptr) eps = *eps_ptr;                     // chained: eps from the device noise model
    const int x0 = blockIdx.x * GTX, y0 = blockIdx.y * GTY;
    const int zs = blockIdx.z * zchunk;
    const int ze = min(nz, zs + zchunk);
    const int t = threadIdx.x;
    const size_t plane = (size_t)ny * nx;
    // per-tile shift: one constant for every window this CTA forms
    const float c = __ldg(in + (size_t)zs * plane + (size_t)y0 * nx + x0);
    for (int i = t; i < G::AXP; i += GNT) {
        const int gx = x0 - R + i;
        sm.rx_s[i] = (gx >= 0 && gx < nx) ? box_recip(gx, nx, R) : 0.f;
    }
    for (int i = t; i < G::AYP; i += GNT) {
        const int gy = y0 - R + i;
        sm.ry_s[i] = (gy >= 0 && gy < ny) ? box_recip(gy, ny, R) : 0.f;
    }
    // step-3 role: support column xa3, support rows 4*rb3 .. +3
    constexpr int N3 = (G::AYP / 4) * G::AXP;
    const bool role3 = t < N3;
    const int xa3 = t % G::AXP, rb3 = t / G::AXP;
    // step-5 role: output column t % 32, output rows 4*(t/32) .. +3
    const bool role5 = t < 4 * GTX;
    const int xc5 = t % GTX, rb5 = t / GTX;
    float r1[NR][4], r2[NR][4], ra[NR][4], rb[NR][4];
#pragma unroll
    for (int q = 0; q < NR; ++q)
#pragma unroll
        for (int k = 0; k < 4; ++k) r1[q][k] = r2[q][k] = ra[q][k] = rb[q][k] = 0.f;
    __syncthreads();

    for (int zi = zs - 2 * R; zi < ze + 2 * R; ++zi) {
        const bool zin = zi >= 0 && zi < nz;
        // 1. stage u
        for (int k = t; k < G::IYP * G::IXP; k += GNT) {
            const int yy = k / G::IXP, xx = k - yy * G::IXP;
            const int gy = y0 - 2 * R + yy, gx = x0 - 2 * R + xx;
            float v = 0.f;
            if (zin && gy >= 0 && gy < ny && gx >= 0 && gx < nx) v = __ldg(in + (size_t)zi * plane + (size_t)gy * nx + gx) - c;
            sm.I[yy][xx] = v;
        }
        __syncthreads();
        // 2. X means of u, u^2 (4 support columns per thread)
        for (int sgi = t; sgi < G::IYP * (G::AXP / 4); sgi += GNT) {
            const int yy = sgi / (G::AXP / 4), x4 = 4 * (sgi % (G::AXP / 4));
            float u[4 + 2 * R];
#pragma unroll
            for (int j = 0; j < 4 + 2 * R; ++j) u[j] = sm.I[yy][x4 + j];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                float s1 = 0.f, s2 = 0.f;
#pragma unroll
                for (int j = 0; j <= 2 * R; ++j) { s1 += u[k + j]; s2 += u[k + j] * u[k + j]; }
                const float rx = sm.rx_s[x4 + k];
                sm.xs1[yy][x4 + k] = s1 * rx;
                sm.xs2[yy][x4 + k] = s2 * rx;
            }
        }
        __syncthreads();
        // 3. Y means -> z ring -> a, b of plane zc over the support
        const int zc = zi - R;
        if (role3) {
#pragma unroll
            for (int q = 0; q < NR - 1; ++q)
#pragma unroll
                for (int k = 0; k < 4; ++k) { r1[q][k] = r1[q + 1][k]; r2[q][k] = r2[q + 1][k]; }
            float a1[4 + 2 * R], a2[4 + 2 * R];
#pragma unroll
            for (int j = 0; j < 4 + 2 * R; ++j) { a1[j] = sm.xs1[4 * rb3 + j][xa3]; a2[j] = sm.xs2[4 * rb3 + j][xa3]; }
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                float s1 = 0.f, s2 = 0.f;
#pragma unroll
                for (int j = 0; j <= 2 * R; ++j) { s1 += a1[k + j]; s2 += a2[k + j]; }
                const float ry = sm.ry_s[4 * rb3 + k];
                r1[NR - 1][k] = s1 * ry;
                r2[NR - 1][k] = s2 * ry;
            }
            const bool zc_ok = zc >= 0 && zc < nz && zc >= zs - R && zc < ze + R;
            const float rz = zc_ok ? box_recip(zc, nz, R) : 0.f;
            const int gx = x0 - R + xa3;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int gy = y0 - R + 4 * rb3 + k;
                float a = 0.f, b = 0.f;
                if (zc_ok && gx >= 0 && gx < nx && gy >= 0 && gy < ny && 4 * rb3 + k < G::AY && xa3 < G::AX) {
                    float s1 = 0.f, s2 = 0.f;
#pragma unroll
                    for (int q = 0; q < NR; ++q) { s1 += r1[q][k]; s2 += r2[q][k]; }
                    const float e1 = s1 * rz, e2 = s2 * rz;      // E[I-c], E[(I-c)^2]
                    float var = e2 - e1 * e1;
                    if (var < 0.f) var = 0.f;
                    const float mean = e1 + c;
                    a = var / (var + eps);                        // guided.c:129
                    b = mean * (1.0f - a);                        // guided.c:131
                }
                sm.pa[4 * rb3 + k][xa3] = a;
                sm.pb[4 * rb3 + k][xa3] = b;
            }
        }
        __syncthreads();
        // 4. X means of a, b over the output columns
        for (int sgi = t; sgi < G::AYP * (GTX / 4); sgi += GNT) {
            const int ya = sgi / (GTX / 4), x4 = 4 * (sgi % (GTX / 4));
            float pa[4 + 2 * R], pb[4 + 2 * R];
#pragma unroll
            for (int j = 0; j < 4 + 2 * R; ++j) { pa[j] = sm.pa[ya][x4 + j]; pb[j] = sm.pb[ya][x4 + j]; }
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                float s1 = 0.f, s2 = 0.f;
#pragma unroll
                for (int j = 0; j <= 2 * R; ++j) { s1 += pa[k + j]; s2 += pb[k + j]; }
                const float rx = sm.rx_s[R + x4 + k];
                sm.xa[ya][x4 + k] = s1 * rx;
                sm.xb[ya][x4 + k] = s2 * rx;
            }
        }
        __syncthreads();
        // 5. Y means -> z ring -> output plane zo
        if (role5) {
#pragma unroll
            for (int q = 0; q < NR - 1; ++q)
#pragma unroll
                for (int k = 0; k < 4; ++k) { ra[q][k] = ra[q + 1][k]; rb[q][k] = rb[q + 1][k]; }
            float sa[4 + 2 * R], sb[4 + 2 * R];
#pragma unroll
            for (int j = 0; j < 4 + 2 * R; ++j) { sa[j] = sm.xa[4 * rb5 + j][xc5]; sb[j] = sm.xb[4 * rb5 + j][xc5]; }
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                float s1 = 0.f, s2 = 0.f;
#pragma unroll
                for (int j = 0; j <= 2 * R; ++j) { s1 += sa[k + j]; s2 += sb[k + j]; }
                const float ry = sm.ry_s[R + 4 * rb5 + k];
                ra[NR - 1][k] = s1 * ry;
                rb[NR - 1][k] = s2 * ry;
            }
            const int zo = zi - 2 * R;
            if (zo >= zs && zo < ze) {
                const float rz = box_recip(zo, nz, R);
                const int gx = x0 + xc5;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const int gy = y0 + 4 * rb5 + k;
                    if (gy >= ny || gx >= nx) continue;
                    float s1 = 0.f, s2 = 0.f;
#pragma unroll
                    for (int q = 0; q < NR; ++q) { s1 += ra[q][k]; s2 += rb[q][k]; }
                    const size_t o = (size_t)zo * plane + (size_t)gy * nx + gx;
                    if (MODE == 0) out[o] = (s1 * rz) * __ldg(in + o) + s2 * rz;
                    else { out[o] = s1 * rz; out_b[o] = s2 * rz; }
                }
            }
        }
        // next plane: step 1 writes I (last read in step 2), step 2 writes xs (read in step 3),
        // step 3 writes pa/pb (read in step 4) and step 4 writes xa/xb (read in step 5): each
        // is separated from its reader by at least one barrier above.
    }
}

}  // namespace

int fy_guided_fused_max_radius() { return 4; }

size_t fy_guided_fused_smem(int r) { return r >= 1 && r <= 4 ? 0 : 0; }   // static shared memory

// Fused exact guided filter, r in [1,4]. in != out required (out planes are written
// while neighbouring tiles still read their input halos). mode 1 writes box(a) to out and
// box(b) to out_b instead of the filtered volume.
cudaError_t fy_launch_guided_fused(const float* in, float* out, float* out_b, int nz, int ny, int nx, int r,
                                   float eps, int mode, int sms, cudaStream_t st, const float* eps_ptr) {
    const dim3 tiles(ceil_div_i(nx, GTX), ceil_div_i(ny, GTY), 1);
    // z chunks: enough CTAs for ~4 waves, but chunks of >= 8r planes so the 4r-plane
    // warm-up stays a small fraction
    const long tiles_xy = (long)tiles.x * tiles.y;
    int nchunk = (int)((6L * sms + tiles_xy - 1) / tiles_xy);
    const int min_chunk = 8 * r;
    if (nchunk > nz / min_chunk) nchunk = nz / min_chunk;
    if (nchunk < 1) nchunk = 1;
    const int zchunk = ceil_div_i(nz, nchunk);
    dim3 grid(tiles.x, tiles.y, ceil_div_i(nz, zchunk));
#define FY_GF(RR, MM) k_guided_fused<RR, MM><<<grid, GNT, 0, st>>>(in, out, out_b, nz, ny, nx, eps, eps_ptr, zchunk);
    if (mode == 0) {
        switch (r) {
            case 1: FY_GF(1, 0) break;
            case 2: FY_GF(2, 0) break;
            case 3: FY_GF(3, 0) break;
            case 4: FY_GF(4, 0) break;
            default: return cudaErrorInvalidValue;
        }
    } else {
        switch (r) {
            case 1: FY_GF(1, 1) break;
            case 2: FY_GF(2, 1) break;
            case 3: FY_GF(3, 1) break;
            case 4: FY_GF(4, 1) break;
            default: return cudaErrorInvalidValue;
        }
    }
#undef FY_GF
    return cudaGetLastError();
}

// ---------------------------------------------------------------- fast (s-decimated) variant
namespace {
// Il[z][y][x] = in[(z*s)][(y*s)][(x*s)]  (guided.c:163-168: decimation, not a mean)
__global__ void k_decimate(const float* __restrict__ in, float* __restrict__ lo, int ny, int nx,
                           int lz, int ly, int lx, int s) {
    const size_t nl = (size_t)lz * ly * lx;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < nl; i += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % lx);
        const size_t zy = i / lx;
        const int y = (int)(zy % ly), z = (int)(zy / ly);
        lo[i] = __ldg(in + ((size_t)z * s * ny + (size_t)y * s) * nx + (size_t)x * s);
    }
}

// out = a*I + b with a, b trilinear from the low grid (guided.c:188-228): low sample i sits
// at full coordinate i*s; u = (float)x/s, i0 = min((int)u, l-2), f = min(u - i0, 1); the
// four (z,y) rows are blended with w00..w11 first, then lerped in x.
__global__ void __launch_bounds__(256) k_upsample_apply(const float* __restrict__ in, float* __restrict__ out,
                                                        const float* __restrict__ ma, const float* __restrict__ mb,
                                                        int nz, int ny, int nx, int lz, int ly, int lx, int s) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y, z = blockIdx.z;
    if (x >= nx) return;
    const float fs = (float)s;
    const float uz = (float)z / fs;
    int z0 = (int)uz; if (z0 > lz - 2) z0 = lz - 2;
    float zf = uz - z0; if (zf > 1.0f) zf = 1.0f;
    const float uy = (float)y / fs;
    int y0 = (int)uy; if (y0 > ly - 2) y0 = ly - 2;
    float yfr = uy - y0; if (yfr > 1.0f) yfr = 1.0f;
    const float ux = (float)x / fs;
    int x0 = (int)ux; if (x0 > lx - 2) x0 = lx - 2;
    float fx = ux - x0; if (fx > 1.0f) fx = 1.0f;
    const float gx = 1 - fx;
    const size_t r00 = ((size_t)z0 * ly + y0) * lx, r01 = r00 + lx;
    const size_t r10 = r00 + (size_t)ly * lx, r11 = r10 + lx;
    const float w00 = (1 - zf) * (1 - yfr), w01 = (1 - zf) * yfr;
    const float w10 = zf * (1 - yfr), w11 = zf * yfr;
    float ar[2], br[2];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const int k = x0 + q;
        ar[q] = w00 * __ldg(ma + r00 + k) + w01 * __ldg(ma + r01 + k) + w10 * __ldg(ma + r10 + k) + w11 * __ldg(ma + r11 + k);
        br[q] = w00 * __ldg(mb + r00 + k) + w01 * __ldg(mb + r01 + k) + w10 * __ldg(mb + r10 + k) + w11 * __ldg(mb + r11 + k);
    }
    const float a = gx * ar[0] + fx * ar[1];
    const float b = gx * br[0] + fx * br[1];
    const size_t i = ((size_t)z * ny + y) * nx + x;
    out[i] = a * in[i] + b;
}
}  // namespace

// Fast guided filter (s >= 2, all low dims >= 2, rl = max(1, r/s) <= 4). ws: >= 3*nl floats.
cudaError_t fy_launch_guided_fast(const float* in, float* out, float* ws, int nz, int ny, int nx, int r,
                                  float eps, int s, int sms, cudaStream_t st, int& launches, const float* eps_ptr) {
    const int lz = (nz + s - 1) / s, ly = (ny + s - 1) / s, lx = (nx + s - 1) / s;
    const size_t nl = (size_t)lz * ly * lx;
    float *il = ws, *ma = ws + nl, *mb = ws + 2 * nl;
    int rl = r / s;
    if (rl < 1) rl = 1;
    k_decimate<<<grid_1d(nl), 256, 0, st>>>(in, il, ny, nx, lz, ly, lx, s);
    cudaError_t e = fy_launch_guided_fused(il, ma, mb, lz, ly, lx, rl, eps, 1, sms, st, eps_ptr);
    if (e != cudaSuccess) return e;
    dim3 grid(ceil_div_i(nx, 128), ny, nz);
    k_upsample_apply<<<grid, 128, 0, st>>>(in, out, ma, mb, nz, ny, nx, lz, ly, lx, s);
    launches += 3;
    return cudaGetLastError();
}

// Generic exact guided filter: ws holds 4n floats (fy_guided_ws_floats); in/out may alias
// each other but not ws. Returns the number of kernels launched through `launches`.
cudaError_t fy_launch_guided_generic(const float* in, float* out, float* ws, int nz, int ny, int nx, int r,
                                     float eps, cudaStream_t st, int& launches) {
    const size_t n = (size_t)nz * ny * nx;
    float *mean = ws, *corr = ws + n, *ab = ws + 2 * n, *tmp = ws + 3 * n;
    cudaError_t e;
    if ((e = box3(in, mean, tmp, nz, ny, nx, r, st, launches))) return e;
    k_square<<<grid_1d(n), 256, 0, st>>>(in, corr, n);
    if ((e = box3(corr, ab, tmp, nz, ny, nx, r, st, launches))) return e;
    k_ab<<<grid_1d(n), 256, 0, st>>>(mean, corr, ab, n, eps);
    if ((e = box3(corr, mean, tmp, nz, ny, nx, r, st, launches))) return e;   // mean := box(a)
    if ((e = box3(ab, corr, tmp, nz, ny, nx, r, st, launches))) return e;     // corr := box(b)
    k_apply<<<grid_1d(n), 256, 0, st>>>(mean, corr, in, out, n);
    launches += 3;
    return cudaGetLastError();
}

cudaError_t fy_launch_box_mean(const float* in, float* out, float* tmp, int nz, int ny, int nx, int r,
                               cudaStream_t st, int& launches) {
    return box3(in, out, tmp, nz, ny, nx, r, st, launches);
}
