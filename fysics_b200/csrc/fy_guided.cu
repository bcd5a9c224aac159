// fy_guided.cu -- 3-D self-guided filter (guided.c:113-241) and box mean (guided.c:19-106).
//
// Box semantics (guided.c:22-28, 35-98): the mean over the IN-BOUNDS part of a (2r+1)^3
// window, taken axis by axis, each axis dividing by its own clamped count with the
// reciprocal 1.0f/(float)count. Guided math per voxel (guided.c:121-135):
//   var = max(corr - mean^2, 0), a = var/(var + eps), b = mean*(1 - a),
//   out = box(a)*I + box(b).
//
// Exact path (r <= 4): two z-sliding box passes (fy_zbox.cuh). The first forms a and b
// from box means of (I - c) and (I - c)^2 with a per-tile shift c, which makes
// E[(I-c)^2] - E[I-c]^2 = E[I^2] - E[I]^2 exactly while removing most of the FP32
// cancellation that dominates the reference's error (guided.c:127); the second boxes a and
// b and applies them. 12 + 16 B/voxel of HBM traffic. In a chain whose noise model uses the
// same window, the noise statistics pass also writes (mean, var) and only the second pass
// runs here (fy_launch_guided_apply_mv).
//
// Generic path (any r, and fy_box_smooth): separable direct-sum box passes along x, y, z
// plus elementwise a/b and output kernels.
#include "fy_internal.h"
#include "fy_zbox.cuh"

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

}  // namespace

int fy_guided_fused_max_radius() { return 4; }

static size_t round64(size_t v) { return (v + 63) & ~(size_t)63; }
size_t fy_guided_fused_scratch_floats(size_t n) { return 2 * round64(n); }

// Exact guided filter for r in [1, 4] as two z-sliding box passes (fy_zbox.cuh):
// in -> interleaved (a, b) pairs into ab_ws, then box(a), box(b) -> out. ab_ws holds
// fy_guided_fused_scratch_floats(n) floats; out may alias in. mode 1 writes box(a) to out
// and box(b) to out_b instead of the filtered volume.
cudaError_t fy_launch_guided_fused(const float* in, float* out, float* out_b, float* ab_ws, int nz, int ny, int nx,
                                   int r, float eps, int mode, int sms, cudaStream_t st, const float* eps_ptr,
                                   const RingApply* rings) {
    if (r < 1 || r > 4) return cudaErrorInvalidValue;
    fyzb::Params p{};
    p.nz = nz; p.ny = ny; p.nx = nx;
    p.f0 = in; p.o0 = ab_ws; p.eps = eps; p.eps_ptr = eps_ptr;
    cudaError_t e = fyzb::launch<fyzb::ZB_GUIDED_AB>(p, r, sms, st);
    if (e != cudaSuccess) return e;
    fyzb::Params q{};
    q.nz = nz; q.ny = ny; q.nx = nx;
    q.f0 = ab_ws; q.guide = in; q.o0 = out; q.o1 = out_b; q.out_mode = mode;
    if (rings && mode == 0) q.ra = *rings;
    return fyzb::launch<fyzb::ZB_GUIDED_OUT>(q, r, sms, st);
}

// Output pass alone, from the guided (mean, var) pairs that the noise model's statistics pass
// wrote for the same window (fy_launch_estimate_noise with guided_mv): (a, b) are formed per
// staged voxel with the a/b pass's expressions, then boxed and applied as above. eps (or
// *eps_ptr) must be > 0.
cudaError_t fy_launch_guided_apply_mv(const float* mv, const float* in, float* out, int nz, int ny, int nx, int r,
                                      float eps, int sms, cudaStream_t st, const float* eps_ptr,
                                      const RingApply* rings) {
    if (r < 1 || r > 4) return cudaErrorInvalidValue;
    fyzb::Params q{};
    q.nz = nz; q.ny = ny; q.nx = nx;
    q.f0 = mv; q.guide = in; q.o0 = out; q.out_mode = 0; q.eps = eps; q.eps_ptr = eps_ptr;
    if (rings) q.ra = *rings;
    return fyzb::launch<fyzb::ZB_GUIDED_OUT_MV>(q, r, sms, st);
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

size_t fy_guided_fast_scratch_floats(int lz, int ly, int lx) {
    const size_t nl = round64((size_t)lz * ly * lx);
    return 3 * nl + fy_guided_fused_scratch_floats((size_t)lz * ly * lx);
}

// Fast guided filter (s >= 2, all low dims >= 2, rl = max(1, r/s) <= 4).
// ws: fy_guided_fast_scratch_floats(lz, ly, lx) floats.
cudaError_t fy_launch_guided_fast(const float* in, float* out, float* ws, int nz, int ny, int nx, int r,
                                  float eps, int s, int sms, cudaStream_t st, int& launches, const float* eps_ptr) {
    const int lz = (nz + s - 1) / s, ly = (ny + s - 1) / s, lx = (nx + s - 1) / s;
    const size_t nl = (size_t)lz * ly * lx, nlr = round64(nl);
    float *il = ws, *ma = ws + nlr, *mb = ws + 2 * nlr, *ab = ws + 3 * nlr;
    int rl = r / s;
    if (rl < 1) rl = 1;
    k_decimate<<<grid_1d(nl), 256, 0, st>>>(in, il, ny, nx, lz, ly, lx, s);
    cudaError_t e = fy_launch_guided_fused(il, ma, mb, ab, lz, ly, lx, rl, eps, 1, sms, st, eps_ptr);
    if (e != cudaSuccess) return e;
    const int tpb = nx < 256 ? (nx + 31) / 32 * 32 : 256;     // whole warps across a row
    dim3 grid(ceil_div_i(nx, tpb), ny, nz);
    k_upsample_apply<<<grid, tpb, 0, st>>>(in, out, ma, mb, nz, ny, nx, lz, ly, lx, s);
    launches += 4;
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

// Bounded waits of this unit's box passes that expired (see fy_zbox.cuh); 0 expected.
int fy_guided_wait_timeouts() { return fyzb::timeouts(); }
cudaError_t fy_guided_set_first_wait_polls(int polls) { return fyzb::set_first_wait_polls(polls); }
