// fy_cfft.cu -- full complex 3-D FFT over split re/im arrays (fy_fft1d / fy_fft3d /
// fy_fft3d_normalize, fft.c:168-228) and the plan-time fy_kernel_halo (paganin.c:93-118).
//
// Device layout: interleaved float2 c[(z*ny + y)*nxp + x], nxp = nx rounded up to 16 so
// W=16 column tiles never leave a row. X is a row pass staged through shared memory; Y and
// Z are column passes whose first/last Stockham pass reads/writes global memory directly.
// Unnormalised, sign -1 forward / +1 inverse, like the reference.
#include <math.h>
#include <vector>

#include "fy_context.h"

using fy::ctx;
using fy::fail;
using fy::fail_cuda;

namespace {

template <int E> struct KBc { static constexpr int nt = (E % 3 == 0) ? 256 : 512; };

struct Lane {
    int l, tl;
    FY_D Lane(int wlog) : l(threadIdx.x & ((1 << wlog) - 1)), tl(threadIdx.x >> wlog) {}
};

__global__ void k_interleave(const float* __restrict__ re, const float* __restrict__ im, float2* __restrict__ c,
                             long rows, int nx, int nxp) {
    const long n = rows * nx;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const long r = i / nx;
        const int x = (int)(i - r * nx);
        c[r * nxp + x] = make_float2(re[i], im[i]);
    }
}
__global__ void k_deinterleave(const float2* __restrict__ c, float* __restrict__ re, float* __restrict__ im,
                               long rows, int nx, int nxp, float scale) {
    const long n = rows * nx;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const long r = i / nx;
        const int x = (int)(i - r * nx);
        const float2 v = c[r * nxp + x];
        re[i] = v.x * scale;
        im[i] = v.y * scale;
    }
}

// X: W rows per CTA, rows staged through shared memory (pitch W+1).
template <int E>
__global__ void __launch_bounds__(KBc<E>::nt, 2) k_crow(float2* __restrict__ c, long rows, int nxp,
                                                        const __grid_constant__ FftPlan pl,
                                                        const float2* __restrict__ tw, float sign, int wlog,
                                                        FastDiv dn) {
    extern __shared__ float4 smem4[];
    const int W = 1 << wlog, LP = W + 1, n = pl.n;
    float2* s = reinterpret_cast<float2*>(smem4);
    float2* stw = s + n * LP;
    const long r0 = (long)blockIdx.x * W;
    load_twiddles(stw, tw, n);
    for (int idx = threadIdx.x; idx < W * n; idx += blockDim.x) {
        const int l = dn.div(idx), x = idx - l * n;
        const long r = r0 + l;
        s[x * LP + l] = r < rows ? c[r * nxp + x] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    const Lane ln(wlog);
    line_fft<E>(s + ln.l, LP, ln.tl, pl, stw, sign,
                [&](int i) { return s[i * LP + ln.l]; },
                [&](int i, float2 v) { s[i * LP + ln.l] = v; });
    __syncthreads();
    for (int idx = threadIdx.x; idx < W * n; idx += blockDim.x) {
        const int l = dn.div(idx), x = idx - l * n;
        const long r = r0 + l;
        if (r < rows) c[r * nxp + x] = s[x * LP + l];
    }
}

// Column pass: CTA = (column tile, batch b); point i of column k at c + b*bstride + i*pstride + k.
template <int E>
__global__ void __launch_bounds__(KBc<E>::nt, 2) k_ccol(float2* __restrict__ c, size_t bstride, size_t pstride,
                                                        const __grid_constant__ FftPlan pl,
                                                        const float2* __restrict__ tw, float sign, int wlog) {
    extern __shared__ float4 smem4[];
    const int W = 1 << wlog;
    float2* s = reinterpret_cast<float2*>(smem4);
    float2* stw = s + pl.n * W;
    const Lane ln(wlog);
    float2* col = c + (size_t)blockIdx.y * bstride + (size_t)blockIdx.x * W + ln.l;
    load_twiddles(stw, tw, pl.n);
    __syncthreads();
    line_fft<E>(s + ln.l, W, ln.tl, pl, stw, sign,
                [&](int i) { return col[(size_t)i * pstride]; },
                [&](int i, float2 v) { col[(size_t)i * pstride] = v; });
}

unsigned grid1(long n) {
    long g = (n + 255) / 256;
    return (unsigned)(g < 4096 ? (g ? g : 1) : 4096);
}

cudaError_t row_pass(float2* c, long rows, int n, int nxp, float sign, cudaStream_t st) {
    if (n == 1) return cudaSuccess;
    const FftPlan pl = fy_make_plan(n);
    const float2* tw = fy::twiddles(n);
    if (!tw) return cudaErrorMemoryAllocation;
    const TileShape t = fy_tile_shape(n);
    const size_t smem = (size_t)n * (t.W + 1) * sizeof(float2) + (size_t)n * sizeof(float2);
    const unsigned grid = (unsigned)((rows + t.W - 1) / t.W);
    return fy_with_e(t.E, [&](auto ec) -> cudaError_t {
        constexpr int E = decltype(ec)::value;
        cudaError_t e = fy_smem_optin(k_crow<E>, smem);
        if (e != cudaSuccess) return e;
        k_crow<E><<<grid, t.NT, smem, st>>>(c, rows, nxp, pl, tw, sign, t.wlog, FastDiv(n));
        return cudaGetLastError();
    });
}

cudaError_t col_pass(float2* c, int n, int ncols, int nbatch, size_t bstride, size_t pstride, float sign,
                     cudaStream_t st) {
    if (n == 1) return cudaSuccess;
    const FftPlan pl = fy_make_plan(n);
    const float2* tw = fy::twiddles(n);
    if (!tw) return cudaErrorMemoryAllocation;
    const TileShape t = fy_tile_shape(n);
    const size_t smem = (size_t)n * t.W * sizeof(float2) + (size_t)n * sizeof(float2);
    dim3 grid(ceil_div_i(ncols, t.W), nbatch);
    return fy_with_e(t.E, [&](auto ec) -> cudaError_t {
        constexpr int E = decltype(ec)::value;
        cudaError_t e = fy_smem_optin(k_ccol<E>, smem);
        if (e != cudaSuccess) return e;
        k_ccol<E><<<grid, t.NT, smem, st>>>(c, bstride, pstride, pl, tw, sign, t.wlog);
        return cudaGetLastError();
    });
}

}  // namespace

// Complex 3-D transform of an interleaved, row-pitched device volume (nxp >= nx, multiple of 16).
cudaError_t fy_launch_cfft3d(float2* c, int nz, int ny, int nx, int nxp, int sign, cudaStream_t st) {
    const float sg = sign < 0 ? -1.f : 1.f;
    cudaError_t e;
    if ((e = row_pass(c, (long)nz * ny, nx, nxp, sg, st)) != cudaSuccess) return e;
    if (ny > 1 && (e = col_pass(c, ny, nx, nz, (size_t)ny * nxp, (size_t)nxp, sg, st)) != cudaSuccess) return e;
    if (nz > 1 && (e = col_pass(c, nz, nx, ny, (size_t)nxp, (size_t)ny * nxp, sg, st)) != cudaSuccess) return e;
    return cudaSuccess;
}

namespace {
// host split re/im -> GPU -> host; scale_only: skip the transform and multiply by 1/N
int host_cfft(float* re, float* im, int nz, int ny, int nx, int sign, bool scale_only, const char* what) {
    if (!re || !im) return fail(FY_EINVAL, "%s: null pointer", what);
    if (nz < 1 || ny < 1 || nx < 1) return fail(FY_EINVAL, "%s: bad dims", what);
    if (!scale_only && (!fy_fft_len_ok(nz) || !fy_fft_len_ok(ny) || !fy_fft_len_ok(nx)))
        return fail(FY_EUNSUPPORTED, "%s: sizes must be 2^k or 3*2^k <= %d (got %dx%dx%d)", what, FY_FFT_MAXN, nz, ny,
                    nx);
    int rc = fy::ensure_ctx();
    if (rc) return rc;
    fy::ThreadCtx& c = ctx();
    cudaStream_t st = c.st;
    const size_t n = (size_t)nz * ny * nx;
    const int nxp = (nx + 15) & ~15;
    const long rows = (long)nz * ny;
    fy::ws_acquire(st);
    cudaError_t e;
    if ((e = c.vin.ensure(2 * n * sizeof(float))) != cudaSuccess) return fail_cuda(e, what);
    if ((e = c.spec.ensure((size_t)rows * nxp * sizeof(float2))) != cudaSuccess) return fail_cuda(e, what);
    float* dre = c.vin.as<float>();
    float* dim = dre + n;
    if ((e = cudaMemcpyAsync(dre, re, n * 4, cudaMemcpyHostToDevice, st)) != cudaSuccess) return fail_cuda(e, what);
    if ((e = cudaMemcpyAsync(dim, im, n * 4, cudaMemcpyHostToDevice, st)) != cudaSuccess) return fail_cuda(e, what);
    float2* cbuf = c.spec.as<float2>();
    k_interleave<<<grid1((long)n), 256, 0, st>>>(dre, dim, cbuf, rows, nx, nxp);
    float scale = 1.0f;
    if (scale_only) scale = 1.0f / (float)n;                      // fft.c:226
    else if ((e = fy_launch_cfft3d(cbuf, nz, ny, nx, nxp, sign, st)) != cudaSuccess) return fail_cuda(e, what);
    k_deinterleave<<<grid1((long)n), 256, 0, st>>>(cbuf, dre, dim, rows, nx, nxp, scale);
    if ((e = cudaGetLastError()) != cudaSuccess) return fail_cuda(e, what);
    fy::count_launch(scale_only ? 2 : 5);
    if ((e = cudaMemcpyAsync(re, dre, n * 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess) return fail_cuda(e, what);
    if ((e = cudaMemcpyAsync(im, dim, n * 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess) return fail_cuda(e, what);
    fy::ws_release(st);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return fail_cuda(e, what);
    return FY_OK;
}
}  // namespace

extern "C" void fy_fft1d(float* re, float* im, int n, int sign) {
    fy::enter();
    host_cfft(re, im, 1, 1, n, sign, false, "fy_fft1d");
}
extern "C" void fy_fft3d(float* re, float* im, int nz, int ny, int nx, int sign) {
    fy::enter();
    host_cfft(re, im, nz, ny, nx, sign, false, "fy_fft3d");
}
extern "C" void fy_fft3d_normalize(float* re, float* im, int nz, int ny, int nx) {
    fy::enter();
    host_cfft(re, im, nz, ny, nx, 0, true, "fy_fft3d_normalize");
}

// paganin.c:93-118: impulse response of H/(H^2+0.05) along one axis (256-point inverse
// transform on the GPU), last lag above 1% of the peak, clamped to [8, 96]; 16 if the
// transform cannot run (the reference's allocation-failure value).
extern "C" int fy_kernel_halo(const fy_physics* p) {
    fy::enter();
    const int n = 256;
    std::vector<float> re(n), im(n, 0.0f);
    for (int i = 0; i < n; i++) {
        const double f = (i <= n / 2) ? (double)i / n : (double)(i - n) / n;
        const double H = fy_recon_transfer(fabs(f), p);
        re[i] = (float)(H / (H * H + 0.05));
    }
    if (host_cfft(re.data(), im.data(), 1, 1, n, +1, false, "fy_kernel_halo") != FY_OK) return 16;
    float peak = 0.0f;
    for (int i = 0; i < n; i++) { const float a = fabsf(re[i]); if (a > peak) peak = a; }
    int half = 8;
    for (int d = 1; d < n / 2; d++)
        if (fabsf(re[d]) > 0.01f * peak) half = d;
    if (half < 8) half = 8;
    if (half > 96) half = 96;
    return half;
}
