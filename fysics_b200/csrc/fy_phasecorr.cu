// fy_phasecorr.cu -- sub-voxel translation by phase correlation (fy_phase_correlate,
// phasecorr.c:38-186) on the half-spectrum engine.
//
//   k_pc_means  double-precision means of the UNWINDOWED inputs (phasecorr.c:66-74):
//               per-thread compensated float sums, per-CTA pairs combined once in double
//   k_pc_x      rows: (f - mean_f)*w | (m - mean_m)*w packed as one complex line per row
//               (w = wz*wy*wx, Hann or ones, phasecorr.c:76-87), zero padding to the next
//               power of two, forward FFT, untangle into the F and M half spectra
//   Y pass      forward on both spectra (rows >= ny are zero)
//   k_pc_z      forward Z of F and M columns (planes >= nz zero), phase-only cross power
//               R = conj(F)M/|conj(F)M| (|.| <= 1e-12 -> 0, phasecorr.c:101-109) with the
//               max magnitude tracked, inverse Z of R
//   Y pass      inverse (all padded rows)
//   k_pc_c2r    C2R of every padded row -> correlation surface (real part of the inverse,
//               phasecorr.c:118), with the argmax fused: strictly greater wins, ties go to
//               the first index (phasecorr.c:121-122), via one 64-bit atomicMax
//   k_pc_fit    FP64: fftfreq unwrap and Foroosh subvoxel fit per axis (phasecorr.c:127-182)
#include <math.h>
#include <vector>

#include "fy_context.h"

using fy::ctx;
using fy::fail;
using fy::fail_cuda;

// Device-resident results of one correlation.
struct PcCtl {
    double sum_f, sum_m;
    float mean_f, mean_m;
    unsigned int maxmag_bits;            // float bits of the largest |conj(F)M| (>= 0)
    unsigned long long best;             // (orderable value << 32) | (0xffffffff - index)
    double shift[3];
    double peak;
    long long peak_index;
    int status;                          // 0 ok, 1 degenerate (flat input)
};

namespace {

template <int E> struct KBp { static constexpr int nt = (E % 3 == 0) ? 256 : 512; };

struct Lane {
    int l, tl;
    FY_D Lane(int wlog) : l(threadIdx.x & ((1 << wlog) - 1)), tl(threadIdx.x >> wlog) {}
};

FY_D uint32_t fkey(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
FY_D float funkey(uint32_t k) {
    const uint32_t u = (k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k;
    return __uint_as_float(u);
}

// ---------------------------------------------------------------- means
__global__ void __launch_bounds__(256) k_pc_means(const float* __restrict__ f, const float* __restrict__ m, long n,
                                                  float4* __restrict__ part) {
    float sf = 0.f, cf = 0.f, sm = 0.f, cm = 0.f;         // Kahan-compensated per thread
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        float y = __ldg(f + i) - cf, t = sf + y;
        cf = (t - sf) - y; sf = t;
        y = __ldg(m + i) - cm; t = sm + y;
        cm = (t - sm) - y; sm = t;
    }
    __shared__ double red[2][256];
    red[0][threadIdx.x] = (double)sf - (double)cf;
    red[1][threadIdx.x] = (double)sm - (double)cm;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            red[0][threadIdx.x] += red[0][threadIdx.x + w];
            red[1][threadIdx.x] += red[1][threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double a = red[0][0], b = red[1][0];
        const float ah = (float)a, bh = (float)b;
        part[blockIdx.x] = make_float4(ah, (float)(a - ah), bh, (float)(b - bh));
    }
}

__global__ void k_pc_means_final(const float4* __restrict__ part, int nparts, long n, PcCtl* ctl) {
    if (threadIdx.x != 0) return;
    double sf = 0, sm = 0;
    for (int i = 0; i < nparts; ++i) {
        const float4 p = part[i];
        sf += (double)p.x + (double)p.y;
        sm += (double)p.z + (double)p.w;
    }
    ctl->sum_f = sf; ctl->sum_m = sm;
    ctl->mean_f = (float)(sf / n);                       // phasecorr.c:74
    ctl->mean_m = (float)(sm / n);
    ctl->maxmag_bits = 0;
    ctl->best = 0;
    ctl->status = 0;
}

// ---------------------------------------------------------------- X forward (pair packing)
template <int E>
__global__ void __launch_bounds__(KBp<E>::nt, 2) k_pc_x(const float* __restrict__ fix, const float* __restrict__ mov,
                                                        const float* __restrict__ wz, const float* __restrict__ wy,
                                                        const float* __restrict__ wx, const PcCtl* __restrict__ ctl,
                                                        float2* __restrict__ specF, float2* __restrict__ specM,
                                                        SpecGeom g, const __grid_constant__ FftPlan pl,
                                                        const float2* __restrict__ tw, int wlog, FastDiv dpx,
                                                        FastDiv dhx) {
    extern __shared__ float4 smem4[];
    const int W = 1 << wlog, LP = W + 1;
    float2* s = reinterpret_cast<float2*>(smem4);
    float2* stw = s + pl.n * LP;
    const long Q = (long)g.nz * g.ny;
    const long q0 = (long)blockIdx.x * W;
    const float mf = ctl->mean_f, mm = ctl->mean_m;
    load_twiddles(stw, tw, pl.n);
    for (int idx = threadIdx.x; idx < W * g.px; idx += blockDim.x) {
        const int l = dpx.div(idx), x = idx - l * g.px;
        const long q = q0 + l;
        float a = 0.f, b = 0.f;
        if (q < Q && x < g.nx) {
            const int z = (int)(q / g.ny), y = (int)(q - (long)z * g.ny);
            const float wzy = wz[z] * wy[y];
            const float w = wzy * wx[x];
            a = (__ldg(fix + q * g.nx + x) - mf) * w;
            b = (__ldg(mov + q * g.nx + x) - mm) * w;
        }
        s[x * LP + l] = make_float2(a, b);
    }
    __syncthreads();
    const Lane ln(wlog);
    line_fft<E>(s + ln.l, LP, ln.tl, pl, stw, -1.f,
                [&](int i) { return s[i * LP + ln.l]; },
                [&](int i, float2 v) { s[i * LP + ln.l] = v; });
    __syncthreads();
    for (int idx = threadIdx.x; idx < W * g.hx; idx += blockDim.x) {
        const int l = dhx.div(idx), k = idx - l * g.hx;
        const long q = q0 + l;
        if (q >= Q) continue;
        const int mk = k == 0 ? 0 : g.px - k;
        float2 A, B;
        untangle(s[k * LP + l], s[mk * LP + l], A, B);
        const size_t row = ((size_t)(q / g.ny) * g.py + (q % g.ny)) * g.hxp;
        specF[row + k] = A;
        specM[row + k] = B;
    }
}

// ---------------------------------------------------------------- Z: cross power
template <int E>
__global__ void __launch_bounds__(KBp<E>::nt, 1) k_pc_z(float2* __restrict__ specF, const float2* __restrict__ specM,
                                                        SpecGeom g, const __grid_constant__ FftPlan pl,
                                                        const float2* __restrict__ tw, int wlog, PcCtl* __restrict__ ctl) {
    extern __shared__ float4 smem4[];
    const int W = 1 << wlog, n = pl.n;
    float2* sf = reinterpret_cast<float2*>(smem4);
    float2* sm = sf + n * W;
    float2* stw = sm + n * W;
    __shared__ float s_max;
    const Lane ln(wlog);
    const int k = blockIdx.x * W + ln.l;
    const size_t zstride = (size_t)g.py * g.hxp;
    const size_t coff = (size_t)blockIdx.y * g.hxp + (size_t)blockIdx.x * W + ln.l;
    if (threadIdx.x == 0) s_max = 0.f;
    load_twiddles(stw, tw, n);
    __syncthreads();
    line_fft<E>(sf + ln.l, W, ln.tl, pl, stw, -1.f,
                [&](int i) { return i < g.nz ? specF[coff + (size_t)i * zstride] : make_float2(0.f, 0.f); },
                [&](int i, float2 v) { sf[i * W + ln.l] = v; });
    __syncthreads();
    line_fft<E>(sm + ln.l, W, ln.tl, pl, stw, -1.f,
                [&](int i) { return i < g.nz ? specM[coff + (size_t)i * zstride] : make_float2(0.f, 0.f); },
                [&](int i, float2 v) { sm[i * W + ln.l] = v; });
    __syncthreads();
    float lmax = 0.f;
    for (int z = ln.tl; z < n; z += blockDim.x >> wlog) {
        const float2 F = sf[z * W + ln.l], M = sm[z * W + ln.l];
        const float cr = F.x * M.x + F.y * M.y;
        const float ci = F.x * M.y - F.y * M.x;
        const float mag = sqrtf(cr * cr + ci * ci);
        if (k < g.hx && mag > lmax) lmax = mag;
        sf[z * W + ln.l] = mag > 1e-12f ? make_float2(cr / mag, ci / mag) : make_float2(0.f, 0.f);
    }
    atomicMax((unsigned int*)&s_max, __float_as_uint(lmax));   // non-negative floats order as uints
    __syncthreads();
    if (threadIdx.x == 0) atomicMax(&ctl->maxmag_bits, __float_as_uint(s_max));
    line_fft<E>(sf + ln.l, W, ln.tl, pl, stw, +1.f,
                [&](int i) { return sf[i * W + ln.l]; },
                [&](int i, float2 v) { specF[coff + (size_t)i * zstride] = v; });
}

// ---------------------------------------------------------------- C2R + argmax
template <int E>
__global__ void __launch_bounds__(KBp<E>::nt, 2) k_pc_c2r(const float2* __restrict__ spec, float* __restrict__ surf,
                                                          SpecGeom g, const __grid_constant__ FftPlan pl,
                                                          const float2* __restrict__ tw, int wlog, FastDiv dhx,
                                                          FastDiv dpx, PcCtl* __restrict__ ctl) {
    extern __shared__ float4 smem4[];
    const int W = 1 << wlog, LP = W + 1;
    float2* s = reinterpret_cast<float2*>(smem4);
    float2* stw = s + pl.n * LP;
    __shared__ unsigned long long s_best;
    const long Q = (long)g.pz * g.py;                       // every padded row
    const long q0 = (long)blockIdx.x * 2 * W;
    if (threadIdx.x == 0) s_best = 0;
    load_twiddles(stw, tw, pl.n);
    const int hi_max = g.px - g.hx;
    for (int idx = threadIdx.x; idx < W * g.hx; idx += blockDim.x) {
        const int l = dhx.div(idx), k = idx - l * g.hx;
        const long qa = q0 + 2 * l, qb = qa + 1;
        const float2 A = qa < Q ? spec[(size_t)qa * g.hxp + k] : make_float2(0.f, 0.f);
        const float2 B = qb < Q ? spec[(size_t)qb * g.hxp + k] : make_float2(0.f, 0.f);
        s[k * LP + l] = pack_lo(A, B);
        if (k >= 1 && k <= hi_max) s[(g.px - k) * LP + l] = pack_hi(A, B);
    }
    __syncthreads();
    const Lane ln(wlog);
    line_fft<E>(s + ln.l, LP, ln.tl, pl, stw, +1.f,
                [&](int i) { return s[i * LP + ln.l]; },
                [&](int i, float2 v) { s[i * LP + ln.l] = v; });
    __syncthreads();
    unsigned long long mine = 0;
    for (int idx = threadIdx.x; idx < W * g.px; idx += blockDim.x) {
        const int l = dpx.div(idx), x = idx - l * g.px;
        const long qa = q0 + 2 * l, qb = qa + 1;
        const float2 v = s[x * LP + l];
        if (qa < Q) {
            const size_t i = (size_t)qa * g.px + x;
            surf[i] = v.x;
            const unsigned long long key = ((unsigned long long)fkey(v.x) << 32) | (0xffffffffull - i);
            if (key > mine) mine = key;
        }
        if (qb < Q) {
            const size_t i = (size_t)qb * g.px + x;
            surf[i] = v.y;
            const unsigned long long key = ((unsigned long long)fkey(v.y) << 32) | (0xffffffffull - i);
            if (key > mine) mine = key;
        }
    }
    atomicMax(&s_best, mine);
    __syncthreads();
    if (threadIdx.x == 0) atomicMax(&ctl->best, s_best);
}

// ---------------------------------------------------------------- FP64 Foroosh fit
__global__ void k_pc_fit(const float* __restrict__ surf, SpecGeom g, PcCtl* ctl) {
    if (threadIdx.x != 0) return;
    const int pz = g.pz, py = g.py, px = g.px;
    const double maxmag = (double)__uint_as_float(ctl->maxmag_bits);
    if (maxmag < 1e-20) {                                  // phasecorr.c:111-114
        ctl->status = 1;
        ctl->shift[0] = ctl->shift[1] = ctl->shift[2] = 0.0;
        ctl->peak = 0.0;
        ctl->peak_index = -1;
        return;
    }
    const unsigned long long b = ctl->best;
    const size_t pk = 0xffffffffull - (b & 0xffffffffull);
    const float best = funkey((uint32_t)(b >> 32));
    const int kz = (int)(pk / ((size_t)py * px)), ky = (int)((pk / px) % py), kx = (int)(pk % px);
    const int kk[3] = {kz, ky, kx}, pp[3] = {pz, py, px};
    const double c0 = best;
    for (int a = 0; a < 3; ++a) {
        int im[3] = {kz, ky, kx}, ip[3] = {kz, ky, kx};
        im[a] = (kk[a] - 1 + pp[a]) % pp[a];
        ip[a] = (kk[a] + 1) % pp[a];
        const double cm = surf[((size_t)im[0] * py + im[1]) * px + im[2]];
        const double cp = surf[((size_t)ip[0] * py + ip[1]) * px + ip[2]];
        const double c1 = (cp >= cm) ? cp : cm;             // larger side lobe
        const double sg = (cp >= cm) ? 1.0 : -1.0;
        double d = 0.0;
        if (fabs(c1 - c0) > 1e-20 && fabs(c1 + c0) > 1e-20) {
            const double d1 = c1 / (c1 - c0), d2 = c1 / (c1 + c0);
            d = sg * ((fabs(d1) <= fabs(d2)) ? d1 : d2);
        }
        if (d > 0.5) d = 0.5;
        if (d < -0.5) d = -0.5;
        const int iu = (kk[a] <= pp[a] / 2) ? kk[a] : kk[a] - pp[a];   // fftfreq unwrap
        ctl->shift[a] = iu + d;
    }
    ctl->peak = (double)best / (double)((size_t)pz * py * px);   // phasecorr.c:182
    ctl->peak_index = (long long)pk;
}

// 1-D Hann weights (phasecorr.c:38-42), float cosf as the reference; ones when !window.
void hann(std::vector<float>& w, int n, int window) {
    w.assign((size_t)n, 1.0f);
    if (!window) return;
    if (n == 1) { w[0] = 1.0f; return; }
    for (int i = 0; i < n; i++) w[(size_t)i] = 0.5f - 0.5f * cosf(2.0f * (float)M_PI * i / (float)(n - 1));
}

}  // namespace

// Workspace layout for one correlation of (nz,ny,nx) padded to powers of two.
struct PcLayout {
    SpecGeom g;
    size_t off_specF, off_specM, off_surf, off_win, off_part, off_ctl, total;
};

static PcLayout pc_layout(int nz, int ny, int nx) {
    PcLayout L{};
    SpecGeom& g = L.g;
    g.nz = nz; g.ny = ny; g.nx = nx;
    g.pz = fy_next_pow2(nz); g.py = fy_next_pow2(ny); g.px = fy_next_pow2(nx);
    g.hx = g.px / 2 + 1;
    g.hxp = (g.hx + 15) & ~15;
    g.zero_pad = 1;
    size_t o = 0;
    auto take = [&](size_t bytes) { const size_t at = o; o += (bytes + 255) & ~(size_t)255; return at; };
    L.off_specF = take((size_t)g.pz * g.py * g.hxp * sizeof(float2));
    L.off_specM = take((size_t)g.nz * g.py * g.hxp * sizeof(float2));
    L.off_surf = take((size_t)g.pz * g.py * g.px * sizeof(float));
    L.off_win = take(((size_t)nz + ny + nx) * sizeof(float));
    L.off_part = take(1024 * sizeof(float4));
    L.off_ctl = take(sizeof(PcCtl));
    L.total = o;
    return L;
}

size_t fy_pc_scratch_bytes(int nz, int ny, int nx) { return pc_layout(nz, ny, nx).total; }

// Enqueue one correlation; d_win must already hold the wz|wy|wx windows.
static cudaError_t pc_enqueue(const float* fix, const float* mov, char* ws, const PcLayout& L, int sms,
                              cudaStream_t st, int& launches) {
    const SpecGeom& g = L.g;
    float2* specF = (float2*)(ws + L.off_specF);
    float2* specM = (float2*)(ws + L.off_specM);
    float* surf = (float*)(ws + L.off_surf);
    const float* wz = (const float*)(ws + L.off_win);
    const float* wy = wz + g.nz;
    const float* wx = wy + g.ny;
    float4* part = (float4*)(ws + L.off_part);
    PcCtl* ctl = (PcCtl*)(ws + L.off_ctl);
    const long n = (long)g.nz * g.ny * g.nx;
    cudaError_t e;
    int nparts = (int)((n + 255) / 256);
    if (nparts > 4 * sms) nparts = 4 * sms;
    if (nparts > 1024) nparts = 1024;
    k_pc_means<<<nparts, 256, 0, st>>>(fix, mov, n, part);
    k_pc_means_final<<<1, 32, 0, st>>>(part, nparts, n, ctl);
    const FftPlan plx = fy_make_plan(g.px), ply = fy_make_plan(g.py), plz = fy_make_plan(g.pz);
    const float2 *twx = fy::twiddles(g.px), *twy = fy::twiddles(g.py), *twz = fy::twiddles(g.pz);
    if (!twx || !twy || !twz) return cudaErrorMemoryAllocation;
    {   // X forward of the packed pair
        const TileShape t = fy_tile_shape(g.px);
        const size_t smem = (size_t)g.px * (t.W + 1) * sizeof(float2) + (size_t)g.px * sizeof(float2);
        const unsigned grid = (unsigned)(((long)g.nz * g.ny + t.W - 1) / t.W);
        e = fy_with_e(t.E, [&](auto ec) -> cudaError_t {
            constexpr int E = decltype(ec)::value;
            cudaError_t e2 = fy_smem_optin(k_pc_x<E>, smem);
            if (e2 != cudaSuccess) return e2;
            k_pc_x<E><<<grid, t.NT, smem, st>>>(fix, mov, wz, wy, wx, ctl, specF, specM, g, plx, twx, t.wlog,
                                                FastDiv(g.px), FastDiv(g.hx));
            return cudaGetLastError();
        });
        if (e != cudaSuccess) return e;
    }
    if ((e = fy_launch_spec_y(specF, g, ply, twy, g.nz, -1, g.py, st)) != cudaSuccess) return e;
    if ((e = fy_launch_spec_y(specM, g, ply, twy, g.nz, -1, g.py, st)) != cudaSuccess) return e;
    {   // Z: cross power
        const TileShape t = fy_tile_shape(g.pz);
        const size_t smem = 2 * (size_t)g.pz * t.W * sizeof(float2) + (size_t)g.pz * sizeof(float2);
        dim3 grid(ceil_div_i(g.hx, t.W), g.py);
        e = fy_with_e(t.E, [&](auto ec) -> cudaError_t {
            constexpr int E = decltype(ec)::value;
            cudaError_t e2 = fy_smem_optin(k_pc_z<E>, smem);
            if (e2 != cudaSuccess) return e2;
            k_pc_z<E><<<grid, t.NT, smem, st>>>(specF, specM, g, plz, twz, t.wlog, ctl);
            return cudaGetLastError();
        });
        if (e != cudaSuccess) return e;
    }
    if ((e = fy_launch_spec_y(specF, g, ply, twy, g.pz, +1, g.py, st)) != cudaSuccess) return e;
    {   // C2R + argmax over every padded row
        const TileShape t = fy_tile_shape(g.px);
        const size_t smem = (size_t)g.px * (t.W + 1) * sizeof(float2) + (size_t)g.px * sizeof(float2);
        const unsigned grid = (unsigned)(((long)g.pz * g.py + 2 * t.W - 1) / (2 * t.W));
        e = fy_with_e(t.E, [&](auto ec) -> cudaError_t {
            constexpr int E = decltype(ec)::value;
            cudaError_t e2 = fy_smem_optin(k_pc_c2r<E>, smem);
            if (e2 != cudaSuccess) return e2;
            k_pc_c2r<E><<<grid, t.NT, smem, st>>>(specF, surf, g, plx, twx, t.wlog, FastDiv(g.hx), FastDiv(g.px), ctl);
            return cudaGetLastError();
        });
        if (e != cudaSuccess) return e;
    }
    k_pc_fit<<<1, 32, 0, st>>>(surf, g, ctl);
    launches += 9;
    return cudaGetLastError();
}

static int pc_check(int nz, int ny, int nx, const char* what) {
    const int pz = fy_next_pow2(nz), py = fy_next_pow2(ny), px = fy_next_pow2(nx);
    if (!fy_fft_len_ok(pz) || !fy_fft_len_ok(py) || !fy_fft_len_ok(px))
        return fail(FY_EUNSUPPORTED, "%s: padded size %dx%dx%d exceeds %d per axis", what, pz, py, px, FY_FFT_MAXN);
    if ((size_t)pz * py * px >= 0xffffffffull)
        return fail(FY_EUNSUPPORTED, "%s: padded volume exceeds 2^32 voxels", what);
    return FY_OK;
}

static int pc_upload_windows(char* ws, const PcLayout& L, int window, cudaStream_t st, std::vector<float>& h) {
    std::vector<float> wz, wy, wx;
    hann(wz, L.g.nz, window); hann(wy, L.g.ny, window); hann(wx, L.g.nx, window);
    h.clear();
    h.insert(h.end(), wz.begin(), wz.end());
    h.insert(h.end(), wy.begin(), wy.end());
    h.insert(h.end(), wx.begin(), wx.end());
    cudaError_t e = cudaMemcpyAsync(ws + L.off_win, h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice, st);
    return e == cudaSuccess ? FY_OK : fail_cuda(e, "phase correlation windows");
}

extern "C" int fy_phase_correlate(const float* fixed, const float* moving, int nz, int ny, int nx, double* shift,
                                  double* peak, int window) {
    fy::enter();
    const char* what = "fy_phase_correlate";
    if (!fixed || !moving || !shift || nz < 2 || ny < 2 || nx < 2) return 1;   // phasecorr.c:47
    int rc = pc_check(nz, ny, nx, what);
    if (rc) return rc;
    if ((rc = fy::ensure_ctx())) return rc;
    fy::ThreadCtx& c = ctx();
    cudaStream_t st = c.st;
    const PcLayout L = pc_layout(nz, ny, nx);
    const size_t n = (size_t)nz * ny * nx;
    fy::ws_acquire(st);
    cudaError_t e;
    if ((e = c.vin.ensure(2 * n * sizeof(float))) != cudaSuccess) return fail_cuda(e, what);
    if ((e = c.spec.ensure(L.total)) != cudaSuccess) return fail_cuda(e, what);
    if ((e = c.pin.ensure(sizeof(PcCtl))) != cudaSuccess) return fail_cuda(e, what);
    float* dfix = c.vin.as<float>();
    float* dmov = dfix + n;
    char* ws = (char*)c.spec.p;
    std::vector<float> hwin;
    if ((rc = pc_upload_windows(ws, L, window, st, hwin))) return rc;
    if ((e = cudaMemcpyAsync(dfix, fixed, n * 4, cudaMemcpyHostToDevice, st)) != cudaSuccess) return fail_cuda(e, what);
    if ((e = cudaMemcpyAsync(dmov, moving, n * 4, cudaMemcpyHostToDevice, st)) != cudaSuccess) return fail_cuda(e, what);
    int launches = 0;
    if ((e = pc_enqueue(dfix, dmov, ws, L, c.sms, st, launches)) != cudaSuccess) return fail_cuda(e, what);
    fy::count_launch(launches);
    if ((e = cudaMemcpyAsync(c.pin.p, ws + L.off_ctl, sizeof(PcCtl), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return fail_cuda(e, what);
    fy::ws_release(st);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return fail_cuda(e, what);
    const PcCtl* r = (const PcCtl*)c.pin.p;
    if (r->status) {
        shift[0] = shift[1] = shift[2] = 0.0;
        if (peak) *peak = 0.0;
        return 1;
    }
    shift[0] = r->shift[0]; shift[1] = r->shift[1]; shift[2] = r->shift[2];
    if (peak) *peak = r->peak;
    return 0;
}

// Device form for batches: `npairs` pairs of device volumes (fixed[i], moving[i] at stride
// nz*ny*nx floats), results written to the host arrays shift[3*npairs], peak[npairs],
// peak_index[npairs] (nullable) and status[npairs]. Synchronises `stream` at the end.
extern "C" size_t fy_gpu_phase_correlate_scratch_bytes(int nz, int ny, int nx) { return fy_pc_scratch_bytes(nz, ny, nx); }

extern "C" int fy_gpu_phase_correlate_batch(const float* d_fixed, const float* d_moving, int npairs, int nz, int ny,
                                            int nx, int window, void* d_scratch, double* shift, double* peak,
                                            long long* peak_index, int* status, void* stream) {
    fy::enter();
    const char* what = "fy_gpu_phase_correlate_batch";
    if (!d_fixed || !d_moving || !d_scratch || !shift || !status || npairs < 0) return fail(FY_EINVAL, "%s: bad args", what);
    if (nz < 2 || ny < 2 || nx < 2) return fail(FY_EINVAL, "%s: dims < 2", what);
    int rc = pc_check(nz, ny, nx, what);
    if (rc) return rc;
    if ((rc = fy::ensure_ctx())) return rc;
    fy::ThreadCtx& c = ctx();
    cudaStream_t st = (cudaStream_t)stream;
    const PcLayout L = pc_layout(nz, ny, nx);
    const size_t n = (size_t)nz * ny * nx;
    char* ws = (char*)d_scratch;
    std::vector<float> hwin;
    if ((rc = pc_upload_windows(ws, L, window, st, hwin))) return rc;
    cudaError_t e;
    if ((e = c.pin.ensure(sizeof(PcCtl) * (size_t)(npairs > 0 ? npairs : 1))) != cudaSuccess) return fail_cuda(e, what);
    PcCtl* host = (PcCtl*)c.pin.p;
    int launches = 0;
    for (int i = 0; i < npairs; ++i) {
        if ((e = pc_enqueue(d_fixed + (size_t)i * n, d_moving + (size_t)i * n, ws, L, c.sms, st, launches)) != cudaSuccess)
            return fail_cuda(e, what);
        if ((e = cudaMemcpyAsync(host + i, ws + L.off_ctl, sizeof(PcCtl), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
            return fail_cuda(e, what);
    }
    fy::count_launch(launches);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return fail_cuda(e, what);
    for (int i = 0; i < npairs; ++i) {
        for (int a = 0; a < 3; ++a) shift[3 * i + a] = host[i].status ? 0.0 : host[i].shift[a];
        if (peak) peak[i] = host[i].status ? 0.0 : host[i].peak;
        if (peak_index) peak_index[i] = host[i].peak_index;
        status[i] = host[i].status;
    }
    return FY_OK;
}
