// fy_noise.cu -- per-volume noise model fy_estimate_noise (noise.c:75-192) on the GPU.
//
//   1. k_noise_stats: local box sums over (2r+1)^3 windows with zero outside the volume and
//      the FIXED divisor win^3 (noise.c:20-59, 92-101): mean m and variance
//      v = max(S2/wc - m^2, 0). z-sliding like the guided kernel; sums are direct
//      (2r+1)-tap float sums of (I - c) and (I - c)^2 with a per-tile shift c, and interior
//      voxels use v = S2'/wc - (S1'/wc)^2, which equals the reference's S2/wc - (S1/wc)^2
//      without its cancellation.
//   2. Exact order statistics by radix select on orderable 32-bit float keys: the 1st and
//      99th percentiles of m (noise.c:104-108) and, per intensity bin with >= 200 voxels,
//      the flat_pct percentile of v (noise.c:117-134), each interpolated between
//      order statistics k and k+1 exactly as percentile() does (noise.c:66-73).
//   3. k_noise_fit: one thread, FP64: IRLS line fit var = g*I + b (noise.c:137-172) and
//      noise_ref = sqrt(max(g*ref + b, ..))*1.15 (noise.c:181-187), plus the guided eps
//      (3*noise_ref)^2 floored at 1e-8 (noise.c:197-202).
// The launch sequence is fixed (no host decisions), so a chain can keep it on one stream.
#include "fy_internal.h"

namespace {

constexpr int NB = 24;                 // intensity bins, noise.c:111
constexpr int NT_MAX = 64;             // selection targets: 2 per bin + spare
constexpr int DB_ALL = 11;             // digit bits for whole-volume selections (11/11/10)
constexpr int DB_BIN = 8;              // digit bits for per-bin selections (4 x 8)

FY_D uint32_t fkey(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
FY_HD float funkey(uint32_t k) {
#ifdef __CUDA_ARCH__
    const uint32_t u = (k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k;
    return __uint_as_float(u);
#else
    const uint32_t u = (k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k;
    float f;
    memcpy(&f, &u, 4);
    return f;
#endif
}

}  // namespace

// Device-resident control block of one estimate (lives in the caller's scratch).
struct NoiseCtl {
    // inputs
    long long n;
    double flat_pct, ref_intensity;
    // selection targets
    int ntarget;
    int tgroup[NT_MAX];                // group id: -1 = whole volume, 0..23 = bin
    long long trank[NT_MAX];           // remaining rank within the current prefix
    uint32_t tprefix[NT_MAX];          // decided high bits
    int tactive[NT_MAX];
    // results
    double lo, hi;
    double edge[NB + 1];
    long long bcount[NB];
    double bfloor[NB];
    int pct_k_lo, mode;                // mode: 0 means lo/hi, 1 bins, 2 whole-volume var fallback
    double pct_f_lo, pct_f_hi;
    double out_g, out_b, out_noise_ref, out_ref_intensity;
    int out_used;
    float eps;                         // fy_guided_eps_for_noise(noise_ref), for a chained guided filter
    unsigned int hist[NT_MAX * 256];   // per-target histogram (bins: 256; whole: up to 2048 over 4 targets)
};

namespace {

constexpr int SNT = 256, STY = 16, STX = 32;

// ---------------------------------------------------------------- 1. local stats
template <int R>
struct StatSmem {
    static constexpr int IY = STY + 2 * R, IX = STX + 2 * R, NR = 2 * R + 1;
    float I[NR][IY][IX];
    float xs1[IY][STX], xs2[IY][STX];
    float m1[NR][STY][STX], m2[NR][STY][STX];
};

template <int R>
__global__ void __launch_bounds__(SNT) k_noise_stats(const float* __restrict__ in, float* __restrict__ mean,
                                                     float* __restrict__ var, int nz, int ny, int nx,
                                                     float inv_wc, int wci, int zchunk) {
    using S = StatSmem<R>;
    extern __shared__ float4 smem4[];
    S& sm = *reinterpret_cast<S*>(smem4);
    const int x0 = blockIdx.x * STX, y0 = blockIdx.y * STY;
    const int zs = blockIdx.z * zchunk, ze = min(nz, zs + zchunk);
    const int t = threadIdx.x;
    const size_t plane = (size_t)ny * nx;
    const float c = __ldg(in + (size_t)zs * plane + (size_t)y0 * nx + x0);
    for (int zi = zs - R; zi < ze + R; ++zi) {
        const int slot = ((zi % S::NR) + S::NR) % S::NR;
        const bool zin = zi >= 0 && zi < nz;
        for (int k = t; k < S::IY * S::IX; k += SNT) {
            const int yy = k / S::IX, xx = k - yy * S::IX;
            const int gy = y0 - R + yy, gx = x0 - R + xx;
            float v = 0.f;
            if (zin && gy >= 0 && gy < ny && gx >= 0 && gx < nx) v = __ldg(in + (size_t)zi * plane + (size_t)gy * nx + gx) - c;
            sm.I[slot][yy][xx] = v;
        }
        __syncthreads();
        // X sums (shifted values, zero outside)
        for (int k = t; k < S::IY * STX; k += SNT) {
            const int yy = k / STX, xt = k - yy * STX;
            const int gx0 = x0 + xt;
            float s1 = 0.f, s2 = 0.f;
#pragma unroll
            for (int d = -R; d <= R; ++d) {
                const int g = gx0 + d;
                if (g >= 0 && g < nx) { const float u = sm.I[slot][yy][xt + R + d]; s1 += u; s2 += u * u; }
            }
            sm.xs1[yy][xt] = s1; sm.xs2[yy][xt] = s2;
        }
        __syncthreads();
        for (int k = t; k < STY * STX; k += SNT) {
            const int yt = k / STX, xt = k - yt * STX;
            float s1 = 0.f, s2 = 0.f;
#pragma unroll
            for (int d = -R; d <= R; ++d) { s1 += sm.xs1[yt + R + d][xt]; s2 += sm.xs2[yt + R + d][xt]; }
            sm.m1[slot][yt][xt] = s1; sm.m2[slot][yt][xt] = s2;
        }
        __syncthreads();
        const int zo = zi - R;
        if (zo >= zs && zo < ze) {
            const int cz = min(zo + R, nz - 1) - max(zo - R, 0) + 1;
            for (int k = t; k < STY * STX; k += SNT) {
                const int yt = k / STX, xt = k - yt * STX;
                const int gy = y0 + yt, gx = x0 + xt;
                if (gy >= ny || gx >= nx) continue;
                float s1 = 0.f, s2 = 0.f;
#pragma unroll
                for (int q = 0; q < S::NR; ++q) { s1 += sm.m1[q][yt][xt]; s2 += sm.m2[q][yt][xt]; }
                const int cy = min(gy + R, ny - 1) - max(gy - R, 0) + 1;
                const int cx = min(gx + R, nx - 1) - max(gx - R, 0) + 1;
                const int nini = cz * cy * cx;
                const float nin = (float)nini;
                // raw sums: S1 = S1' + nin*c, S2 = S2' + 2c*S1' + nin*c^2
                const float m = (s1 + nin * c) * inv_wc;
                float v;
                if (nini == wci) {                        // interior: shifted, cancellation-free
                    const float e1 = s1 * inv_wc;
                    v = s2 * inv_wc - e1 * e1;
                } else {
                    v = (s2 + 2.0f * c * s1 + nin * c * c) * inv_wc - m * m;
                }
                if (v < 0.f) v = 0.f;
                const size_t o = (size_t)zo * plane + (size_t)gy * nx + gx;
                mean[o] = m;
                var[o] = v;
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------- 2. radix select
// Group of element i: -1 (whole volume) for modes 0/2; bin id (or -2 = no bin) for mode 1.
FY_D int bin_of(float mv, const NoiseCtl* __restrict__ ctl) {
    const double m = (double)mv;
    if (!(m >= ctl->edge[0] && m < ctl->edge[NB])) return -2;
    int b = (int)((m - ctl->lo) / (ctl->hi - ctl->lo) * NB);
    if (b < 0) b = 0;
    if (b > NB - 1) b = NB - 1;
    while (b > 0 && m < ctl->edge[b]) --b;               // exact edges (noise.c:118-122)
    while (b < NB - 1 && m >= ctl->edge[b + 1]) ++b;
    return b;
}

// Histogram one digit (bits [shift, shift+db)) of every active target's prefix group.
template <int DB>
__global__ void __launch_bounds__(256) k_sel_hist(const float* __restrict__ mean, const float* __restrict__ var,
                                                  NoiseCtl* __restrict__ ctl, int shift, int want_mode) {
    extern __shared__ unsigned int h[];                  // ntarget << DB counters
    __shared__ int s_act;
    if (ctl->mode != want_mode) return;
    constexpr int NBK = 1 << DB;
    const int nt = ctl->ntarget;
    if (threadIdx.x == 0) {
        int a = 0;
        for (int t = 0; t < nt; ++t) a |= ctl->tactive[t];
        s_act = a;
    }
    for (int i = threadIdx.x; i < nt * NBK; i += blockDim.x) h[i] = 0;
    __syncthreads();
    if (!s_act) return;
    const long long n = ctl->n;
    const int mode = ctl->mode;
    const int top = shift + DB;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float mv = __ldg(mean + i);
        uint32_t key;
        int grp;
        if (mode == 0) { key = fkey(mv); grp = -1; }
        else if (mode == 1) { grp = bin_of(mv, ctl); if (grp < 0) continue; key = fkey(__ldg(var + i)); }
        else { key = fkey(__ldg(var + i)); grp = -1; }
        const uint32_t hi_bits = top >= 32 ? 0u : (key >> top);
        const int dig = (key >> shift) & (NBK - 1);
        if (mode == 1) {
            for (int t = 2 * grp; t < 2 * grp + 2; ++t)
                if (ctl->tactive[t] && ctl->tprefix[t] == hi_bits) atomicAdd(&h[t * NBK + dig], 1u);
        } else {
            for (int t = 0; t < nt; ++t)
                if (ctl->tactive[t] && ctl->tprefix[t] == hi_bits) atomicAdd(&h[t * NBK + dig], 1u);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nt * NBK; i += blockDim.x)
        if (h[i]) atomicAdd(&ctl->hist[i], h[i]);
}

// After a digit pass: every target picks the bucket holding its rank (one warp per target).
__global__ void k_sel_scan(NoiseCtl* __restrict__ ctl, int db, int want_mode) {
    if (ctl->mode != want_mode) return;
    const int t = blockIdx.x;
    if (t >= ctl->ntarget || !ctl->tactive[t]) return;
    const int nbk = 1 << db;
    unsigned int* h = ctl->hist + (size_t)t * nbk;
    if (threadIdx.x == 0) {
        long long r = ctl->trank[t], acc = 0;
        int b = 0;
        for (; b < nbk; ++b) {
            if (acc + (long long)h[b] > r) break;
            acc += h[b];
        }
        if (b == nbk) b = nbk - 1;                       // cannot happen for a valid rank
        ctl->trank[t] = r - acc;
        ctl->tprefix[t] = (ctl->tprefix[t] << db) | (uint32_t)b;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nbk; i += blockDim.x) h[i] = 0;
}

// percentile() interpolation (noise.c:69-72) from the two selected order statistics
FY_D double interp(const NoiseCtl* ctl, int t0, double f, bool has_next) {
    const double v0 = (double)funkey(ctl->tprefix[t0]);
    if (!has_next) return v0;
    const double v1 = (double)funkey(ctl->tprefix[t0 + 1]);
    return v0 * (1 - f) + v1 * f;
}

__global__ void k_noise_setup(NoiseCtl* ctl, long long n, double flat_pct, double ref_intensity) {
    ctl->n = n;
    ctl->flat_pct = flat_pct;
    ctl->ref_intensity = ref_intensity;
    ctl->mode = 0;
    // targets: 1st percentile (k, k+1) and 99th (k, k+1) of the means
    for (int t = 0; t < NT_MAX; ++t) { ctl->tactive[t] = 0; ctl->tprefix[t] = 0; ctl->trank[t] = 0; ctl->tgroup[t] = -1; }
    const double i1 = 1.0 / 100.0 * (double)(n - 1), i99 = 99.0 / 100.0 * (double)(n - 1);
    const long long k1 = (long long)i1, k99 = (long long)i99;
    ctl->pct_f_lo = i1 - (double)k1;
    ctl->pct_f_hi = i99 - (double)k99;
    ctl->trank[0] = k1;  ctl->tactive[0] = 1;
    ctl->trank[1] = k1 + 1; ctl->tactive[1] = (k1 + 1 < n);
    ctl->trank[2] = k99; ctl->tactive[2] = 1;
    ctl->trank[3] = k99 + 1; ctl->tactive[3] = (k99 + 1 < n);
    ctl->ntarget = 4;
}

// lo/hi from the selected means; bin edges; bin counts are filled by k_bin_count next.
__global__ void k_noise_bins_setup(NoiseCtl* ctl) {
    const long long n = ctl->n;
    const double i1 = 1.0 / 100.0 * (double)(n - 1), i99 = 99.0 / 100.0 * (double)(n - 1);
    const long long k1 = (long long)i1, k99 = (long long)i99;
    double lo = interp(ctl, 0, ctl->pct_f_lo, k1 + 1 < n);
    double hi = interp(ctl, 2, ctl->pct_f_hi, k99 + 1 < n);
    if (hi <= lo) hi = lo + 1e-6;                       // noise.c:109
    ctl->lo = lo; ctl->hi = hi;
    for (int k = 0; k <= NB; ++k) ctl->edge[k] = lo + (hi - lo) * k / NB;   // noise.c:118-119
    for (int b = 0; b < NB; ++b) ctl->bcount[b] = 0;
    ctl->mode = 1;
}

__global__ void __launch_bounds__(256) k_bin_count(const float* __restrict__ mean, NoiseCtl* __restrict__ ctl) {
    __shared__ unsigned long long cnt[NB];
    if (threadIdx.x < NB) cnt[threadIdx.x] = 0;
    __syncthreads();
    const long long n = ctl->n;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int b = bin_of(__ldg(mean + i), ctl);
        if (b >= 0) atomicAdd(&cnt[b], 1ull);
    }
    __syncthreads();
    if (threadIdx.x < NB && cnt[threadIdx.x]) atomicAdd((unsigned long long*)&ctl->bcount[threadIdx.x], cnt[threadIdx.x]);
}

// per-bin targets (k, k+1) of the flat_pct percentile, bins with >= 200 voxels (noise.c:123)
__global__ void k_bin_targets(NoiseCtl* ctl) {
    ctl->ntarget = 2 * NB;
    for (int b = 0; b < NB; ++b) {
        const long long c = ctl->bcount[b];
        const bool on = c >= 200;
        const double idx = ctl->flat_pct / 100.0 * (double)(c - 1);
        const long long k = on ? (long long)idx : 0;
        ctl->tgroup[2 * b] = ctl->tgroup[2 * b + 1] = b;
        ctl->tprefix[2 * b] = ctl->tprefix[2 * b + 1] = 0;
        ctl->trank[2 * b] = k; ctl->tactive[2 * b] = on;
        ctl->trank[2 * b + 1] = k + 1; ctl->tactive[2 * b + 1] = on && (k + 1 < c);
    }
}

FY_D void sort_small(double* v, int n) {
    for (int i = 1; i < n; ++i) {
        const double k = v[i];
        int j = i - 1;
        while (j >= 0 && v[j] > k) { v[j + 1] = v[j]; --j; }
        v[j + 1] = k;
    }
}
FY_D double pct_small(double* v, int n, double pct) {       // percentile() on <= 24 values
    if (n <= 0) return 0.0;
    sort_small(v, n);
    const double idx = pct / 100.0 * (n - 1);
    const int lo = (int)idx;
    const double f = idx - lo;
    if (lo + 1 < n) return v[lo] * (1 - f) + v[lo + 1] * f;
    return v[lo];
}

// Collect bin floors, then either fit (>= 1 bin) or arm the whole-volume var fallback.
__global__ void k_noise_fit(NoiseCtl* ctl, int stage) {
    if (stage == 0) {
        int used = 0;
        for (int b = 0; b < NB; ++b) {
            const long long c = ctl->bcount[b];
            if (c < 200) continue;
            const double idx = ctl->flat_pct / 100.0 * (double)(c - 1);
            const long long k = (long long)idx;
            ctl->bfloor[b] = interp(ctl, 2 * b, idx - (double)k, k + 1 < c);
            ++used;
        }
        ctl->out_used = used;
        if (used == 0) {                                  // noise.c:166-171 fallback
            const long long n = ctl->n;
            const double idx = ctl->flat_pct / 100.0 * (double)(n - 1);
            const long long k = (long long)idx;
            ctl->pct_f_lo = idx - (double)k;
            for (int t = 0; t < NT_MAX; ++t) { ctl->tactive[t] = 0; ctl->tprefix[t] = 0; }
            ctl->ntarget = 2;
            ctl->trank[0] = k; ctl->tactive[0] = 1;
            ctl->trank[1] = k + 1; ctl->tactive[1] = k + 1 < n;
            ctl->mode = 2;
        } else {
            ctl->mode = 3;
        }
        return;
    }
    // stage 1: the fit itself (FP64)
    double bin_i[NB], bin_f[NB], wv[NB];
    long long bin_c[NB];
    int used = 0;
    for (int b = 0; b < NB; ++b) {
        if (ctl->bcount[b] < 200) continue;
        bin_i[used] = 0.5 * (ctl->edge[b] + ctl->edge[b + 1]);
        bin_f[used] = ctl->bfloor[b];
        bin_c[used] = ctl->bcount[b];
        ++used;
    }
    double g = 0, bb = 0;
    if (ctl->mode == 2) {
        const long long n = ctl->n;
        const double idx = ctl->flat_pct / 100.0 * (double)(n - 1);
        bb = interp(ctl, 0, ctl->pct_f_lo, (long long)idx + 1 < n);
        g = 0;
    } else if (used >= 3) {                               // IRLS, noise.c:139-161
        for (int i = 0; i < used; i++) wv[i] = sqrt((double)bin_c[i]);
        for (int it = 0; it < 4; it++) {
            double Sw = 0, Swx = 0, Swy = 0, Swxx = 0, Swxy = 0;
            for (int i = 0; i < used; i++) {
                const double wi = wv[i], xi = bin_i[i], yi = bin_f[i];
                Sw += wi; Swx += wi * xi; Swy += wi * yi; Swxx += wi * xi * xi; Swxy += wi * xi * yi;
            }
            const double det = Sw * Swxx - Swx * Swx;
            if (fabs(det) < 1e-20) break;
            g = (Sw * Swxy - Swx * Swy) / det;
            bb = (Swxx * Swy - Swx * Swxy) / det;
            double resid[NB], rc[NB];
            for (int i = 0; i < used; i++) { resid[i] = fabs(bin_f[i] - (g * bin_i[i] + bb)); rc[i] = resid[i]; }
            const double med = pct_small(rc, used, 50.0) + 1e-9;
            for (int i = 0; i < used; i++) {
                const double rr = resid[i] / (2.0 * med);
                wv[i] = sqrt((double)bin_c[i]) / (1.0 + rr * rr);
            }
        }
    } else if (used > 0) {                                // noise.c:162-165
        double s = 0;
        for (int i = 0; i < used; i++) s += bin_f[i];
        bb = s / used; g = 0;
    }
    if (!isfinite(g)) g = 0;
    if (!isfinite(bb)) bb = 0;
    double var_ref = g * ctl->ref_intensity + bb;
    if (var_ref < 0) var_ref = bb > 0 ? bb : 0;
    const double noise_ref = sqrt(var_ref) * 1.15;
    ctl->out_g = g; ctl->out_b = bb;
    ctl->out_noise_ref = noise_ref;
    ctl->out_ref_intensity = ctl->ref_intensity;
    double eps = (3.0 * noise_ref) * (3.0 * noise_ref);
    if (!(eps > 1e-8)) eps = 1e-8;
    ctl->eps = (float)eps;
}

unsigned grid_sel(long long n, int sms) {
    long long g = (n + 255) / 256;
    const long long cap = (long long)sms * 4;
    return (unsigned)(g < cap ? (g ? g : 1) : cap);
}

}  // namespace

size_t fy_noise_ctl_bytes() { return (sizeof(NoiseCtl) + 255) & ~(size_t)255; }

size_t fy_noise_stats_smem(int r) {
    switch (r) {
        case 1: return sizeof(StatSmem<1>);
        case 2: return sizeof(StatSmem<2>);
        case 3: return sizeof(StatSmem<3>);
        case 4: return sizeof(StatSmem<4>);
        default: return 0;
    }
}

// Enqueue the whole estimate. scratch: 2n floats (mean, var); ctl: fy_noise_ctl_bytes().
// Supports win in {3..9} (r = win/2 <= 4).
cudaError_t fy_launch_estimate_noise(const float* in, int nz, int ny, int nx, int win, double flat_pct,
                                     double ref_intensity, float* scratch, void* ctl_mem, int sms,
                                     cudaStream_t st, int& launches) {
    NoiseCtl* ctl = (NoiseCtl*)ctl_mem;
    const long long n = (long long)nz * ny * nx;
    float* mean = scratch;
    float* var = scratch + n;
    const int r = win / 2;
    const float inv_wc = (float)(1.0 / ((double)win * win * win));
    // 1. stats
    {
        const dim3 tiles(ceil_div_i(nx, STX), ceil_div_i(ny, STY), 1);
        const long txy = (long)tiles.x * tiles.y;
        int nchunk = (int)((4L * sms + txy - 1) / txy);
        if (nchunk > nz / (8 * r)) nchunk = nz / (8 * r);
        if (nchunk < 1) nchunk = 1;
        const int zchunk = ceil_div_i(nz, nchunk);
        dim3 grid(tiles.x, tiles.y, ceil_div_i(nz, zchunk));
        const size_t smem = fy_noise_stats_smem(r);
        cudaError_t e0;
#define FY_NS(RR)                                                                            \
        if ((e0 = fy_smem_optin(k_noise_stats<RR>, smem)) != cudaSuccess) return e0;         \
        k_noise_stats<RR><<<grid, SNT, smem, st>>>(in, mean, var, nz, ny, nx, inv_wc, win * win * win, zchunk);
        switch (r) {
            case 1: FY_NS(1) break;
            case 2: FY_NS(2) break;
            case 3: FY_NS(3) break;
            case 4: FY_NS(4) break;
            default: return cudaErrorInvalidValue;
        }
#undef FY_NS
        launches += 1;
    }
    const unsigned g = grid_sel(n, sms);
    unsigned int* hist = ctl->hist;
    const size_t hist_bytes = sizeof(ctl->hist);
    const size_t smem_all = 4 * 2048 * sizeof(unsigned int), smem_bin = 2 * NB * 256 * sizeof(unsigned int);
    cudaError_t e;
    if ((e = fy_smem_optin(k_sel_hist<DB_ALL>, smem_all)) != cudaSuccess) return e;
    if ((e = fy_smem_optin(k_sel_hist<DB_BIN>, smem_bin)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(hist, 0, hist_bytes, st)) != cudaSuccess) return e;
    k_noise_setup<<<1, 1, 0, st>>>(ctl, n, flat_pct, ref_intensity);
    // 2a. 1st/99th percentile of the means: 11 + 11 + 10 bits
    const int all_digits[3][2] = {{21, 11}, {10, 11}, {0, 10}};
    for (auto& dg : all_digits) {
        k_sel_hist<DB_ALL><<<g, 256, smem_all, st>>>(mean, var, ctl, dg[0], 0);
        k_sel_scan<<<4, 256, 0, st>>>(ctl, dg[1], 0);
    }
    k_noise_bins_setup<<<1, 1, 0, st>>>(ctl);
    k_bin_count<<<g, 256, 0, st>>>(mean, ctl);
    k_bin_targets<<<1, 1, 0, st>>>(ctl);
    if ((e = cudaMemsetAsync(hist, 0, hist_bytes, st)) != cudaSuccess) return e;
    // 2b. per-bin flat_pct percentile of the variance: 4 x 8 bits
    for (int sh = 24; sh >= 0; sh -= 8) {
        k_sel_hist<DB_BIN><<<g, 256, smem_bin, st>>>(mean, var, ctl, sh, 1);
        k_sel_scan<<<2 * NB, 256, 0, st>>>(ctl, 8, 1);
    }
    k_noise_fit<<<1, 1, 0, st>>>(ctl, 0);
    if ((e = cudaMemsetAsync(hist, 0, hist_bytes, st)) != cudaSuccess) return e;
    // 2c. fallback (mode 2 only): flat_pct percentile over all voxels' variance
    for (auto& dg : all_digits) {
        k_sel_hist<DB_ALL><<<g, 256, smem_all, st>>>(mean, var, ctl, dg[0], 2);
        k_sel_scan<<<2, 256, 0, st>>>(ctl, dg[1], 2);
    }
    k_noise_fit<<<1, 1, 0, st>>>(ctl, 1);
    launches += 1 + 6 + 3 + 8 + 1 + 6 + 1;
    return cudaGetLastError();
}

// Copy the model out of a finished control block (device -> host, async on st).
cudaError_t fy_noise_read(const void* ctl_mem, double* g, double* b, double* noise_ref, double* ref_intensity,
                          int* used, cudaStream_t st) {
    static_assert(sizeof(double) == 8, "");
    const NoiseCtl* ctl = (const NoiseCtl*)ctl_mem;
    cudaError_t e;
    if ((e = cudaMemcpyAsync(g, &ctl->out_g, 8, cudaMemcpyDeviceToHost, st))) return e;
    if ((e = cudaMemcpyAsync(b, &ctl->out_b, 8, cudaMemcpyDeviceToHost, st))) return e;
    if ((e = cudaMemcpyAsync(noise_ref, &ctl->out_noise_ref, 8, cudaMemcpyDeviceToHost, st))) return e;
    if ((e = cudaMemcpyAsync(ref_intensity, &ctl->out_ref_intensity, 8, cudaMemcpyDeviceToHost, st))) return e;
    return cudaMemcpyAsync(used, &ctl->out_used, 4, cudaMemcpyDeviceToHost, st);
}

const float* fy_noise_eps_ptr(const void* ctl_mem) { return &((const NoiseCtl*)ctl_mem)->eps; }
