// fy_fft.cuh -- CTA-cooperative shared-memory FFTs for sizes 2^k and 3*2^k (k >= 0).
//
// A tile is W independent complex lines of n points. Each line is transformed by
// TPL = n/E threads that each own E points in registers (E = 16 for 2^k, 24 for 3*2^k,
// E = n below those sizes), so every radix pass is E/R in-register butterflies per
// thread and the data crosses shared memory only between passes. Shared memory holds a
// tile point-major, element (point i, line l) at s[i*LP + l]; with the line index the
// fastest-varying thread index, every exchange is a run of consecutive float2s (no bank
// conflicts beyond the two wavefronts of a 256-byte warp access).
//
// The transform is a mixed-radix Stockham autosort (no bit reversal): one radix-3 pass
// first for n = 3*2^k, then radix-8 passes and a final radix-4 or radix-2 pass. It
// computes the same unnormalised DFT as fy_fft1d (fft.c:168-173):
// X[k] = sum_t x[t] exp(sign*2*pi*i*k*t/n), sign -1 forward, +1 inverse.
// Twiddles come from a per-size table of exp(+2*pi*i*m/n) generated in FP64 on the host and
// rounded once to float (fft.c:47-61 does the same); the sign multiplies the imaginary
// part (fft.c:93).
//
// Pass p with radix R and span Ns = C*2^m (C = 3 after a radix-3 pass, else 1): butterfly
// j < n/R reads points j + r*n/R, multiplies input r by w^(r*(j mod Ns)) with
// w = exp(sign*2*pi*i/(Ns*R)), applies a radix-R DFT and writes point
// (j div Ns)*Ns*R + (j mod Ns) + r*Ns. Thread tl of a line owns butterflies
// j = tl + TPL*b, b < E/R. Pass 0 inputs and last-pass outputs both sit at
// j + r*n/R, so a caller can load/store them straight from/to global memory.
#pragma once
#include <type_traits>
#include "fy_common.cuh"

#define FY_FFT_MAXPASS 14
#define FY_FFT_TILE_ELEMS 8192   // W * n per tile (64 KB of float2)
#define FY_FFT_MAXN 4096
#define FY_FFT_MAXNT 512

struct FftPlan {
    int n;
    int npass;
    int has3;                       // first pass is radix 3
    int radix[FY_FFT_MAXPASS];
    int nslog[FY_FFT_MAXPASS];      // Ns = (has3 && p > 0 ? 3 : 1) << nslog[p]
};

// Supported FFT length (2^k or 3*2^k) -- the sizes fy_next_fft_size produces.
FY_HD bool fy_fft_len_ok(int n) {
    if (n < 1 || n > FY_FFT_MAXN) return false;
    if (n % 3 == 0) n /= 3;
    return (n & (n - 1)) == 0;
}

// Elements per thread for a length-n line.
FY_HD int fy_fft_e(int n) {
    if (n % 3 == 0) return n >= 24 ? 24 : n;
    return n >= 16 ? 16 : n;
}

inline FftPlan fy_make_plan(int n) {
    FftPlan p{};
    p.n = n;
    int m = n, lg = 0;
    if (m % 3 == 0) { p.has3 = 1; p.radix[p.npass] = 3; p.nslog[p.npass++] = 0; m /= 3; }
    while (m % 8 == 0) { p.radix[p.npass] = 8; p.nslog[p.npass++] = lg; lg += 3; m /= 8; }
    if (m % 4 == 0) { p.radix[p.npass] = 4; p.nslog[p.npass++] = lg; lg += 2; m /= 4; }
    if (m % 2 == 0) { p.radix[p.npass] = 2; p.nslog[p.npass++] = lg; lg += 1; m /= 2; }
    return p;
}

// Lines per tile: largest power of two <= 16 with W*n <= FY_FFT_TILE_ELEMS.
FY_HD int fy_tile_lines(int n) {
    int w = 16;
    while (w > 1 && w * n > FY_FFT_TILE_ELEMS) w >>= 1;
    return w;
}
FY_HD int fy_log2i(int w) { int l = 0; while ((1 << l) < w) ++l; return l; }

// ---------------------------------------------------------------- radix butterflies
// In-register DFT of size R with omega = exp(sign*2*pi*i/R).
template <int R> struct Bfly;
template <> struct Bfly<2> {
    static FY_D void run(float2* v, float) {
        float2 a = v[0], b = v[1];
        v[0] = cadd(a, b); v[1] = csub(a, b);
    }
};
template <> struct Bfly<3> {
    static FY_D void run(float2* v, float sign) {
        const float c3 = 0.86602540378443864676f;           // sqrt(3)/2
        float2 t1 = cadd(v[1], v[2]);
        float2 t2 = make_float2(v[0].x - 0.5f * t1.x, v[0].y - 0.5f * t1.y);
        float2 t3 = cmul_is(csub(v[1], v[2]), sign * c3);   // i*sign*(sqrt3/2)*(v1-v2)
        v[0] = cadd(v[0], t1);
        v[1] = cadd(t2, t3);
        v[2] = csub(t2, t3);
    }
};
template <> struct Bfly<4> {
    static FY_D void run(float2* v, float sign) {
        float2 a = cadd(v[0], v[2]), b = csub(v[0], v[2]);
        float2 c = cadd(v[1], v[3]), d = cmul_is(csub(v[1], v[3]), sign);
        v[0] = cadd(a, c); v[2] = csub(a, c);
        v[1] = cadd(b, d); v[3] = csub(b, d);
    }
};
template <> struct Bfly<8> {
    static FY_D void run(float2* v, float sign) {
        float2 e[4] = {v[0], v[2], v[4], v[6]};
        float2 o[4] = {v[1], v[3], v[5], v[7]};
        Bfly<4>::run(e, sign);
        Bfly<4>::run(o, sign);
        const float h = 0.70710678118654752440f;             // sqrt(2)/2
        // o[k] *= omega8^k, omega8 = h*(1 + i*sign)
        float2 o1 = make_float2(h * (o[1].x - sign * o[1].y), h * (o[1].y + sign * o[1].x));
        float2 o2 = cmul_is(o[2], sign);
        float2 o3 = make_float2(h * (-o[3].x - sign * o[3].y), h * (-o[3].y + sign * o[3].x));
        v[0] = cadd(e[0], o[0]); v[4] = csub(e[0], o[0]);
        v[1] = cadd(e[1], o1);   v[5] = csub(e[1], o1);
        v[2] = cadd(e[2], o2);   v[6] = csub(e[2], o2);
        v[3] = cadd(e[3], o3);   v[7] = csub(e[3], o3);
    }
};

// ---------------------------------------------------------------- per-pass helpers
// Input point of slot (b, r) for a radix-R pass: j + r*n/R, j = tl + tpl*b.
template <int E, int R, class LD>
FY_D void pass_load(float2 (&v)[E], int n, int tl, int tpl, LD ld) {
    const int nR = n / R;
#pragma unroll
    for (int b = 0; b < E / R; ++b)
#pragma unroll
        for (int r = 0; r < R; ++r) v[b * R + r] = ld(tl + tpl * b + r * nR);
}

// Twiddle + butterfly. C is the odd factor of Ns (3 after a radix-3 pass, else 1).
template <int E, int R, int C>
FY_D void pass_compute(float2 (&v)[E], int n, int tl, int tpl, int nslog,
                       const float2* __restrict__ tw, float sign) {
    const int Ns = C << nslog;
    if (Ns > 1) {
        const int tws = (n / (C * R)) >> nslog;              // n / (Ns*R)
#pragma unroll
        for (int b = 0; b < E / R; ++b) {
            const int j = tl + tpl * b;
            const int k = j - ((j >> nslog) / C) * Ns;       // j mod Ns
#pragma unroll
            for (int r = 1; r < R; ++r) {
                float2 w = tw[r * k * tws];
                w.y *= sign;
                v[b * R + r] = cmul(v[b * R + r], w);
            }
        }
    }
#pragma unroll
    for (int b = 0; b < E / R; ++b) Bfly<R>::run(&v[b * R], sign);
}

// Output point of slot (b, r): (j div Ns)*Ns*R + (j mod Ns) + r*Ns.
template <int E, int R, int C, class ST>
FY_D void pass_store(const float2 (&v)[E], int tl, int tpl, int nslog, ST st) {
    const int Ns = C << nslog;
#pragma unroll
    for (int b = 0; b < E / R; ++b) {
        const int j = tl + tpl * b;
        const int q = (j >> nslog) / C;
        const int base = q * Ns * R + (j - q * Ns);
#pragma unroll
        for (int r = 0; r < R; ++r) st(base + r * Ns, v[b * R + r]);
    }
}

// Radix dispatch restricted to radices that divide E (others cannot occur for that E).
template <int E, class F>
FY_D void with_radix(int R, F&& f) {
    if constexpr (E % 8 == 0) { if (R == 8) { f(std::integral_constant<int, 8>{}); return; } }
    if constexpr (E % 4 == 0) { if (R == 4) { f(std::integral_constant<int, 4>{}); return; } }
    if constexpr (E % 3 == 0) { if (R == 3) { f(std::integral_constant<int, 3>{}); return; } }
    if constexpr (E % 2 == 0) { if (R == 2) { f(std::integral_constant<int, 2>{}); return; } }
}

// Full line transform. `ld(i)` supplies input point i (called once per owned point,
// before any shared-memory write); `st(i, v)` receives output point i. Pass boundaries
// exchange through shared memory at sline[i*ps] (sline = this thread's line: s + l for a
// point-major tile of pitch ps, or s + l*pitch with ps = 1 for a line-major tile). All
// threads of the CTA must call this together (it contains __syncthreads()).
template <int E, class LD, class ST>
FY_D void line_fft(float2* __restrict__ sline, int ps, int tl, const FftPlan& pl,
                   const float2* __restrict__ tw, float sign, LD ld, ST st) {
    constexpr int C = (E % 3 == 0) ? 3 : 1;
    const int n = pl.n, tpl = n / E;
    float2 v[E];
    if (pl.npass == 0) {                                     // n == 1: identity
        v[0] = ld(0);
        __syncthreads();
        st(0, v[0]);
        return;
    }
    with_radix<E>(pl.radix[0], [&](auto Rc) { pass_load<E, decltype(Rc)::value>(v, n, tl, tpl, ld); });
    __syncthreads();
    auto sld = [&](int i) { return sline[i * ps]; };
    auto sst = [&](int i, float2 x) { sline[i * ps] = x; };
    for (int p = 0; p < pl.npass; ++p) {
        const int R = pl.radix[p];
        const int nslog = pl.nslog[p];
        const bool last = p + 1 == pl.npass;
        with_radix<E>(R, [&](auto Rc) {
            constexpr int RR = decltype(Rc)::value;
            // the radix-3 pass (always first) has Ns = 1: odd factor 1
            if (RR == 3 || p == 0) {
                pass_compute<E, RR, 1>(v, n, tl, tpl, nslog, tw, sign);
                if (last) pass_store<E, RR, 1>(v, tl, tpl, nslog, st);
                else pass_store<E, RR, 1>(v, tl, tpl, nslog, sst);
            } else {
                pass_compute<E, RR, C>(v, n, tl, tpl, nslog, tw, sign);
                if (last) pass_store<E, RR, C>(v, tl, tpl, nslog, st);
                else pass_store<E, RR, C>(v, tl, tpl, nslog, sst);
            }
        });
        if (last) break;
        __syncthreads();
        with_radix<E>(pl.radix[p + 1], [&](auto Rc) { pass_load<E, decltype(Rc)::value>(v, n, tl, tpl, sld); });
        __syncthreads();
    }
}

// ---------------------------------------------------------------- compile-time plans
// The same transform with n, the pass sequence and the exchange pitch PS known at compile
// time, so every index and twiddle offset folds to a constant or a single multiply-add.
// Results are bit-identical to line_fft (same twiddles, same butterfly order).
constexpr bool ct_has3(int n) { return n % 3 == 0; }
constexpr int ct_log2(int m) { return m <= 1 ? 0 : 1 + ct_log2(m / 2); }
constexpr int ct_lg(int n) { return ct_log2(ct_has3(n) ? n / 3 : n); }
constexpr int ct_npass(int n) { return (ct_has3(n) ? 1 : 0) + ct_lg(n) / 3 + (ct_lg(n) % 3 ? 1 : 0); }
constexpr int ct_radix(int n, int p) {
    return (ct_has3(n) && p == 0) ? 3
           : ((p - (ct_has3(n) ? 1 : 0)) < ct_lg(n) / 3 ? 8 : (ct_lg(n) % 3 == 2 ? 4 : 2));
}
constexpr int ct_nslog(int n, int p) { return (ct_has3(n) && p == 0) ? 0 : 3 * (p - (ct_has3(n) ? 1 : 0)); }
constexpr int ct_odd(int n, int p) { return (ct_has3(n) && p > 0) ? 3 : 1; }
constexpr int ct_tile_lines(int n) {
    return n * 16 <= FY_FFT_TILE_ELEMS ? 16
           : (n * 8 <= FY_FFT_TILE_ELEMS ? 8 : (n * 4 <= FY_FFT_TILE_ELEMS ? 4 : (n * 2 <= FY_FFT_TILE_ELEMS ? 2 : 1)));
}

template <int N, int E, int R, int PS, class LD>
FY_D void ct_load(float2 (&v)[E], int tl, LD ld) {
    constexpr int TPL = N / E, NR = N / R;
#pragma unroll
    for (int b = 0; b < E / R; ++b)
#pragma unroll
        for (int r = 0; r < R; ++r) v[b * R + r] = ld(tl + TPL * b + r * NR);
}

template <int N, int E, int R, int C, int NSLOG, int SIGN>
FY_D void ct_compute(float2 (&v)[E], int tl, const float2* __restrict__ tw) {
    constexpr int TPL = N / E, NS = C << NSLOG, TWS = N / (NS * R);
    if constexpr (NS > 1) {
#pragma unroll
        for (int b = 0; b < E / R; ++b) {
            const int j = tl + TPL * b;
            const int k = C == 1 ? (j & (NS - 1)) : j - ((j >> NSLOG) / C) * NS;   // j mod Ns
            const int kt = k * TWS;
#pragma unroll
            for (int r = 1; r < R; ++r) {
                float2 w = tw[r * kt];
                if (SIGN < 0) w.y = -w.y;
                v[b * R + r] = cmul(v[b * R + r], w);
            }
        }
    }
#pragma unroll
    for (int b = 0; b < E / R; ++b) Bfly<R>::run(&v[b * R], (float)SIGN);
}

template <int N, int E, int R, int C, int NSLOG, class ST>
FY_D void ct_store(const float2 (&v)[E], int tl, ST st) {
    constexpr int TPL = N / E, NS = C << NSLOG;
#pragma unroll
    for (int b = 0; b < E / R; ++b) {
        const int j = tl + TPL * b;
        const int q = C == 1 ? (j >> NSLOG) : (j >> NSLOG) / C;
        const int base = q * NS * R + (j - q * NS);
#pragma unroll
        for (int r = 0; r < R; ++r) st(base + r * NS, v[b * R + r]);
    }
}

template <int N, int E, int PS, int SIGN, int P, class ST>
FY_D void ct_passes(float2 (&v)[E], float2* __restrict__ sline, int tl, const float2* __restrict__ tw, ST st) {
    constexpr int R = ct_radix(N, P), C = ct_odd(N, P), NSLOG = ct_nslog(N, P);
    ct_compute<N, E, R, C, NSLOG, SIGN>(v, tl, tw);
    if constexpr (P + 1 == ct_npass(N)) {
        ct_store<N, E, R, C, NSLOG>(v, tl, st);
    } else {
        ct_store<N, E, R, C, NSLOG>(v, tl, [&](int i, float2 x) { sline[i * PS] = x; });
        __syncthreads();
        ct_load<N, E, ct_radix(N, P + 1), PS>(v, tl, [&](int i) { return sline[i * PS]; });
        __syncthreads();
        ct_passes<N, E, PS, SIGN, P + 1>(v, sline, tl, tw, st);
    }
}

// Compile-time counterpart of line_fft (N >= 2): same contract, sign as SIGN = -1 / +1.
template <int N, int E, int PS, int SIGN, class LD, class ST>
FY_D void line_fft_ct(float2* __restrict__ sline, int tl, const float2* __restrict__ tw, LD ld, ST st) {
    static_assert(N % E == 0 && E % ct_radix(N, 0) == 0, "E must hold whole radix groups");
    float2 v[E];
    ct_load<N, E, ct_radix(N, 0), PS>(v, tl, ld);
    __syncthreads();
    ct_passes<N, E, PS, SIGN, 0>(v, sline, tl, tw, st);
}

// cooperative copy of the n-entry twiddle table into shared memory
FY_D void load_twiddles(float2* __restrict__ dst, const float2* __restrict__ src, int n) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
}
