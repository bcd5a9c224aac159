// fy_psf.cu -- the PSF edge fit of pass-1 calibration (measure_tile_psf_sigma,
// pipeline.c:107-196) on the GPU, one CTA.
//
// The reference draws candidate lines from an LCG reseeded to 1 per call (:111-112, :124):
// up to 2500 y lines, then up to 2500 x lines, keeping the first 400 that pass the edge
// tests, in draw order. Here every candidate of an axis is tested at once (its generator
// state by jumping the LCG ahead, three draws per candidate), one thread walks the accept
// flags in draw order, the kept profiles are rebuilt in shared memory, one thread per grid
// point accumulates the super-sampled edge spread function over the profiles in order, and
// one thread fits the line spread function's second moment. FP64 throughout, operation for
// operation as the oracle restatement.
#include "fy_context.h"

#include <math.h>

using fy::ctx;
using fy::fail;
using fy::fail_cuda;

namespace {

constexpr int kHalf = 7, kPlen = 2 * kHalf + 1, kGlen = 2 * kHalf * 8 + 1, kMaxE = 400, kIters = 2500;
constexpr int kT = 512;

struct Lcg {
    unsigned a, c;            // s -> a*s + c (mod 2^32)
};
__device__ __forceinline__ Lcg lcg_after(Lcg f, Lcg g) { return {f.a * g.a, f.a * g.c + f.c}; }
// the generator applied n times
__device__ Lcg lcg_pow(unsigned n) {
    Lcg r{1u, 0u}, b{1103515245u, 12345u};
    while (n) {
        if (n & 1u) r = lcg_after(b, r);
        b = lcg_after(b, b);
        n >>= 1;
    }
    return r;
}
__device__ __forceinline__ unsigned draw(unsigned& s) {
    s = s * 1103515245u + 12345u;
    return (s >> 16) & 0x7fffu;
}

// Candidate `k` of axis `ax` with the generator `off` draws in: 1 and e[], *cross when the
// line is an accepted edge (pipeline.c:126-161).
__device__ int psf_candidate(const uint8_t* __restrict__ vol, int Z, int Y, int X, int ax, unsigned off, int k,
                             double* e, double* cross) {
    const Lcg j = lcg_pow(off + 3u * (unsigned)k);
    unsigned s = j.a * 1u + j.c;
    int line[kPlen];
    if (ax == 1) {
        const int z = (int)(draw(s) % (unsigned)Z);
        const int y = kHalf + (int)(draw(s) % (unsigned)(Y - 2 * kHalf));
        const int x = (int)(draw(s) % (unsigned)X);
        for (int i = 0; i < kPlen; i++) line[i] = vol[((size_t)z * Y + (y - kHalf + i)) * X + x];
    } else {
        const int z = (int)(draw(s) % (unsigned)Z);
        const int y = (int)(draw(s) % (unsigned)Y);
        const int x = kHalf + (int)(draw(s) % (unsigned)(X - 2 * kHalf));
        for (int i = 0; i < kPlen; i++) line[i] = vol[((size_t)z * Y + y) * X + (x - kHalf + i)];
    }
    const double lo = __dmul_rn(0.5, (double)(line[0] + line[1]));
    const double hi = __dmul_rn(0.5, (double)(line[kPlen - 1] + line[kPlen - 2]));
    if (fabs(__dsub_rn(hi, lo)) < 40.0) return 0;
    int sv[kPlen];
    for (int i = 0; i < kPlen; i++) sv[i] = hi > lo ? line[i] : line[kPlen - 1 - i];
    double dmin = 1e9, dmax = -1e9;
    int amax = 0;
    for (int i = 0; i < kPlen - 1; i++) {
        const double d = __dsub_rn((double)sv[i + 1], (double)sv[i]);
        if (d < dmin) dmin = d;
        if (d > dmax) { dmax = d; amax = i; }
    }
    if (dmin < -8) return 0;
    if (!(amax == kHalf - 1 || amax == kHalf || amax == kHalf + 1)) return 0;
    int smin = sv[0];
    for (int i = 1; i < kPlen; i++) smin = sv[i] < smin ? sv[i] : smin;
    double emax = 0;
    for (int i = 0; i < kPlen; i++) { e[i] = (double)(sv[i] - smin); emax = e[i] > emax ? e[i] : emax; }
    if (emax <= 0) return 0;
    for (int i = 0; i < kPlen; i++) e[i] = __ddiv_rn(e[i], emax);
    int idx0 = -1;
    for (int i = 0; i < kPlen; i++)
        if (e[i] >= 0.5) { idx0 = i; break; }
    if (idx0 <= 0) return 0;
    const double frac = __ddiv_rn(__dsub_rn(0.5, e[idx0 - 1]), __dadd_rn(__dsub_rn(e[idx0], e[idx0 - 1]), 1e-9));
    *cross = __dadd_rn((double)(idx0 - 1), frac);
    return 1;
}

struct PsfOut {
    double sigma;
    int nprof;
};

__global__ void __launch_bounds__(kT) k_psf(const uint8_t* __restrict__ vol, int Z, int Y, int X, PsfOut* out) {
    __shared__ unsigned char flag[kIters];
    __shared__ short pick[kMaxE];            // kept candidates: index (axis 2 offset by kIters)
    __shared__ double cross[kMaxE];
    __shared__ double esf[kGlen];
    __shared__ int s_n;
    extern __shared__ double prof[];         // [kMaxE][kPlen]
    const int t = threadIdx.x;
    const bool ax1 = Y - 2 * kHalf > 0, ax2 = X - 2 * kHalf > 0;
    double e[kPlen], cr;
    // axis 1 (y lines): accept flags, then the first kMaxE in draw order
    if (t == 0) s_n = 0;
    if (ax1)
        for (int k = t; k < kIters; k += kT) flag[k] = (unsigned char)psf_candidate(vol, Z, Y, X, 1, 0u, k, e, &cr);
    __syncthreads();
    if (t == 0 && ax1) {
        int n = 0;
        for (int k = 0; k < kIters && n < kMaxE; k++)
            if (flag[k]) pick[n++] = (short)k;
        s_n = n;
    }
    __syncthreads();
    const int n1 = s_n;
    // axis 2 (x lines) only while fewer than kMaxE: its draws follow axis 1's 2500 candidates
    const unsigned off2 = ax1 ? 3u * kIters : 0u;
    if (n1 < kMaxE && ax2) {
        for (int k = t; k < kIters; k += kT) flag[k] = (unsigned char)psf_candidate(vol, Z, Y, X, 2, off2, k, e, &cr);
        __syncthreads();
        if (t == 0) {
            int n = n1;
            for (int k = 0; k < kIters && n < kMaxE; k++)
                if (flag[k]) pick[n++] = (short)(kIters + k);
            s_n = n;
        }
    }
    __syncthreads();
    const int n = s_n;
    // rebuild the kept profiles
    for (int p = t; p < n; p += kT) {
        const int k = pick[p];
        const int ok = k < kIters ? psf_candidate(vol, Z, Y, X, 1, 0u, k, prof + p * kPlen, &cross[p])
                                  : psf_candidate(vol, Z, Y, X, 2, off2, k - kIters, prof + p * kPlen, &cross[p]);
        (void)ok;
    }
    __syncthreads();
    if (n < 30) {
        if (t == 0) { out->sigma = -1.0; out->nprof = n; }
        return;
    }
    // edge spread function on the super-sampled grid, profiles summed in draw order
    if (t < kGlen) {
        const double g = __dadd_rn(-(double)kHalf, __ddiv_rn(__dmul_rn((double)t, 2.0 * kHalf), (double)(kGlen - 1)));
        double acc = 0.0;
        for (int p = 0; p < n; p++) {
            const double xs = __dadd_rn(g, cross[p]);
            double v;
            if (xs <= 0) v = 0.0;
            else if (xs >= kPlen - 1) v = 1.0;
            else {
                const int i = (int)xs;
                const double f = __dsub_rn(xs, (double)i);
                const double* ep = prof + p * kPlen;
                v = __fma_rn(ep[i + 1], f, __dmul_rn(ep[i], __dsub_rn(1.0, f)));
            }
            acc = __dadd_rn(acc, v);
        }
        esf[t] = __dmul_rn(acc, __ddiv_rn(1.0, (double)n));
    }
    __syncthreads();
    if (t != 0) return;
    // line spread function and its second moment (pipeline.c:177-191)
    double lsf[kGlen], lsum = 0.0;
    for (int gi = 0; gi < kGlen; gi++) {
        double d;
        if (gi == 0) d = __dsub_rn(esf[1], esf[0]);
        else if (gi == kGlen - 1) d = __dsub_rn(esf[kGlen - 1], esf[kGlen - 2]);
        else d = __dmul_rn(0.5, __dsub_rn(esf[gi + 1], esf[gi - 1]));
        if (d < 0) d = 0;
        lsf[gi] = d;
        lsum = __dadd_rn(lsum, d);
    }
    double sig = -1.0;
    if (lsum > 0) {
        const double rl = __ddiv_rn(1.0, lsum);
        double mu = 0.0, var = 0.0;
        for (int gi = 0; gi < kGlen; gi++) {
            const double g = __dadd_rn(-(double)kHalf, __ddiv_rn(__dmul_rn((double)gi, 2.0 * kHalf), (double)(kGlen - 1)));
            lsf[gi] = __dmul_rn(lsf[gi], rl);
            mu = __fma_rn(g, lsf[gi], mu);
        }
        for (int gi = 0; gi < kGlen; gi++) {
            const double g = __dadd_rn(-(double)kHalf, __ddiv_rn(__dmul_rn((double)gi, 2.0 * kHalf), (double)(kGlen - 1)));
            const double dg = __dsub_rn(g, mu);
            var = __fma_rn(__dmul_rn(dg, dg), lsf[gi], var);
        }
        sig = __dsqrt_rn(var);
        if (!(sig > 0.3 && sig < 5.0)) sig = -1.0;
    }
    out->sigma = sig;
    out->nprof = n;
}

int enqueue_psf(const uint8_t* d_vol, int Z, int Y, int X, void* d_out, cudaStream_t st, const char* what) {
    const size_t smem = (size_t)kMaxE * kPlen * sizeof(double);
    cudaError_t e = fy_smem_optin(k_psf, smem);
    if (e != cudaSuccess) return fail_cuda(e, what);
    k_psf<<<1, kT, smem, st>>>(d_vol, Z, Y, X, (PsfOut*)d_out);
    if ((e = cudaGetLastError()) != cudaSuccess) return fail_cuda(e, what);
    fy::count_launch();
    return FY_OK;
}

}  // namespace

extern "C" int fy_gpu_measure_psf_sigma(const unsigned char* d_vol, int Z, int Y, int X, void* d_out, void* stream) {
    fy::enter();
    const char* what = "fy_gpu_measure_psf_sigma";
    if (!d_vol || !d_out) return fail(FY_EINVAL, "%s: null pointer", what);
    if (Z < 1 || Y < 1 || X < 1) return fail(FY_EINVAL, "%s: bad dims", what);
    int rc = fy::ensure_ctx();
    if (rc) return rc;
    return enqueue_psf(d_vol, Z, Y, X, d_out, (cudaStream_t)stream, what);
}

extern "C" double fy_measure_psf_sigma(const unsigned char* vol, int Z, int Y, int X, int* nprof) {
    fy::enter();
    const char* what = "fy_measure_psf_sigma";
    const double nan = NAN;
    if (!vol) { fail(FY_EINVAL, "%s: null pointer", what); return nan; }
    if (Z < 1 || Y < 1 || X < 1) { fail(FY_EINVAL, "%s: bad dims", what); return nan; }
    if (fy::ensure_ctx()) return nan;
    fy::ThreadCtx& c = ctx();
    cudaStream_t st = c.st;
    const size_t n = (size_t)Z * Y * X;
    fy::ws_acquire(st);
    cudaError_t e;
    if ((e = c.vin.ensure(n)) != cudaSuccess || (e = c.small.ensure(sizeof(PsfOut))) != cudaSuccess ||
        (e = c.pin.ensure(sizeof(PsfOut))) != cudaSuccess) {
        fail_cuda(e, what);
        return nan;
    }
    if ((e = cudaMemcpyAsync(c.vin.p, vol, n, cudaMemcpyHostToDevice, st)) != cudaSuccess) { fail_cuda(e, what); return nan; }
    if (enqueue_psf(c.vin.as<uint8_t>(), Z, Y, X, c.small.p, st, what)) return nan;
    if ((e = cudaMemcpyAsync(c.pin.p, c.small.p, sizeof(PsfOut), cudaMemcpyDeviceToHost, st)) != cudaSuccess) {
        fail_cuda(e, what);
        return nan;
    }
    fy::ws_release(st);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) { fail_cuda(e, what); return nan; }
    const PsfOut* o = (const PsfOut*)c.pin.p;
    if (nprof) *nprof = o->nprof;
    return o->sigma;
}
