// fy_noise.cu -- per-volume noise model fy_estimate_noise (noise.c:75-192) on the GPU.
//
//   1. Local stats, a z-sliding box pass (fy_zbox.cuh): box sums over (2r+1)^3 windows with
//      zero outside the volume and the FIXED divisor win^3 (noise.c:20-59, 92-101): mean m
//      and variance v = max(S2/wc - m^2, 0). Sums are direct
//      (2r+1)-tap float sums of (I - c) and (I - c)^2 with a per-tile shift c, and interior
//      voxels use v = S2'/wc - (S1'/wc)^2, which equals the reference's S2/wc - (S1/wc)^2
//      without its cancellation.
//   2. Exact order statistics on orderable 32-bit float keys: the 1st and 99th percentiles
//      of m (noise.c:104-108) through a sample-guided window, one pass over m and a radix
//      select of the window's candidates (falling back to radix passes over m when the
//      window misses), and, per intensity bin with >= 200 voxels, the flat_pct percentile of
//      v (noise.c:117-134) through the same scheme over mean and variance (falling back to
//      radix passes over v); each interpolated between order statistics k and k+1 exactly
//      as percentile() does (noise.c:66-73).
//   3. k_noise_fit: one thread, FP64: IRLS line fit var = g*I + b (noise.c:137-172) and
//      noise_ref = sqrt(max(g*ref + b, ..))*1.15 (noise.c:181-187), plus the guided eps
//      (3*noise_ref)^2 floored at 1e-8 (noise.c:197-202).
// The launch sequence is fixed (no host decisions), so a chain can keep it on one stream.
#include <cuda/std/tuple>
#include <vector>

#include "fy_internal.h"
#include "fysics_b200.h"
#include "fy_zbox.cuh"

namespace {

constexpr int NB = 24;                 // intensity bins, noise.c:111
constexpr int NT_MAX = 64;             // selection targets: 2 per bin + spare
// ctl->mode: 0 mean percentiles by radix passes, 1 bin percentiles by radix passes, 2
// variance fallback, 3 done; kModeWin0: the mean percentiles through the sample-guided
// window (section 2w), which falls back to mode 0 when the window misses.
constexpr int kModeWin0 = 4;
constexpr int kModeBinCand = 6;        // the bins' last digit runs on a candidate list (cc)
constexpr int kModeBinWin = 7;         // the bins' percentiles through the sample-guided window (2bw)
constexpr int kModeBinDone = 8;        // the window found them: the bins' radix passes stand aside

FY_D uint32_t fkey(float f) {
    const uint32_t u = __float_as_uint(f);
    return u ^ ((uint32_t)((int32_t)u >> 31) | 0x80000000u);   // negative: ~u, else u | sign
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
// Selection targets: target t selects the order statistic k_t (0-based) of the keys of
// group g_t. Bins: t = bin id. Whole volume: t = 0, 1 (1st/99th percentile) or t = 0
// (variance fallback). After the digit passes, prefix_t is the k-th key, eq_t the number of
// keys equal to it and rank_t its rank among them; the (k+1)-th key is the same key when
// rank_t + 1 < eq_t, else the smallest key greater than it (k_sel_next).
struct NoiseCtl {
    long long n;
    double flat_pct, ref_intensity;
    int ntarget, mode;                 // mode 0 means lo/hi, 1 bins, 2 variance fallback, 3 done
    long long tk[NT_MAX];              // requested rank k
    long long trank[NT_MAX];           // remaining rank inside the decided prefix
    long long tgroup_n[NT_MAX];        // group size
    unsigned long long teq[NT_MAX];    // keys equal to the selected key
    uint32_t tprefix[NT_MAX];
    uint32_t tnext[NT_MAX];            // min key > selected key (when needed)
    int tactive[NT_MAX];
    int tneed_next[NT_MAX];
    double lo, hi;
    double edge[NB + 1];
    float fedge[NB + 1];               // smallest float >= edge[k]: exact float membership test
    float fscale;                      // NB/(hi-lo) for the bin guess
    unsigned long long bcount[NB];
    double bfloor[NB];
    double out_g, out_b, out_noise_ref, out_ref_intensity;
    int out_used;
    float eps;                         // fy_guided_eps_for_noise(noise_ref), for a chained guided filter
    alignas(16) unsigned int hist[NT_MAX * 256];   // per-target histogram (bins: 24 x 256; whole: 2 x 2048)
    // Sample-guided window (section 2w): per target the window keys [wlo, whi] and the count
    // of keys below wlo.
    uint32_t wlo[2], whi[2];
    unsigned long long wbelow[2];
    unsigned long long ncand;          // candidates appended (may exceed the capacity)
    int wfail;                         // the window missed: the radix passes run instead
    // The bins' windows (section 2bw): per bin the variance keys [bwlo, bwhi] and the counts
    // of the bin's keys below, inside and above it.
    uint32_t bwlo[NB], bwhi[NB];
    unsigned long long bwc[NB * 3];
    unsigned int done_ctas;            // CTAs of the current digit pass that have flushed (0 between passes)
};

namespace {


// The block index and grid size along x of the CTA's volume, which every selection body uses
// in place of blockIdx.x / gridDim.x: k_one sets them from its launch, k_many from the step's
// table of CTAs per volume (a batch launch holds every volume's CTAs along x).
static __shared__ unsigned s_vbx, s_vgx;
FY_D unsigned vbx() { return s_vbx; }
FY_D unsigned vgx() { return s_vgx; }

// ---------------------------------------------------------------- 1. local stats
// z-sliding box pass (fy_zbox.cuh, ZB_NOISE): 4 B read + 8 B written per voxel.

// ---------------------------------------------------------------- 2. radix select
// Exact bin of a float mean: m >= edge[k] <=> m >= fedge[k] with fedge[k] the smallest float
// >= edge[k] (noise.c:118-122 in double), so membership needs only float compares.
FY_D int bin_of(float m, const float* __restrict__ fe, float lo_f, float scale) {
    if (!(m >= fe[0] && m < fe[NB])) return -1;
    int b = (int)((m - lo_f) * scale);
    b = b < 0 ? 0 : (b > NB - 1 ? NB - 1 : b);
    while (b > 0 && m < fe[b]) --b;
    while (b < NB - 1 && m >= fe[b + 1]) ++b;
    return b;
}

// bin_of with at most one step from the float guess (the guess is within one bin of the
// exact one unless the range [lo, hi] is degenerate; then the exact walk runs): the common
// path has no loop. lo_e, hi_e: fe[0], fe[NB].
FY_D int bin_fast(float m, const float* __restrict__ fe, float lo_e, float hi_e, float lo_f, float scale) {
    if (!(m >= lo_e && m < hi_e)) return -1;
    int b = (int)((m - lo_f) * scale);
    b = b < 0 ? 0 : (b > NB - 1 ? NB - 1 : b);
    b -= (int)(m < fe[b]);                      // m >= fe[0], so b stays >= 0
    b += (int)(m >= fe[b + 1]);                 // m < fe[NB], so b stays <= NB - 1
    if (m < fe[b] || m >= fe[b + 1]) b = bin_of(m, fe, lo_f, scale);
    return b;
}

// Histogram increments with thread-local run merging: a thread's consecutive equal codes
// are counted in a register and added with one shared atomic per run. Neighbouring voxels
// mostly share intensity bins and high digits, so concentrated passes make few atomics,
// and spread-out passes pay only bank conflicts; no warp collectives are needed.
struct RunAcc {
    int cur = -1;
    unsigned int cnt = 0;
    FY_D void add(unsigned int* h, int code) {
        if (code != cur) {
            if (cur >= 0) atomicAdd(&h[cur], cnt);
            cur = code;
            cnt = 0;
        }
        ++cnt;
    }
    FY_D void flush(unsigned int* h) {
        if (cur >= 0) atomicAdd(&h[cur], cnt);
        cur = -1;
        cnt = 0;
    }
};

constexpr int kWarpBuf = 256;
struct WarpCands {
    float* v;                          // this warp's kWarpBuf values in shared memory
    uint8_t* l;                        // and labels
    int cnt = 0;                       // warp-uniform fill
    FY_D void flush(float* __restrict__ cval, uint8_t* __restrict__ clab, unsigned long long* ncand, long long cap) {
        const unsigned full = 0xffffffffu;
        __syncwarp();
        if (cnt) {
            unsigned long long base = 0;
            if ((threadIdx.x & 31) == 0) base = atomicAdd(ncand, (unsigned long long)cnt);
            base = __shfl_sync(full, base, 0);
            for (int i = threadIdx.x & 31; i < cnt; i += 32)
                if ((long long)(base + i) < cap) { cval[base + i] = v[i]; clab[base + i] = l[i]; }
        }
        cnt = 0;
        __syncwarp();
    }
};

// Streaming passes read SU float4 (and uchar4 bin labels) per thread before using any, so
// enough bytes are in flight per SM to cover HBM latency. Full chunks of the grid-stride
// loop run without per-element range checks; the one partial chunk is checked.
constexpr int SU = 4;

// One digit pass (bits [shift, shift + DB)) for every active target whose prefix matches.
// MODE 0: keys of mean, targets 0 and 1 over all voxels; MODE 1: keys of var, target = bin;
// MODE 2: keys of var, target 0 over all voxels. A key matches at most one distinct prefix,
// so in modes 0/2 targets whose prefixes are equal share one shared-memory histogram
// (group) and every voxel makes at most one increment; the flush copies a group's counts
// to each of its targets. Inactive targets and bin label 255 carry the prefix 0xffffffff,
// which no key's high part (< 2^(32 - shift - DB)) can equal.
// LABEL (the first variance pass only): the bin of each voxel is computed from its mean here
// and its u8 label written for the later passes, so no separate labelling pass runs.
// COMPACT (a MODE 1 digit pass): each voxel whose key matches its bin target's prefix is also
// appended, with its bin, to the candidate list (cval, clab; counter ctl->ncand): every key of
// the prefixes that the following digits narrow is then in the list.
// scan >= 0: the CTA that flushes last (a ticket on ctl->done_ctas) then does every active
// target's bookkeeping (warp_scan_target; scan 1: after the last digit), so no separate scan
// launch follows the pass.
constexpr int kCompactBuf = 1152;        // per warp: one step's worst case (32 x 4*SU) + slack

// The bookkeeping after a digit pass for target t, by one warp: the bucket that holds the
// target's rank (a warp scan of the lanes' bucket sums), the prefix extended by it, the keys
// equal to the selected key and, after the last digit, the next non-empty bucket (the
// smallest key above the selected one within the prefix; k_sel_next scans only when there is
// none). The histogram is read through L2 (other CTAs' atomics) and cleared.
// With at most 8 buckets per lane (8-bit digits) the lane's buckets stay in registers: one
// round of loads (with the target's rank and prefix) instead of one per reading.
template <int DB>
FY_D void warp_scan_target(NoiseCtl* ctl, int t, bool last) {
    constexpr int nbk = 1 << DB, per = nbk / 32;
    constexpr bool REG = per <= 8;
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    unsigned int* h = ctl->hist + (size_t)t * nbk;
    const int b0 = lane * per;
    const long long r = ctl->trank[t];
    const uint32_t pre = ctl->tprefix[t];
    unsigned int hv[REG ? per : 1];
    unsigned long long mine = 0;
    if (REG) {
#pragma unroll
        for (int i = 0; i < (REG ? per : 1); ++i) hv[i] = __ldcg(h + b0 + i);
#pragma unroll
        for (int i = 0; i < (REG ? per : 1); ++i) mine += hv[i];
    } else {
        for (int b = b0; b < b0 + per; ++b) mine += __ldcg(h + b);
    }
    unsigned long long incl = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(full, incl, o);
        if (lane >= o) incl += y;
    }
    const unsigned long long before = incl - mine;
    unsigned int sel = (unsigned)nbk;
    if ((unsigned long long)r >= before && (unsigned long long)r < incl) {
        unsigned long long acc = before;
        unsigned int hsel = 0;
        if (REG) {
#pragma unroll
            for (int i = 0; i < (REG ? per : 1); ++i) {
                if (sel == (unsigned)nbk && acc + hv[i] > (unsigned long long)r) { sel = (unsigned)(b0 + i); hsel = hv[i]; }
                else if (sel == (unsigned)nbk) acc += hv[i];
            }
        } else {
            for (int b = b0; b < b0 + per; ++b) {
                const unsigned int hb = __ldcg(h + b);
                if (acc + hb > (unsigned long long)r) { sel = (unsigned)b; hsel = hb; break; }
                acc += hb;
            }
        }
        if (sel != (unsigned)nbk) {
            ctl->trank[t] = r - (long long)acc;
            ctl->tprefix[t] = (pre << DB) | sel;
            if (last) ctl->teq[t] = hsel;
        }
    }
    sel = __reduce_min_sync(full, sel);
    unsigned int nextb = 0xffffffffu;
    if (last) {
        if (REG) {
#pragma unroll
            for (int i = (REG ? per : 1) - 1; i >= 0; --i)
                if (b0 + i > (int)sel && hv[i]) nextb = (unsigned)(b0 + i);
        } else {
            for (int b = b0 > (int)sel + 1 ? b0 : (int)sel + 1; b < b0 + per; ++b)
                if (__ldcg(h + b)) { nextb = (unsigned)b; break; }
        }
        nextb = __reduce_min_sync(full, nextb);
    }
    __syncwarp();
    for (int b = b0; b < b0 + per; ++b) h[b] = 0;
    __syncwarp();
    if (last && lane == 0) {
        ctl->tneed_next[t] = (ctl->trank[t] + 1 >= (long long)ctl->teq[t]) && (ctl->tk[t] + 1 < ctl->tgroup_n[t]);
        ctl->tnext[t] = nextb != 0xffffffffu ? ((ctl->tprefix[t] >> DB) << DB) | nextb : 0xffffffffu;
    }
}
template <int DB, int MODE, bool LABEL = false, bool COMPACT = false>
FY_D void k_sel_hist(const float* __restrict__ mean, const float* __restrict__ var,
                                                  uint8_t* __restrict__ bin, NoiseCtl* __restrict__ ctl,
                                                  int shift, float* __restrict__ cval = nullptr,
                                                  uint8_t* __restrict__ clab = nullptr, long long cap = 0,
                                                  int scan = -1) {
    fy_pdl_wait();
    extern __shared__ unsigned int h[];
    __shared__ uint32_t sp[256];
    __shared__ float fe[NB + 1];
    if (ctl->mode != MODE) return;
    if (LABEL && threadIdx.x <= NB) fe[threadIdx.x] = ctl->fedge[threadIdx.x];
    const float lo_f = LABEL ? ctl->fedge[0] : 0.f, fscale = LABEL ? ctl->fscale : 0.f;
    auto lab = [&](float m) -> unsigned { const int b = bin_of(m, fe, lo_f, fscale); return b < 0 ? 255u : (unsigned)b; };
    constexpr int NBK = 1 << DB;
    const int nt = ctl->ntarget;
    if (MODE == 1)
        for (int i = threadIdx.x; i < 256; i += blockDim.x) sp[i] = i < nt && ctl->tactive[i] ? ctl->tprefix[i] : 0xffffffffu;
    // modes 0/2: at most two targets; group of target 1 is 0 when it shares target 0's prefix
    uint32_t p0 = 0xffffffffu, p1 = 0xffffffffu;
    int g1 = 1;
    if (MODE != 1) {
        p0 = ctl->tactive[0] ? ctl->tprefix[0] : 0xffffffffu;
        if (nt > 1 && ctl->tactive[1]) {
            p1 = ctl->tprefix[1];
            if (p1 == p0) { g1 = 0; p1 = 0xfffffffeu; }   // never matches: target 1 reads group 0
        }
    }
    const int ngroup = MODE == 1 ? nt : 2;
    for (int i = threadIdx.x; i < ngroup * NBK; i += blockDim.x) h[i] = 0;
    __syncthreads();
    const int top = shift + DB;
    const long long n = ctl->n, n4 = (n + 3) / 4, n4f = n / 4;
    const float* src = MODE == 0 ? mean : var;
    const int step = blockDim.x;
    const long long chunk = (long long)SU * step;
    RunAcc acc;
    auto code_of = [&](float v, int g) -> int {
        const uint32_t key = fkey(v);
        const uint32_t hb = top >= 32 ? 0u : (key >> top);
        const int dig = (key >> shift) & (NBK - 1);
        if (MODE == 1) return sp[g] == hb ? g * NBK + dig : -1;
        return hb == p0 ? dig : (hb == p1 ? NBK + dig : -1);
    };
    WarpCands wc;
    if (COMPACT) {
        float* bv = reinterpret_cast<float*>(h + ngroup * NBK);
        wc.v = bv + (threadIdx.x >> 5) * kCompactBuf;
        wc.l = reinterpret_cast<uint8_t*>(bv + (blockDim.x >> 5) * kCompactBuf) + (threadIdx.x >> 5) * kCompactBuf;
    }
    long long base = (long long)vbx() * chunk;
    const long long stride = (long long)vgx() * chunk;        // read once: the loop body has syncs
    for (; base + chunk <= n4f; base += stride) {
        float4 x[SU];
        uchar4 bb[SU];
        float4 mm[LABEL ? SU : 1];
#pragma unroll
        for (int u = 0; u < SU; ++u) {
            const long long q = base + threadIdx.x + (long long)u * step;
            x[u] = __ldg(reinterpret_cast<const float4*>(src) + q);
            if (LABEL) mm[u] = __ldg(reinterpret_cast<const float4*>(mean) + q);
            else if (MODE == 1) bb[u] = __ldg(reinterpret_cast<const uchar4*>(bin) + q);
        }
        if (LABEL) {
#pragma unroll
            for (int u = 0; u < SU; ++u) {
                bb[u] = make_uchar4(lab(mm[u].x), lab(mm[u].y), lab(mm[u].z), lab(mm[u].w));
                reinterpret_cast<uchar4*>(bin)[base + threadIdx.x + (long long)u * step] = bb[u];
            }
        }
        if (!COMPACT) {
#pragma unroll
            for (int u = 0; u < SU; ++u) {
                acc.add(h, code_of(x[u].x, MODE == 1 ? bb[u].x : 0));
                acc.add(h, code_of(x[u].y, MODE == 1 ? bb[u].y : 0));
                acc.add(h, code_of(x[u].z, MODE == 1 ? bb[u].z : 0));
                acc.add(h, code_of(x[u].w, MODE == 1 ? bb[u].w : 0));
            }
        } else {
            float xv[4 * SU];
            unsigned xl[4 * SU];
            unsigned hit = 0;
#pragma unroll
            for (int u = 0; u < SU; ++u) {
                xv[4 * u] = x[u].x; xv[4 * u + 1] = x[u].y; xv[4 * u + 2] = x[u].z; xv[4 * u + 3] = x[u].w;
                xl[4 * u] = bb[u].x; xl[4 * u + 1] = bb[u].y; xl[4 * u + 2] = bb[u].z; xl[4 * u + 3] = bb[u].w;
            }
#pragma unroll
            for (int q = 0; q < 4 * SU; ++q) {
                const int code = code_of(xv[q], (int)xl[q]);
                acc.add(h, code);
                hit |= (unsigned)(code >= 0) << q;
            }
            // place this step's hits in the warp's buffer (one scan), append it when nearly full
            const unsigned full = 0xffffffffu;
            const int lane = threadIdx.x & 31, c = __popc(hit);
            int incl = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(full, incl, o);
                if (lane >= o) incl += y;
            }
            const int tot = __shfl_sync(full, incl, 31);
            if (tot) {
                if (wc.cnt + tot > kCompactBuf) wc.flush(cval, clab, &ctl->ncand, cap);
                int pos = wc.cnt + incl - c;
#pragma unroll
                for (int q = 0; q < 4 * SU; ++q)
                    if ((hit >> q) & 1u) { wc.v[pos] = xv[q]; wc.l[pos] = (uint8_t)xl[q]; ++pos; }
                wc.cnt += tot;
                __syncwarp();
            }
        }
    }
    if (base < n4) {                                     // the grid's partial chunk
        for (int u = 0; u < SU; ++u)
            for (int j = 0; j < 4; ++j) {
                const long long i = 4 * (base + threadIdx.x + (long long)u * step) + j;
                if (i >= n) continue;
                int g = 0;
                if (LABEL) { g = (int)lab(__ldg(mean + i)); bin[i] = (uint8_t)g; }
                else if (MODE == 1) g = (int)__ldg(bin + i);
                const float v = __ldg(src + i);
                const int code = code_of(v, g);
                acc.add(h, code);
                if (COMPACT && code >= 0) {
                    const unsigned long long pos = atomicAdd(&ctl->ncand, 1ull);
                    if ((long long)pos < cap) { cval[pos] = v; clab[pos] = (uint8_t)g; }
                }
            }
    }
    if (COMPACT) wc.flush(cval, clab, &ctl->ncand, cap);
    acc.flush(h);
    __syncthreads();
    if (MODE == 1) {
        for (int i = threadIdx.x; i < nt * NBK; i += blockDim.x)
            if (h[i]) atomicAdd(&ctl->hist[i], h[i]);
    } else {
        for (int i = threadIdx.x; i < nt * NBK; i += blockDim.x) {
            const int t = i / NBK, grp = t == 0 ? 0 : g1;
            const unsigned int cnt = h[grp * NBK + (i - t * NBK)];
            if (cnt) atomicAdd(&ctl->hist[i], cnt);
        }
    }
    if (scan < 0) return;
    __shared__ int s_last;
    __threadfence();                                     // this CTA's counts before its ticket
    __syncthreads();
    if (threadIdx.x == 0) s_last = atomicAdd(&ctl->done_ctas, 1u) == vgx() - 1;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    for (int t = threadIdx.x >> 5; t < nt; t += blockDim.x >> 5)
        if (ctl->tactive[t]) warp_scan_target<DB>(ctl, t, scan == 1);
    if (threadIdx.x == 0) ctl->done_ctas = 0;
}

// After a digit pass: target t (one block) finds the bucket holding its rank by a block
// scan of the histogram, extends its prefix, records how many keys share the final key.
// After the last digit, the next non-empty bucket of that digit is the smallest key above
// the selected one within the prefix; k_sel_next scans only when there is none.
FY_D void k_sel_scan(NoiseCtl* __restrict__ ctl, int db, int want_mode, int last) {
    fy_pdl_wait();
    __shared__ unsigned long long part[256];
    __shared__ int s_sel;
    __shared__ unsigned int s_nextb;
    if (ctl->mode != want_mode) return;
    const int t = vbx();
    if (t >= ctl->ntarget || !ctl->tactive[t]) return;
    const int nbk = 1 << db, per = nbk / 256 > 0 ? nbk / 256 : 1;
    unsigned int* h = ctl->hist + (size_t)t * nbk;
    const int b0 = threadIdx.x * per;
    unsigned long long mine = 0;
    for (int b = b0; b < b0 + per && b < nbk; ++b) mine += h[b];
    part[threadIdx.x] = mine;
    if (threadIdx.x == 0) { s_sel = nbk; s_nextb = 0xffffffffu; }
    __syncthreads();
    for (int off = 1; off < 256; off <<= 1) {                // inclusive scan
        const unsigned long long add = threadIdx.x >= off ? part[threadIdx.x - off] : 0ull;
        __syncthreads();
        part[threadIdx.x] += add;
        __syncthreads();
    }
    const long long r = ctl->trank[t];
    const unsigned long long before = threadIdx.x ? part[threadIdx.x - 1] : 0ull;
    if ((unsigned long long)r >= before && (unsigned long long)r < part[threadIdx.x]) {
        unsigned long long acc = before;
        for (int b = b0; b < b0 + per && b < nbk; ++b) {
            if (acc + h[b] > (unsigned long long)r) {
                ctl->trank[t] = r - (long long)acc;
                ctl->tprefix[t] = (ctl->tprefix[t] << db) | (uint32_t)b;
                if (last) ctl->teq[t] = h[b];
                s_sel = b;
                break;
            }
            acc += h[b];
        }
    }
    __syncthreads();
    if (last) {
        const int sel = s_sel;
        for (int b = b0 > sel + 1 ? b0 : sel + 1; b < b0 + per && b < nbk; ++b)
            if (h[b]) { atomicMin(&s_nextb, (unsigned)b); break; }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nbk; i += blockDim.x) h[i] = 0;
    if (last && threadIdx.x == 0) {
        ctl->tneed_next[t] = (ctl->trank[t] + 1 >= (long long)ctl->teq[t]) && (ctl->tk[t] + 1 < ctl->tgroup_n[t]);
        ctl->tnext[t] = s_nextb != 0xffffffffu ? ((ctl->tprefix[t] >> db) << db) | s_nextb : 0xffffffffu;
    }
}

// Smallest key greater than the selected key, for targets whose k+1 lies past it and whose
// last digit histogram held no larger key (k_sel_scan resolves every other target).
FY_D void k_sel_next(const float* __restrict__ mean, const float* __restrict__ var,
                                                  const uint8_t* __restrict__ bin, NoiseCtl* __restrict__ ctl,
                                                  int want_mode) {
    fy_pdl_wait();
    __shared__ uint32_t sp[NT_MAX];
    __shared__ int sn[NT_MAX];
    __shared__ unsigned int smin[NT_MAX];
    __shared__ int s_any;
    if (ctl->mode != want_mode) return;
    const int nt = ctl->ntarget;
    if (threadIdx.x == 0) s_any = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < nt; i += blockDim.x) {
        sp[i] = ctl->tprefix[i];
        sn[i] = ctl->tactive[i] && ctl->tneed_next[i] && ctl->tnext[i] == 0xffffffffu;
        smin[i] = 0xffffffffu;
        if (sn[i]) s_any = 1;
    }
    __syncthreads();
    if (!s_any) return;
    const long long n = ctl->n;
    const float* src = want_mode == 0 ? mean : var;
    auto visit = [&](float v, int g) {
        const uint32_t key = fkey(v);
        if (want_mode == 1) {            // one target per voxel: its bin
            if (g < NB && g < nt && sn[g] && key > sp[g] && key < smin[g]) atomicMin(&smin[g], key);
        } else {
            for (int t = 0; t < nt; ++t)
                if (sn[t] && key > sp[t] && key < smin[t]) atomicMin(&smin[t], key);
        }
    };
    // SU float4 (and uchar4 labels) per thread before any is used, as the streaming passes
    const long long n4 = (n + 3) / 4, n4f = n / 4, chunk = (long long)SU * blockDim.x;
    long long base = (long long)vbx() * chunk;
    const long long stride = (long long)vgx() * chunk;        // read once: the loop body has syncs
    for (; base + chunk <= n4f; base += stride) {
        float4 x[SU];
        uchar4 bb[SU];
#pragma unroll
        for (int u = 0; u < SU; ++u) {
            const long long q = base + threadIdx.x + (long long)u * blockDim.x;
            x[u] = __ldg(reinterpret_cast<const float4*>(src) + q);
            bb[u] = want_mode == 1 ? __ldg(reinterpret_cast<const uchar4*>(bin) + q) : make_uchar4(0, 0, 0, 0);
        }
#pragma unroll
        for (int u = 0; u < SU; ++u) {
            visit(x[u].x, bb[u].x);
            visit(x[u].y, bb[u].y);
            visit(x[u].z, bb[u].z);
            visit(x[u].w, bb[u].w);
        }
    }
    if (base < n4)                                       // the grid's partial chunk
        for (int u = 0; u < SU; ++u)
            for (int j = 0; j < 4; ++j) {
                const long long i = 4 * (base + threadIdx.x + (long long)u * blockDim.x) + j;
                if (i < n) visit(__ldg(src + i), want_mode == 1 ? (int)__ldg(bin + i) : 0);
            }
    __syncthreads();
    for (int i = threadIdx.x; i < nt; i += blockDim.x)
        if (sn[i] && smin[i] != 0xffffffffu) atomicMin(&ctl->tnext[i], smin[i]);
}

// value of order statistic k+1 of target t
FY_D double next_value(const NoiseCtl* ctl, int t) {
    return ctl->tneed_next[t] ? (double)funkey(ctl->tnext[t]) : (double)funkey(ctl->tprefix[t]);
}
// percentile() interpolation (noise.c:69-72)
FY_D double interp(const NoiseCtl* ctl, int t, double f, bool has_next) {
    const double v0 = (double)funkey(ctl->tprefix[t]);
    if (!has_next) return v0;
    return v0 * (1 - f) + next_value(ctl, t) * f;
}

FY_D void target_init(NoiseCtl* ctl, int t, long long k, long long group_n, bool on) {
    ctl->tk[t] = k;
    ctl->trank[t] = k;
    ctl->tgroup_n[t] = group_n;
    ctl->tprefix[t] = 0;
    ctl->teq[t] = 0;
    ctl->tactive[t] = on;
    ctl->tneed_next[t] = 0;
    ctl->tnext[t] = 0xffffffffu;
}

// One block of 256 threads: thread t < NT_MAX initialises target t; all clear both blocks'
// histograms.
FY_D void k_noise_setup(NoiseCtl* ctl, NoiseCtl* cc, long long n, double flat_pct, double ref_intensity) {
    fy_pdl_wait();
    const int t = threadIdx.x;
    static_assert(sizeof(ctl->hist) % 16 == 0 && offsetof(NoiseCtl, hist) % 16 == 0, "uint4 clears");
    for (int i = t; i < (int)(sizeof(ctl->hist) / 16); i += blockDim.x) {
        reinterpret_cast<uint4*>(ctl->hist)[i] = make_uint4(0u, 0u, 0u, 0u);
        reinterpret_cast<uint4*>(cc->hist)[i] = make_uint4(0u, 0u, 0u, 0u);
    }
    if (t >= NT_MAX) return;
    const double i1 = 1.0 / 100.0 * (double)(n - 1), i99 = 99.0 / 100.0 * (double)(n - 1);
    if (t == 0) target_init(ctl, 0, (long long)i1, n, true);           // 1st percentile of the means
    else if (t == 1) target_init(ctl, 1, (long long)i99, n, true);     // 99th
    else target_init(ctl, t, 0, 0, false);
    if (t < NB) ctl->bcount[t] = 0;
    if (t == 0) {
        ctl->done_ctas = 0;
        cc->done_ctas = 0;
        ctl->n = n;
        ctl->flat_pct = flat_pct;
        ctl->ref_intensity = ref_intensity;
        ctl->mode = kModeWin0;             // the radix passes run only if the windows fail
        ctl->ntarget = 2;
    }
}

// lo/hi from the selected means; bin edges (noise.c:106-119). One block of NT_MAX threads.
FY_D void k_noise_bins_setup(NoiseCtl* ctl) {
    fy_pdl_wait();
    __shared__ double s_lo, s_hi;
    const int t = threadIdx.x;
    if (t == 0) {
        const long long n = ctl->n;
        const double i1 = 1.0 / 100.0 * (double)(n - 1), i99 = 99.0 / 100.0 * (double)(n - 1);
        const long long k1 = (long long)i1, k99 = (long long)i99;
        const double lo = interp(ctl, 0, i1 - (double)k1, k1 + 1 < n);
        double hi = interp(ctl, 1, i99 - (double)k99, k99 + 1 < n);
        if (hi <= lo) hi = lo + 1e-6;                   // noise.c:109
        s_lo = lo;
        s_hi = hi;
    }
    __syncthreads();                                    // targets 0/1 read before they are reset
    const double lo = s_lo, hi = s_hi;
    if (t <= NB) {
        const double e = lo + (hi - lo) * t / NB;      // noise.c:118-119
        ctl->edge[t] = e;
        float f = (float)e;
        if ((double)f < e) f = nextafterf(f, INFINITY);
        ctl->fedge[t] = f;
    }
    // the radix passes' first variance digit: every bin active with the empty prefix (its
    // histogram gives the bin counts; k_bin_targets then sets the ranks)
    target_init(ctl, t, 0, 0, t < NB);
    for (int i = t; i < NB * 3; i += blockDim.x) ctl->bwc[i] = 0;
    if (t == 0) {
        ctl->lo = lo;
        ctl->hi = hi;
        ctl->fscale = (float)(NB / (hi - lo));
        ctl->ntarget = NB;
        // the bins' window runs first (section 2bw); it hands over to the radix passes
        // (mode 1) when it misses
        ctl->ncand = 0;
        ctl->wfail = 0;
        ctl->mode = kModeBinWin;
    }
}

// After the first variance digit pass (one block per bin): the bin's count is the sum of its
// histogram; targets of the flat_pct percentile for bins with >= 200 voxels (noise.c:123).
// Bins below that drop out and their histogram is cleared.
FY_D void k_bin_targets(NoiseCtl* ctl) {
    fy_pdl_wait();
    __shared__ unsigned long long part[256];
    if (ctl->mode != 1) return;
    const int b = vbx();
    unsigned int* h = ctl->hist + (size_t)b * 256;
    part[threadIdx.x] = h[threadIdx.x];
    __syncthreads();
    for (int off = 128; off > 0; off >>= 1) {
        if (threadIdx.x < off) part[threadIdx.x] += part[threadIdx.x + off];
        __syncthreads();
    }
    const long long c = (long long)part[0];
    const bool on = c >= 200;
    if (!on) h[threadIdx.x] = 0;
    if (threadIdx.x == 0) {
        ctl->bcount[b] = (unsigned long long)c;
        const double idx = ctl->flat_pct / 100.0 * (double)(c - 1);
        target_init(ctl, b, on ? (long long)idx : 0, c, on);
    }
}

// ---------------------------------------------------------------- 2w. sample-guided window
// The 1st/99th percentiles of the means by radix selection read the mean field once per
// digit (3 passes). Here they read it once:
//   sample   m <= kSampleMax means at positions (A*i + B) mod n, a bijection of [0, n) when
//            gcd(A, n) = 1, spread evenly over the volume.
//   window   per target, the sample's order statistics kWinSigmas binomial standard
//            deviations either side of the target's expected sample rank give a key window
//            [wlo, whi] that holds the target's order statistics k and k+1 with
//            overwhelming probability (one CTA per target and window end, radix select in
//            shared memory to the 24-bit key bucket, widened to its ends).
//   count    one pass over the means counts, per target, the keys below wlo and appends the
//            keys inside [wlo, whi] with their target label to a candidate list.
//   select   the radix passes of mode 1 over the candidates with a second control block,
//            targets = labels: the first digit pass's per-target sums are the inside counts,
//            so the target ranks r = k - below are set after it (as the bin counts are in
//            the bin selection). A rank outside [0, inside) -- k or k+1 not in the window --
//            or a candidate list over its capacity sends the selection to the radix passes
//            over the whole field (mode 0), which are exact in every case.
//   finish   the keys of k and k+1 go into the main block in the form the fit reads.
// The result is the same exact order statistics as the radix path: only which pass finds
// them changes. The per-bin variance percentiles use the same scheme (section 2bw).
constexpr int kSampleMax = 16384;
constexpr int kBoundThreads = 512;
constexpr double kWinSigmas = 5.0;
// Test hook: bit 0 forces the mean percentiles, bit 1 the bins, to the radix passes over the
// whole field; noise_window_used records (bits 0/1) which windows produced their result.
static __device__ int noise_force_radix;
static __device__ int noise_window_used;

// Block radix select over keys in shared memory: the rank-th smallest (0-based) of keys[0, c),
// c <= kSampleMax, by kBoundThreads threads. npass 8-bit digit passes from the top: with
// npass < 4 the result is the selected key's top 8*npass bits with the rest zero (the bucket
// that holds it, enough for a window bound). Each warp counts into a
// private 256-bin histogram (wh, [warps][256]); the lanes of a warp that hold the same digit
// are merged with __match_any_sync, so one shared atomic counts them all (the high digits of
// a sample are nearly all equal). Then one thread per digit sums the warps' counts and a
// warp-shuffle scan over the 256 digit totals finds the bucket of the rank.
FY_D uint32_t block_select(const uint32_t* keys, int c, long long rank, unsigned int* wh,
                           unsigned long long* part, uint32_t* s_sel, int npass = 4) {
    constexpr int NTB = kBoundThreads, NW = NTB / 32;
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const unsigned full = 0xffffffffu;
    uint32_t prefix = 0, pmask = 0;
    unsigned int* mine_h = wh + w * 256;
    for (int sh = 24; sh >= 32 - 8 * npass; sh -= 8) {
        for (int i = t; i < NW * 256; i += NTB) wh[i] = 0;
        __syncthreads();
        for (int i0 = 0; i0 < c; i0 += NTB) {             // warp-uniform trip count
            const int i = i0 + t;
            const uint32_t k = i < c ? keys[i] : 0u;
            const bool ok = i < c && (k & pmask) == prefix;
            const unsigned act = __ballot_sync(full, ok);
            if (ok) {
                const unsigned d = (k >> sh) & 255u;
                const unsigned same = __match_any_sync(act, d);
                if (lane == __ffs(same) - 1) atomicAdd(&mine_h[d], (unsigned)__popc(same));
            }
        }
        __syncthreads();
        unsigned long long tot = 0;                     // digit t's count over the warps
        if (t < 256)
            for (int ww = 0; ww < NW; ++ww) tot += wh[ww * 256 + t];
        // inclusive scan of the 256 digit totals: within warps by shuffles, then warp sums
        unsigned long long incl = tot;
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(full, incl, o);
            if (lane >= o) incl += y;
        }
        if (t < 256 && lane == 31) part[w] = incl;
        __syncthreads();
        if (t < 256) {
            unsigned long long off = 0;
            for (int ww = 0; ww < w; ++ww) off += part[ww];
            const unsigned long long hi = off + incl, lo = hi - tot;
            if ((unsigned long long)rank >= lo && (unsigned long long)rank < hi) {
                s_sel[0] = (uint32_t)t;
                s_sel[1] = (uint32_t)(rank - (long long)lo);
            }
        }
        __syncthreads();
        prefix |= s_sel[0] << sh;
        pmask |= 255u << sh;
        rank = s_sel[1];
        __syncthreads();
    }
    return prefix;
}

FY_D void k_win_sample(const float* __restrict__ mean, const NoiseCtl* __restrict__ ctl,
                                                    float* __restrict__ sm, long long m, unsigned long long A,
                                                    unsigned long long B) {
    fy_pdl_wait();
    if (ctl->mode != kModeWin0) return;
    const unsigned long long n = (unsigned long long)ctl->n;
    for (long long i = (long long)vbx() * blockDim.x + threadIdx.x; i < m; i += (long long)vgx() * blockDim.x)
        sm[i] = __ldg(mean + (A * (unsigned long long)i + B) % n);
}

// One CTA (kBoundThreads threads) per target (block x 0/1: 1st/99th percentile) and window
// end (blockIdx.y 0: wlo, 1: whi). Dynamic shared memory: kSampleMax keys, then the warps'
// digit histograms (kBoundThreads/32 x 256 counters).
FY_D void k_win_bounds(const float* __restrict__ sm,
                                                              NoiseCtl* __restrict__ ctl, long long m) {
    fy_pdl_wait();
    extern __shared__ uint32_t wkeys[];
    unsigned int* wh = wkeys + kSampleMax;
    __shared__ unsigned long long part[kBoundThreads];
    __shared__ uint32_t s_sel[2];
    if (ctl->mode != kModeWin0) return;
    const int t = vbx();
    const int c = (int)(m < kSampleMax ? m : kSampleMax);
    for (int i0 = threadIdx.x; i0 < c; i0 += 8 * blockDim.x) {   // eight loads in flight per thread
        float v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int i = i0 + u * blockDim.x;
            v[u] = i < c ? sm[i] : 0.f;
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int i = i0 + u * blockDim.x;
            if (i < c) wkeys[i] = fkey(v[u]);
        }
    }
    __syncthreads();
    const double q = (double)ctl->tk[t] / (double)(ctl->n > 1 ? ctl->n - 1 : 1);   // the target's quantile
    const bool upper = blockIdx.y == 1;
    uint32_t w = upper ? 0xffffffffu : 0u;
    if (c >= 64) {                                      // fewer samples: the whole key range
        const double qc = q < 1.0 / c ? 1.0 / c : (q > 1.0 - 1.0 / c ? 1.0 - 1.0 / c : q);
        const long long ks = (long long)(q * (double)(c - 1));
        const long long d = (long long)ceil(kWinSigmas * sqrt((double)c * qc * (1.0 - qc))) + 4;
        // three digits: the order statistic's 24-bit key bucket, widened to its ends
        if (!upper && ks - d >= 0) w = block_select(wkeys, c, ks - d, wh, part, s_sel, 3);
        if (upper && ks + d + 1 < c) w = block_select(wkeys, c, ks + d + 1, wh, part, s_sel, 3) | 0xffu;
    }
    if (threadIdx.x == 0) {
        if (upper) {
            ctl->whi[t] = w;
        } else {
            ctl->wlo[t] = w;
            ctl->wbelow[t] = 0;
            if (t == 0) ctl->ncand = 0;
        }
    }
}

// Candidate appends go through a per-warp shared buffer; a full buffer is copied out with one
// global atomic for its whole run, so the list's counter sees one atomic per ~kWarpBuf
// candidates instead of one per warp and element.

// The counting pass: mean keys against the windows of targets 0 and 1. The counts below each
// window stay in registers until one warp reduction at the end; the keys inside a window go
// to the candidate list (order is irrelevant to the selection). Per step a thread marks its
// 4*SU keys' window hits in two bit masks; one warp scan of the hit counts places them in the
// warp's shared-memory buffer, which is appended to the list (one atomic) when nearly full.
constexpr int kCountBuf = 1152;          // >= one step's worst case (32 lanes x 4*SU keys x 2); 45 KB static smem
FY_D void k_win_count(const float* __restrict__ mean, NoiseCtl* __restrict__ ctl,
                                                   float* __restrict__ cval, uint8_t* __restrict__ clab,
                                                   long long cap) {
    fy_pdl_wait();
    static_assert(32 * 4 * SU * 2 <= kCountBuf, "one step must fit the warp buffer");
    __shared__ float bufv[256 / 32][kCountBuf];
    __shared__ uint8_t bufl[256 / 32][kCountBuf];
    if (ctl->mode != kModeWin0) return;
    const unsigned full = 0xffffffffu;
    const int t = threadIdx.x, lane = t & 31;
    WarpCands wc;
    wc.v = bufv[t >> 5];
    wc.l = bufl[t >> 5];
    const long long n = ctl->n, n4 = (n + 3) / 4, n4f = n / 4;
    const uint32_t lo0 = ctl->wlo[0], hi0 = ctl->whi[0], lo1 = ctl->wlo[1], hi1 = ctl->whi[1];
    unsigned int bel0 = 0, bel1 = 0;
    const long long chunk = (long long)SU * 256;
    long long base = (long long)vbx() * chunk;
    const long long stride = (long long)vgx() * chunk;        // read once: the loop body has syncs
    // the next chunk's keys are loaded before this chunk's are used, so a warp keeps its loads
    // in flight while it classifies
    float4 xn[SU];
    if (base + chunk <= n4f) {
#pragma unroll
        for (int u = 0; u < SU; ++u) xn[u] = __ldg(reinterpret_cast<const float4*>(mean) + base + t + (long long)u * 256);
    }
    for (; base + chunk <= n4f; base += stride) {
        float4 x[SU];
#pragma unroll
        for (int u = 0; u < SU; ++u) x[u] = xn[u];
        if (base + stride + chunk <= n4f) {
#pragma unroll
            for (int u = 0; u < SU; ++u)
                xn[u] = __ldg(reinterpret_cast<const float4*>(mean) + base + stride + t + (long long)u * 256);
        }
        float mv[4 * SU];
        unsigned m0 = 0, m1 = 0;
#pragma unroll
        for (int u = 0; u < SU; ++u) {
            mv[4 * u] = x[u].x; mv[4 * u + 1] = x[u].y; mv[4 * u + 2] = x[u].z; mv[4 * u + 3] = x[u].w;
        }
#pragma unroll
        for (int q = 0; q < 4 * SU; ++q) {
            const uint32_t k = fkey(mv[q]);
            bel0 += k < lo0;
            bel1 += k < lo1;
            m0 |= (unsigned)(k >= lo0 && k <= hi0) << q;
            m1 |= (unsigned)(k >= lo1 && k <= hi1) << q;
        }
        const int c = __popc(m0) + __popc(m1);
        int incl = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(full, incl, o);
            if (lane >= o) incl += y;
        }
        const int tot = __shfl_sync(full, incl, 31);
        if (tot == 0) continue;
        if (wc.cnt + tot > kCountBuf) wc.flush(cval, clab, &ctl->ncand, cap);     // warp-uniform
        int pos = wc.cnt + incl - c;
#pragma unroll
        for (int q = 0; q < 4 * SU; ++q)          // unrolled, so mv stays in registers
            if ((m0 >> q) & 1u) { wc.v[pos] = mv[q]; wc.l[pos] = 0; ++pos; }
#pragma unroll
        for (int q = 0; q < 4 * SU; ++q)
            if ((m1 >> q) & 1u) { wc.v[pos] = mv[q]; wc.l[pos] = 1; ++pos; }
        wc.cnt += tot;
        __syncwarp();
    }
    if (base < n4) {                                     // the grid's partial chunk
        for (int u = 0; u < SU; ++u)
            for (int j = 0; j < 4; ++j) {
                const long long i = 4 * (base + t + (long long)u * 256) + j;
                if (i >= n) continue;
                const float mv = __ldg(mean + i);
                const uint32_t k = fkey(mv);
                bel0 += k < lo0;
                bel1 += k < lo1;
                for (int g = 0; g < 2; ++g)
                    if (k >= (g ? lo1 : lo0) && k <= (g ? hi1 : hi0)) {
                        const unsigned long long pos = atomicAdd(&ctl->ncand, 1ull);
                        if ((long long)pos < cap) { cval[pos] = mv; clab[pos] = (uint8_t)g; }
                    }
            }
    }
    wc.flush(cval, clab, &ctl->ncand, cap);
    const unsigned int s0 = __reduce_add_sync(full, bel0), s1 = __reduce_add_sync(full, bel1);
    if ((t & 31) == 0) {
        if (s0) atomicAdd(&ctl->wbelow[0], (unsigned long long)s0);
        if (s1) atomicAdd(&ctl->wbelow[1], (unsigned long long)s1);
    }
}

// After the counting pass (one thread): arms the candidate block for its first digit pass
// (both targets active with the empty prefix, like the bin selection's labelling pass), or,
// when the candidate list overflowed, sends the selection to the radix passes.
FY_D void k_win_arm(NoiseCtl* __restrict__ ctl, NoiseCtl* __restrict__ cc, long long cap) {
    fy_pdl_wait();
    if (ctl->mode != kModeWin0) { cc->mode = 3; return; }
    for (int t = 0; t < NT_MAX; ++t) target_init(cc, t, 0, 0, t < 2);
    cc->ntarget = 2;
    cc->n = (long long)(ctl->ncand < (unsigned long long)cap ? ctl->ncand : (unsigned long long)cap);
    ctl->wfail = 0;
    if ((long long)ctl->ncand > cap || (noise_force_radix & 1)) {
        cc->mode = 3;
        ctl->wfail = 1;
        ctl->mode = 0;                     // the radix passes over the whole field
    } else {
        cc->mode = 1;
    }
}

// After the candidates' first digit pass (one block per target): the target's inside count
// is the sum of its histogram; its rank among the candidates is r = k - below, which must
// leave k and (when it exists) k+1 inside. Otherwise the window failed: the candidate passes
// stand aside (cc mode 3) and the radix passes over the whole field run (mode 0). A block
// that finds cc already failed leaves its histogram, which every later user clears first.
FY_D void k_win_targets(NoiseCtl* __restrict__ ctl, NoiseCtl* __restrict__ cc) {
    fy_pdl_wait();
    __shared__ unsigned long long part[256];
    if (cc->mode != 1) return;
    const int t = vbx();
    if (t >= cc->ntarget) return;
    unsigned int* h = cc->hist + (size_t)t * 256;
    part[threadIdx.x] = h[threadIdx.x];
    __syncthreads();
    for (int off = 128; off > 0; off >>= 1) {
        if (threadIdx.x < off) part[threadIdx.x] += part[threadIdx.x + off];
        __syncthreads();
    }
    const long long in = (long long)part[0];
    const long long k = ctl->tk[t];
    const long long r = k - (long long)ctl->wbelow[t];
    const bool has_next = k + 1 < ctl->n;
    const bool ok = r >= 0 && r < in && (!has_next || r + 1 < in);
    __syncthreads();
    if (!ok) h[threadIdx.x] = 0;                         // inactive: its histogram is cleared
    if (threadIdx.x == 0) {
        target_init(cc, t, ok ? r : 0, in, ok);
        if (!ok) {
            ctl->wfail = 1;
            cc->mode = 3;
            ctl->mode = 0;
        }
    }
}

// The bins' candidate list (section 2b). Reset before the compacting pass.
FY_D void k_bin_cand_reset(NoiseCtl* __restrict__ ctl) {
    fy_pdl_wait();
    if (ctl->mode == 1) ctl->ncand = 0;
}
// After the compacting pass and its scan: when the list fits, the bins' targets move to the
// candidate block for the last digit and the whole-field pass stands aside; otherwise the
// candidate pass stands aside.
FY_D void k_bin_arm(NoiseCtl* __restrict__ ctl, NoiseCtl* __restrict__ cc, long long cap) {
    fy_pdl_wait();
    __shared__ int s_go;
    if (threadIdx.x == 0) s_go = ctl->mode == 1 && (long long)ctl->ncand <= cap;
    __syncthreads();
    if (!s_go) {
        if (threadIdx.x == 0) cc->mode = 3;
        return;
    }
    for (int i = threadIdx.x; i < NB * 256; i += blockDim.x) cc->hist[i] = 0;
    for (int t = threadIdx.x; t < NT_MAX; t += blockDim.x) {
        cc->tk[t] = ctl->tk[t];
        cc->trank[t] = ctl->trank[t];
        cc->tgroup_n[t] = ctl->tgroup_n[t];
        cc->tprefix[t] = ctl->tprefix[t];
        cc->tactive[t] = ctl->tactive[t];
        cc->teq[t] = 0;
        cc->tneed_next[t] = 0;
        cc->tnext[t] = 0xffffffffu;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        cc->n = (long long)ctl->ncand;
        cc->ntarget = ctl->ntarget;
        cc->mode = 1;
        ctl->mode = kModeBinCand;
    }
}
// After the candidates' last digit: the selected keys back into the main block.
FY_D void k_bin_finish(NoiseCtl* __restrict__ ctl, const NoiseCtl* __restrict__ cc) {
    fy_pdl_wait();
    if (ctl->mode != kModeBinCand) return;
    for (int t = 0; t < NT_MAX; ++t) {
        ctl->tprefix[t] = cc->tprefix[t];
        ctl->trank[t] = cc->trank[t];
        ctl->teq[t] = cc->teq[t];
        ctl->tneed_next[t] = cc->tneed_next[t];
        ctl->tnext[t] = cc->tnext[t];
    }
    ctl->mode = 1;
}

// Keys of order statistics k and k+1 into the main block's targets 0/1 (interp / next_value
// form); the radix passes of mode 0 then stand aside.
FY_D void k_win_finish(NoiseCtl* __restrict__ ctl, const NoiseCtl* __restrict__ cc) {
    fy_pdl_wait();
    if (ctl->mode != kModeWin0) return;
    for (int t = 0; t < 2; ++t) {
        ctl->tprefix[t] = cc->tprefix[t];
        ctl->tnext[t] = cc->tneed_next[t] ? cc->tnext[t] : cc->tprefix[t];
        ctl->tneed_next[t] = 1;
        ctl->tactive[t] = 1;
    }
    atomicOr(&noise_window_used, 1);
}

// ---------------------------------------------------------------- 2bw. the bins' window
// The flat_pct percentile of the variance per intensity bin by the scheme of section 2w,
// so the variance field is read once instead of once per digit:
//   sample   m (<= kBinSampleMax) voxels at positions (A*i + B) mod n: the key of each
//            variance and the bin of its mean (255: outside every bin).
//   window   one CTA per bin gathers the bin's sample keys in sample order (at most
//            kBinKeysMax) and takes the order statistics kWinSigmas binomial standard
//            deviations either side of the target's sample rank, each widened to its 16-bit
//            key bucket (two digit passes): [bwlo, bwhi]. Under 64 samples: every key.
//   count    one branch-free pass over mean and variance: per bin its voxels (the bin count,
//            noise.c:118-123) and the keys below its window; the keys inside go to the
//            candidate list with their bin.
//   arm      for each bin of >= 200 voxels, r = k - below with k = flat_pct/100*(count - 1);
//            the first digit pass over the candidates (control block cc, targets = bins) gives
//            the inside counts, and k and k+1 must be inside (k_bwin_targets); the other three
//            digit passes then select them. A miss, an overfull list or a failed bin guess
//            sends the bins to the radix passes over the whole field (mode 1).
//   finish   the keys of k and k+1 into the main block; mode kModeBinDone makes the radix
//            passes stand aside.
constexpr int kBinSampleMax = 65536;
constexpr int kBinKeysMax = 4096;      // per bin: enough for a window of ~5% of a large bin

FY_D void k_bwin_sample(const float* __restrict__ mean, const float* __restrict__ var,
                                                     const NoiseCtl* __restrict__ ctl, uint32_t* __restrict__ skey,
                                                     uint8_t* __restrict__ slab, long long m, unsigned long long A,
                                                     unsigned long long B) {
    fy_pdl_wait();
    __shared__ float fe[NB + 1];
    if (ctl->mode != kModeBinWin) return;
    if (threadIdx.x <= NB) fe[threadIdx.x] = ctl->fedge[threadIdx.x];
    __syncthreads();
    const float lo_f = fe[0], fscale = ctl->fscale;
    const unsigned long long n = (unsigned long long)ctl->n;
    for (long long i = (long long)vbx() * blockDim.x + threadIdx.x; i < m; i += (long long)vgx() * blockDim.x) {
        const unsigned long long q = (A * (unsigned long long)i + B) % n;
        const float mv = __ldg(mean + q), vv = __ldg(var + q);
        const int b = bin_of(mv, fe, lo_f, fscale);
        skey[i] = fkey(vv);
        slab[i] = (uint8_t)(b < 0 ? 255 : b);
    }
}

// One CTA (kBoundThreads threads) per bin. Dynamic shared memory as k_win_bounds. Each warp
// owns a contiguous slice of the sample (whole 512-entry steps, 16 labels per lane and step,
// read 16 bytes at a time, the next step's while the current one is placed) and compacts its
// bin's keys in sample order into its own kBinKeysMax/NW slots, with no block barrier; one
// block pass then concatenates the warps' keys (a deterministic subset in sample order).
FY_D void k_bwin_bounds(const uint32_t* __restrict__ skey,
                                                               const uint8_t* __restrict__ slab,
                                                               NoiseCtl* __restrict__ ctl, long long m) {
    fy_pdl_wait();
    constexpr int NTB = kBoundThreads, NW = NTB / 32, U = 16, STEP = 32 * U, WCAP = kBinKeysMax / NW;
    static_assert(2 * kBinKeysMax <= kSampleMax, "staging and compacted keys share the key array");
    extern __shared__ uint32_t wkeys[];
    unsigned int* wh = wkeys + kSampleMax;
    uint32_t* keys = wkeys + kBinKeysMax;                 // the concatenated keys
    __shared__ unsigned long long part[NTB];
    __shared__ uint32_t s_sel[2];
    __shared__ int s_wc[NW];
    if (ctl->mode != kModeBinWin) return;
    const int b = vbx(), t = threadIdx.x, lane = t & 31, w = t >> 5;
    const unsigned full = 0xffffffffu;
    auto load_labels = [&](long long e0, uint8_t* lab) {
        if (e0 + U <= m) {
            const uint4 v = __ldg(reinterpret_cast<const uint4*>(slab + e0));
            const uint32_t wv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (int j = 0; j < U; ++j) lab[j] = (uint8_t)(wv[j >> 2] >> (8 * (j & 3)));
        } else {
#pragma unroll
            for (int j = 0; j < U; ++j) lab[j] = e0 + j < m ? slab[e0 + j] : (uint8_t)255;
        }
    };
    // this warp's slice: whole steps, so every 16-label read is 16-byte aligned
    const long long steps = (m + STEP - 1) / STEP, per = (steps + NW - 1) / NW;
    const long long s0 = (long long)w * per * STEP, s1 = s0 + per * STEP < m ? s0 + per * STEP : m;
    uint32_t* mine = wkeys + w * WCAP;
    int wc = 0;                                           // warp-uniform
    uint8_t nxt[U];
    if (s0 < s1) load_labels(s0 + lane * U, nxt);
    for (long long i0 = s0; i0 < s1 && wc < WCAP; i0 += STEP) {
        uint8_t lab[U];
#pragma unroll
        for (int j = 0; j < U; ++j) lab[j] = nxt[j];
        const long long e0 = i0 + lane * U;
        if (i0 + STEP < s1) load_labels(e0 + STEP, nxt);
        unsigned hit = 0;
#pragma unroll
        for (int j = 0; j < U; ++j) hit |= (unsigned)(lab[j] == (uint8_t)b && e0 + j < s1) << j;
        const int cnt = __popc(hit);
        int incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(full, incl, o);
            if (lane >= o) incl += y;
        }
        int pos = wc + incl - cnt;
#pragma unroll
        for (int j = 0; j < U; ++j)
            if ((hit >> j) & 1u) {
                if (pos < WCAP) mine[pos] = __ldg(skey + e0 + j);
                ++pos;
            }
        const int tot = __shfl_sync(full, incl, 31);
        wc = wc + tot < WCAP ? wc + tot : WCAP;
    }
    if (lane == 0) s_wc[w] = wc;
    __syncthreads();
    int off = 0, c = 0;
#pragma unroll
    for (int ww = 0; ww < NW; ++ww) {
        const int v = s_wc[ww];
        off += ww < w ? v : 0;
        c += v;
    }
    for (int i = lane; i < wc; i += 32) keys[off + i] = mine[i];
    __syncthreads();
    uint32_t lo = 0u, hi = 0xffffffffu;
    if (c >= 64) {
        const double q = ctl->flat_pct / 100.0;
        const double qc = q < 1.0 / c ? 1.0 / c : (q > 1.0 - 1.0 / c ? 1.0 - 1.0 / c : q);
        const long long ks = (long long)(q * (double)(c - 1));
        const long long d = (long long)ceil(kWinSigmas * sqrt((double)c * qc * (1.0 - qc))) + 4;
        if (ks - d >= 0) lo = block_select(keys, c, ks - d, wh, part, s_sel, 2);
        if (ks + d + 1 < c) hi = block_select(keys, c, ks + d + 1, wh, part, s_sel, 2) | 0xffffu;
    }
    if (t == 0) {
        ctl->bwlo[b] = lo;
        ctl->bwhi[b] = hi;
    }
}

// The counting pass of the bins' windows: mean and variance read once, SUB float4 of each
// per thread and step. Every voxel takes the same branch-free path: its bin from the float
// guess corrected by one step (exact unless the range [lo, hi] is degenerate; a voxel whose
// corrected bin fails the exact membership test raises ctl->wfail and the bins fall back to
// the radix passes), the key of its variance against the bin's window, and one
// read-modify-write of the lane's own shared-memory counter of its bin (low 16 bits: the
// bin's voxels, high 16 bits: those below the window; rows of 25 words, so the lanes of a
// warp hit distinct banks when they share a bin; added into the CTA's totals before a field
// can pass 65535). The keys inside the window are placed by one warp scan per step in the
// warp's buffer and appended to the list (one atomic per buffer), as in k_win_count. The
// inside counts come from the candidates' first digit histogram (k_bwin_targets).
constexpr int kBCountBuf = 512;          // per warp: two steps' worst case (32 x 8 each)
constexpr int kLaneRow = 25;             // counter words per lane (NB = 24, odd stride)
FY_D void k_bwin_count(const float* __restrict__ mean, const float* __restrict__ var,
                                                       NoiseCtl* __restrict__ ctl, float* __restrict__ cval,
                                                       uint8_t* __restrict__ clab, long long cap) {
    fy_pdl_wait();
    constexpr int SUB = 2;                               // float4 of each field per thread and step
    static_assert(32 * 4 * SUB <= kBCountBuf && NB < kLaneRow, "buffer and counter rows");
    __shared__ float bufv[256 / 32][kBCountBuf];
    __shared__ uint8_t bufl[256 / 32][kBCountBuf];
    __shared__ unsigned int lc[256 * kLaneRow];          // per-lane counters
    __shared__ float fe[NB + 1];
    __shared__ uint32_t swl[NB], swh[NB];
    __shared__ float4 stab[NB];                          // per bin: its edges and its window
    __shared__ unsigned int sc[NB * 3];
    __shared__ int s_bad;
    if (ctl->mode != kModeBinWin) return;
    const unsigned full = 0xffffffffu;
    const int t = threadIdx.x, lane = t & 31;
    if (t <= NB) fe[t] = ctl->fedge[t];
    if (t < NB) {
        const uint32_t wl = ctl->bwlo[t], wh = ctl->bwhi[t];
        swl[t] = wl;
        swh[t] = wh;
        stab[t] = make_float4(ctl->fedge[t], ctl->fedge[t + 1], __uint_as_float(wl), __uint_as_float(wh));
    }
    for (int i = t; i < NB * 3; i += blockDim.x) sc[i] = 0;
    for (int i = t; i < 256 * kLaneRow; i += blockDim.x) lc[i] = 0;
    if (t == 0) s_bad = 0;
    __syncthreads();
    const float lo_e = fe[0], hi_e = fe[NB], fscale = ctl->fscale;
    unsigned int* row = lc + t * kLaneRow;
    WarpCands wc;
    wc.v = bufv[t >> 5];
    wc.l = bufl[t >> 5];
    bool bad = false;
    // bin (or -1 outside every bin) and whether the key is inside the bin's window. One
    // 16-byte lookup gives the guessed bin's edges and window; when the mean lies outside the
    // guess (rare: rounding at an edge), one step to the neighbour and the exact-membership
    // check of the step run as before.
    auto classify = [&](float m, float v, bool valid, int& bo, bool& inside) {
        const bool inr = valid && m >= lo_e && m < hi_e;
        const float mc = inr ? m : lo_e;
        int b = (int)((mc - lo_e) * fscale);
        b = b < 0 ? 0 : (b > NB - 1 ? NB - 1 : b);
        const float4 e = stab[b];
        uint32_t wl = __float_as_uint(e.z), wh = __float_as_uint(e.w);
        if (!(mc >= e.x && mc < e.y)) {
            b = b - (int)(mc < e.x) + (int)(mc >= e.y);
            bad |= !(mc >= fe[b] && mc < fe[b + 1]);
            wl = swl[b];
            wh = swh[b];
        }
        const uint32_t k = fkey(v);
        row[b] += inr ? (k < wl ? 0x10001u : 1u) : 0u;
        inside = inr && k >= wl && k <= wh;
        bo = b;
    };
    auto flush_rows = [&]() {                             // CTA-uniform
        __syncthreads();
        for (int i = t; i < NB * 2; i += blockDim.x) {   // one thread per bin and field
            const int bb = i >> 1, hi = i & 1;
            unsigned int sum = 0;
            for (int l = 0; l < 256; ++l) {
                const unsigned int w = lc[l * kLaneRow + bb];
                sum += hi ? w >> 16 : w & 0xffffu;
            }
            if (sum) atomicAdd(&sc[3 * bb + (hi ? 0 : 2)], sum);
        }
        __syncthreads();
        for (int i = 0; i < NB; ++i) row[i] = 0;
        __syncthreads();
    };
    const long long n = ctl->n, n4 = (n + 3) / 4, n4f = n / 4;
    const long long chunk = (long long)SUB * 256;
    long long base = (long long)vbx() * chunk;
    const long long stride = (long long)vgx() * chunk;        // read once: the loop body has syncs
    int steps = 0;
    for (; base + chunk <= n4f; base += stride) {
        float4 xm[SUB], xv[SUB];
#pragma unroll
        for (int u = 0; u < SUB; ++u) {
            const long long q = base + (long long)t * SUB + u;
            xm[u] = __ldg(reinterpret_cast<const float4*>(mean) + q);
            xv[u] = __ldg(reinterpret_cast<const float4*>(var) + q);
        }
        float vv[4 * SUB];
        int bq[4 * SUB];
        unsigned hit = 0;
#pragma unroll
        for (int u = 0; u < SUB; ++u) {
            const float mm[4] = {xm[u].x, xm[u].y, xm[u].z, xm[u].w};
            vv[4 * u] = xv[u].x; vv[4 * u + 1] = xv[u].y; vv[4 * u + 2] = xv[u].z; vv[4 * u + 3] = xv[u].w;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                bool ins;
                classify(mm[j], vv[4 * u + j], true, bq[4 * u + j], ins);
                hit |= (unsigned)ins << (4 * u + j);
            }
        }
        if (++steps == 65535 / (4 * SUB)) {              // a 16-bit field could pass 65535
            flush_rows();
            steps = 0;
        }
        const int c = __popc(hit);
        int incl = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(full, incl, o);
            if (lane >= o) incl += y;
        }
        const int tot = __shfl_sync(full, incl, 31);
        if (tot == 0) continue;
        if (wc.cnt + tot > kBCountBuf) wc.flush(cval, clab, &ctl->ncand, cap);     // warp-uniform
        int pos = wc.cnt + incl - c;
#pragma unroll
        for (int q = 0; q < 4 * SUB; ++q)
            if ((hit >> q) & 1u) { wc.v[pos] = vv[q]; wc.l[pos] = (uint8_t)bq[q]; ++pos; }
        wc.cnt += tot;
        __syncwarp();
    }
    if (base < n4) {                                      // the grid's partial chunk (CTA-uniform)
        for (int u = 0; u < SUB; ++u)
            for (int j = 0; j < 4; ++j) {
                const long long i = 4 * (base + (long long)t * SUB + u) + j;
                const bool valid = i < n;
                const float v = valid ? __ldg(var + i) : 0.f;
                int b;
                bool ins;
                classify(valid ? __ldg(mean + i) : 0.f, v, valid, b, ins);
                if (ins) {
                    const unsigned long long pos = atomicAdd(&ctl->ncand, 1ull);
                    if ((long long)pos < cap) { cval[pos] = v; clab[pos] = (uint8_t)b; }
                }
            }
    }
    wc.flush(cval, clab, &ctl->ncand, cap);
    if (bad) s_bad = 1;
    flush_rows();
    for (int i = t; i < NB * 3; i += blockDim.x)
        if (sc[i]) atomicAdd(&ctl->bwc[i], (unsigned long long)sc[i]);
    if (t == 0 && s_bad) atomicExch(&ctl->wfail, 1);
}

// After the counting pass: the bin counts, and, when the list fits and every bin's guess held,
// the candidate block armed for the bins' digit passes with r = k - below for each bin of
// >= 200 voxels (noise.c:123); otherwise the radix passes over the whole field (mode 1).
// ctl->bwc per bin: [0] keys below the window, [2] the bin's voxels.
FY_D void k_bwin_arm(NoiseCtl* __restrict__ ctl, NoiseCtl* __restrict__ cc, long long cap) {
    fy_pdl_wait();
    __shared__ int s_ok;
    if (ctl->mode != kModeBinWin) {
        if (threadIdx.x == 0) cc->mode = 3;
        return;
    }
    const int t = threadIdx.x;
    if (t == 0) s_ok = (long long)ctl->ncand <= cap && !ctl->wfail && !(noise_force_radix & 2);
    __syncthreads();
    long long cnt = 0, r = 0;
    bool on = false;
    if (t < NB) {
        const long long below = (long long)ctl->bwc[3 * t];
        cnt = (long long)ctl->bwc[3 * t + 2];
        on = cnt >= 200;
        if (on) {
            const double idx = ctl->flat_pct / 100.0 * (double)(cnt - 1);
            r = (long long)idx - below;
            if (r < 0) s_ok = 0;
        }
    }
    __syncthreads();
    if (!s_ok) {
        if (t == 0) {
            cc->mode = 3;
            ctl->mode = 1;
        }
        return;
    }
    for (int i = t; i < NB * 256; i += blockDim.x) cc->hist[i] = 0;
    if (t < NT_MAX) target_init(cc, t, on ? r : 0, 0, on);
    if (t < NB) ctl->bcount[t] = (unsigned long long)cnt;
    __syncthreads();
    if (t == 0) {
        cc->n = (long long)ctl->ncand;
        cc->ntarget = NB;
        cc->mode = 1;
    }
}

// After the candidates' first digit pass (one block per bin): the bin's inside count is the sum
// of its histogram; k and (when it exists) k+1 must be inside, else the bins go to the radix
// passes over the whole field.
FY_D void k_bwin_targets(NoiseCtl* __restrict__ ctl, NoiseCtl* __restrict__ cc) {
    fy_pdl_wait();
    __shared__ unsigned long long part[256];
    if (cc->mode != 1 || ctl->mode != kModeBinWin) return;
    const int b = vbx();
    if (!cc->tactive[b]) return;
    unsigned int* h = cc->hist + (size_t)b * 256;
    part[threadIdx.x] = h[threadIdx.x];
    __syncthreads();
    for (int off = 128; off > 0; off >>= 1) {
        if (threadIdx.x < off) part[threadIdx.x] += part[threadIdx.x + off];
        __syncthreads();
    }
    const long long in = (long long)part[0];
    const long long r = cc->trank[b];
    const long long k = r + (long long)ctl->bwc[3 * b];
    const bool has_next = k + 1 < (long long)ctl->bcount[b];
    if (threadIdx.x == 0) {
        if (r < in && (!has_next || r + 1 < in)) {
            target_init(cc, b, r, in, true);
        } else {
            cc->mode = 3;
            ctl->mode = 1;
        }
    }
}

// The bins' selected keys (k and k+1, in the form interp() reads) into the main block.
FY_D void k_bwin_finish(NoiseCtl* __restrict__ ctl, const NoiseCtl* __restrict__ cc) {
    fy_pdl_wait();
    if (ctl->mode != kModeBinWin) return;
    const int t = threadIdx.x;
    if (t < NB) {
        ctl->tprefix[t] = cc->tprefix[t];
        ctl->tnext[t] = cc->tneed_next[t] ? cc->tnext[t] : cc->tprefix[t];
        ctl->tneed_next[t] = 1;
        ctl->tactive[t] = cc->tactive[t];
    }
    __syncwarp();
    if (t == 0) {
        ctl->mode = kModeBinDone;
        atomicOr(&noise_window_used, 2);
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

// stage 0: bin floors; arm the whole-volume fallback when no bin qualifies (mode 2).
// stage 1: IRLS fit (FP64) and outputs.
// One warp: lane b handles bin b's reads, so the bins' loads are in flight together; the
// sequential fit then runs on lane 0 from shared memory.
FY_D void k_noise_fit(NoiseCtl* ctl, int stage) {
    fy_pdl_wait();
    static_assert(NB <= 32, "one lane per bin");
    const int lane = threadIdx.x;
    if (stage == 0) {
        bool use = false;
        if (lane < NB) {
            const long long c = (long long)ctl->bcount[lane];
            if (c >= 200) {
                const double idx = ctl->flat_pct / 100.0 * (double)(c - 1);
                const long long k = (long long)idx;
                ctl->bfloor[lane] = interp(ctl, lane, idx - (double)k, k + 1 < c);
                use = true;
            }
        }
        const int used = __popc(__ballot_sync(0xffffffffu, use));
        if (lane != 0) return;
        ctl->out_used = used;
        if (used == 0) {                                  // noise.c:166-171
            const long long n = ctl->n;
            const double idx = ctl->flat_pct / 100.0 * (double)(n - 1);
            for (int t = 0; t < NT_MAX; ++t) target_init(ctl, t, 0, 0, false);
            target_init(ctl, 0, (long long)idx, n, true);
            ctl->ntarget = 1;
            ctl->mode = 2;
        } else {
            ctl->mode = 3;
        }
        return;
    }
    // stage 1: the used bins compacted in bin order; the weights, residuals and the median
    // of the residuals are formed by one lane per bin, the five weighted sums by lane 0 in the
    // reference's order (noise.c:141-147), so every value equals the sequential fit's
    __shared__ double s_i[NB], s_f[NB], s_w[NB], s_r[NB];
    __shared__ long long s_c[NB];
    __shared__ double s_g, s_b;
    __shared__ int s_brk;
    const unsigned full = 0xffffffffu;
    const bool in_use = lane < NB && (long long)ctl->bcount[lane] >= 200;
    const unsigned um = __ballot_sync(full, in_use);
    const int used = __popc(um);
    if (in_use) {
        const int pos = __popc(um & ((1u << lane) - 1u));
        s_c[pos] = (long long)ctl->bcount[lane];
        s_i[pos] = 0.5 * (ctl->edge[lane] + ctl->edge[lane + 1]);
        s_f[pos] = ctl->bfloor[lane];
    }
    __syncwarp();
    double g = 0, bb = 0;
    if (ctl->mode == 2) {
        if (lane == 0) {
            const long long n = ctl->n;
            const double idx = ctl->flat_pct / 100.0 * (double)(n - 1);
            const long long k = (long long)idx;
            bb = interp(ctl, 0, idx - (double)k, k + 1 < n);
        }
    } else if (used >= 3) {                               // IRLS, noise.c:139-161
        if (lane < used) s_w[lane] = sqrt((double)s_c[lane]);
        __syncwarp();
        for (int it = 0; it < 4; it++) {
            if (lane == 0) {
                double Sw = 0, Swx = 0, Swy = 0, Swxx = 0, Swxy = 0;
                for (int i = 0; i < used; i++) {
                    const double wi = s_w[i], xi = s_i[i], yi = s_f[i];
                    Sw += wi; Swx += wi * xi; Swy += wi * yi; Swxx += wi * xi * xi; Swxy += wi * xi * yi;
                }
                const double det = Sw * Swxx - Swx * Swx;
                s_brk = fabs(det) < 1e-20;
                if (!s_brk) {
                    s_g = (Sw * Swxy - Swx * Swy) / det;
                    s_b = (Swxx * Swy - Swx * Swxy) / det;
                }
            }
            __syncwarp();
            if (s_brk) break;
            g = s_g;
            bb = s_b;
            double res = 0.0;
            if (lane < used) {
                res = fabs(s_f[lane] - (g * s_i[lane] + bb));
                s_r[lane] = res;
            }
            __syncwarp();
            // percentile(resid, used, 50) (noise.c:66-73): the values at sorted positions lo and
            // lo + 1, found by ranking each residual (ties by index)
            const double pidx = 50.0 / 100.0 * (used - 1);
            const int plo = (int)pidx;
            const double pf = pidx - plo;
            int rank = 0;
            if (lane < used)
                for (int j = 0; j < used; ++j) rank += s_r[j] < res || (s_r[j] == res && j < lane);
            const unsigned mlo = __ballot_sync(full, lane < used && rank == plo);
            const unsigned mhi = __ballot_sync(full, lane < used && rank == plo + 1);
            const double vlo = __shfl_sync(full, res, mlo ? __ffs(mlo) - 1 : 0);    // (no rank: NaN residuals)
            const double vhi = __shfl_sync(full, res, mhi ? __ffs(mhi) - 1 : (mlo ? __ffs(mlo) - 1 : 0));
            const double med = (plo + 1 < used ? vlo * (1 - pf) + vhi * pf : vlo) + 1e-9;
            if (lane < used) {
                const double rr = res / (2.0 * med);
                s_w[lane] = sqrt((double)s_c[lane]) / (1.0 + rr * rr);
            }
            __syncwarp();
        }
    } else if (used > 0) {                                // noise.c:162-165
        if (lane == 0) {
            double sum = 0;
            for (int i = 0; i < used; i++) sum += s_f[i];
            bb = sum / used;
        }
    }
    if (lane != 0) return;
    if (!isfinite(g)) g = 0;
    if (!isfinite(bb)) bb = 0;
    double var_ref = g * ctl->ref_intensity + bb;
    if (var_ref < 0) var_ref = bb > 0 ? bb : 0;
    const double noise_ref = sqrt(var_ref) * 1.15;      // noise.c:181-187
    ctl->out_g = g; ctl->out_b = bb;
    ctl->out_noise_ref = noise_ref;
    ctl->out_ref_intensity = ctl->ref_intensity;
    double eps = (3.0 * noise_ref) * (3.0 * noise_ref);  // noise.c:197-202
    if (!(eps > 1e-8)) eps = 1e-8;
    ctl->eps = (float)eps;
}

unsigned grid_sel(long long n, int sms) {
    long long g = (n / 4 + 256 * SU - 1) / (256 * SU);
    const long long cap = (long long)sms * 8;
    return (unsigned)(g < cap ? (g ? g : 1) : cap);
}

}  // namespace

size_t fy_noise_ctl_bytes() { return (sizeof(NoiseCtl) + 255) & ~(size_t)255; }

namespace {
// Scratch layout (floats; every sub-array 256-byte aligned for the vector loads): mean, var,
// bin labels (bytes), the candidates' control block, the sample of means, and the candidate
// list (values, then labels) of capacity n/8 + 4096 (the window holds ~1% of the voxels).
size_t round64(size_t v) { return (v + 63) & ~(size_t)63; }
struct NoiseLayout {
    size_t mean, var, bin, cc, samp, cval, clab, total;
    long long cap;
};
NoiseLayout noise_layout(size_t n) {
    NoiseLayout L;
    const size_t nr = round64(n);
    L.mean = 0;
    L.var = nr;
    L.bin = 2 * nr;
    L.cc = L.bin + round64((n + 3) / 4);
    L.samp = L.cc + round64((sizeof(NoiseCtl) + 3) / 4);
    L.cap = (long long)((n + 7) / 8 + 4096);
    L.cval = L.samp + (size_t)kSampleMax;
    L.clab = L.cval + round64((size_t)L.cap);
    L.total = L.clab + round64(((size_t)L.cap + 3) / 4);
    return L;
}
// Weyl step for the sample positions: a prime a with gcd(a, n) = 1, reduced mod n (for a
// prime a that means n < a, or a not dividing n).
unsigned long long weyl_step(unsigned long long n) {
    if (n <= 1) return 1;
    const unsigned long long primes[4] = {2654435761ull, 2246822519ull, 3266489917ull, 668265263ull};
    for (unsigned long long a : primes)
        if (n < a || n % a != 0) return a % n;
    return 1;
}
}  // namespace

size_t fy_noise_scratch_floats(size_t n) { return noise_layout(n).total; }

namespace {

// ---------------------------------------------------------------- launching: one cube or a batch
// Every selection step above is a __device__ body run by one of two wrappers: k_one, one volume,
// the body's arguments as kernel parameters; k_many, a batch of volumes, the CTA's volume from
// its block index
// and each volume's arguments read from a device array. NoiseLaunch either launches k_one at
// once or, in batch mode, records each volume's arguments and grid for every step of the
// sequence (the same sequence for every volume) and then replays it: one launch per step for
// all volumes, each volume with the CTAs it asked for (their blocks are numbered per volume
// through vbx()/vgx(); the grids that index targets or bins along y are the same for all).
template <int NTB, int MINB, auto F, class... P>
__global__ void __launch_bounds__(NTB, MINB) k_one(P... a) {
    s_vbx = blockIdx.x;                    // every thread stores the same values
    s_vgx = gridDim.x;
    F(a...);
}
// prefix[v] = the first CTA (along x) of volume v, prefix[nvol] = all of them
template <int NTB, int MINB, auto F, class... P>
__global__ void __launch_bounds__(NTB, MINB) k_many(const cuda::std::tuple<P...>* __restrict__ packs,
                                                     const unsigned* __restrict__ prefix, int nvol) {
    int lo = 0, hi = nvol - 1;             // the last volume whose first CTA <= blockIdx.x
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(prefix + mid) <= blockIdx.x) lo = mid; else hi = mid - 1;
    }
    s_vbx = blockIdx.x - __ldg(prefix + lo);
    s_vgx = __ldg(prefix + lo + 1) - __ldg(prefix + lo);
    cuda::std::apply([](auto... x) { F(x...); }, packs[lo]);
}

struct NoiseLaunch {
    cudaStream_t st = nullptr;
    bool record = false;
    struct Step {
        const void* kern;                  // the k_many instance
        dim3 grid, block;
        size_t smem, pack;                 // bytes of one volume's arguments
        std::vector<unsigned char> packs;
        std::vector<unsigned> gx;         // CTAs along x of each volume
    };
    std::vector<Step> steps;
    size_t si = 0;                         // the next step of the volume being recorded
    int cubes = 0;

    template <int NTB, int MINB, auto F, class... P, class... A>
    cudaError_t run_sig(void (*)(P...), dim3 grid, dim3 block, size_t smem, A... a) {
        if (!record) {
            auto k = k_one<NTB, MINB, F, P...>;
            cudaError_t e = fy_smem_optin(k, smem);
            if (e != cudaSuccess) return e;
            return fy_launch_pdl(k, grid, block, smem, st, (P)a...);
        }
        using T = cuda::std::tuple<P...>;
        const void* k = (const void*)k_many<NTB, MINB, F, P...>;
        if (si == steps.size()) {
            if (cubes > 0) return cudaErrorInvalidValue;          // every volume has the same sequence
            cudaError_t e = fy_smem_optin(k_many<NTB, MINB, F, P...>, smem);
            if (e != cudaSuccess) return e;
            steps.push_back(Step{k, grid, block, smem, sizeof(T), {}});
        }
        Step& s = steps[si++];
        if (s.kern != k || s.block.x != block.x || s.smem != smem) return cudaErrorInvalidValue;
        if (s.grid.y != grid.y) return cudaErrorInvalidValue;
        s.gx.push_back(grid.x);
        const T t((P)a...);
        const unsigned char* b = reinterpret_cast<const unsigned char*>(&t);
        s.packs.insert(s.packs.end(), b, b + sizeof(T));
        return cudaSuccess;
    }
    template <int NTB, int MINB, auto F, class... A>
    cudaError_t run(dim3 grid, dim3 block, size_t smem, A... a) {
        return run_sig<NTB, MINB, F>(F, grid, block, smem, a...);
    }
};

#define RUN(NTB, MINB, F, ...)                                                 \
    do {                                                                       \
        const cudaError_t pe_ = L.run<NTB, MINB, F>(__VA_ARGS__);              \
        if (pe_ != cudaSuccess) return pe_;                                    \
        ++launches;                                                            \
    } while (0)

// The estimate's launch sequence for one volume through L. stats: run the statistics pass here
// (a batch runs it for all volumes at once before the sequence).
cudaError_t noise_sequence(NoiseLaunch& L, const float* in, int nz, int ny, int nx, int win, double flat_pct,
                           double ref_intensity, float* scratch, void* ctl_mem, int sms, int& launches,
                           float* guided_mv, bool stats) {
    cudaStream_t st = L.st;
    NoiseCtl* ctl = (NoiseCtl*)ctl_mem;
    const long long n = (long long)nz * ny * nx;
    const NoiseLayout Lay = noise_layout((size_t)n);
    float* mean = scratch + Lay.mean;
    float* var = scratch + Lay.var;
    uint8_t* bin = (uint8_t*)(scratch + Lay.bin);
    NoiseCtl* cc = (NoiseCtl*)(scratch + Lay.cc);
    float* sm = scratch + Lay.samp;
    float* cval = scratch + Lay.cval;
    uint8_t* clab = (uint8_t*)(scratch + Lay.clab);
    const int r = win / 2;
    const float inv_wc = (float)(1.0 / ((double)win * win * win));
    const unsigned g = grid_sel(n, sms), gc = grid_sel(Lay.cap, sms);
    // passes that usually exit at once (the fallbacks, the k+1 scans): one CTA per SM, so the
    // common case schedules few empty CTAs; when they do run, their grid-stride loops cover
    // every voxel
    const unsigned gs = (unsigned)(g < (unsigned)sms ? g : (unsigned)sms);
    // candidate lists hold ~1-2% of the voxels (their capacity is n/8): two CTAs per SM
    const unsigned gcl = (unsigned)(gc < 2u * (unsigned)sms ? gc : 2u * (unsigned)sms);
    const size_t smem_all = 2 * 2048 * sizeof(unsigned int), smem_bin = NB * 256 * sizeof(unsigned int);
    const size_t smem_bin_c = smem_bin + (size_t)(256 / 32) * kCompactBuf * (sizeof(float) + 1);
    const size_t smem_keys = (kSampleMax + 256 * (kBoundThreads / 32)) * sizeof(uint32_t);   // keys + warp digit counts
    const long long m = n < kSampleMax ? n : kSampleMax;
    const unsigned long long wa = weyl_step((unsigned long long)n), wb = (unsigned long long)n / 3;
    RUN(256, 1, k_noise_setup, 1, 256, 0, ctl, cc, n, flat_pct, ref_intensity);
    if (stats) {   // 1. stats
        fyzb::Params sp{};
        sp.nz = nz; sp.ny = ny; sp.nx = nx;
        sp.f0 = in; sp.o0 = mean; sp.o1 = var; sp.o2 = guided_mv;
        sp.inv_wc = inv_wc; sp.wci = win * win * win;
        cudaError_t e0 = fyzb::launch<fyzb::ZB_NOISE>(sp, r, sms, st);
        if (e0 != cudaSuccess) return e0;
        ++launches;
        if (!L.record) fy_prof_mark(st, "noise.stats");
    }
    // 2a. 1st/99th percentile of the means: sample-guided window pass, then the radix passes
    // of mode 1 over the candidates (control block cc, targets = labels); the radix passes
    // over the whole field (11 + 11 + 10 bits, then the k+1 neighbours) run only if the
    // window misses
    RUN(256, 1, k_win_sample, 64, 256, 0, mean, ctl, sm, m, wa, wb);
    RUN(kBoundThreads, 1, k_win_bounds, dim3(2, 2), kBoundThreads, smem_keys, sm, ctl, m);
    RUN(256, 3, k_win_count, g, 256, 0, mean, ctl, cval, clab, Lay.cap);
    RUN(32, 1, k_win_arm, 1, 1, 0, ctl, cc, Lay.cap);
    for (int sh = 24; sh >= 0; sh -= 8) {
        // the first digit's histogram sets the ranks (k_win_targets) before its scan; the
        // later digits' scans run in each pass's last CTA
        RUN(256, 1, (k_sel_hist<8, 1>), gcl, 256, smem_bin, nullptr, cval, clab, cc, sh, nullptr, nullptr, 0LL,
            sh == 24 ? -1 : (sh == 0 ? 1 : 0));
        if (sh == 24) {
            RUN(256, 1, k_win_targets, 2, 256, 0, ctl, cc);
            RUN(256, 1, k_sel_scan, 2, 256, 0, cc, 8, 1, 0);
        }
    }
    RUN(256, 1, k_sel_next, gs, 256, 0, nullptr, cval, clab, cc, 1);
    RUN(32, 1, k_win_finish, 1, 1, 0, ctl, cc);
    const int all_digits[3][2] = {{21, 11}, {10, 11}, {0, 10}};
    for (int i = 0; i < 3; ++i) {
        if (all_digits[i][1] == 11) RUN(256, 1, (k_sel_hist<11, 0>), gs, 256, smem_all, mean, var, bin, ctl, all_digits[i][0], nullptr, nullptr, 0LL, i == 2 ? 1 : 0);
        else RUN(256, 1, (k_sel_hist<10, 0>), gs, 256, smem_all, mean, var, bin, ctl, all_digits[i][0], nullptr, nullptr, 0LL, i == 2 ? 1 : 0);
    }
    RUN(256, 1, k_sel_next, gs, 256, 0, mean, var, bin, ctl, 0);
    RUN(NT_MAX, 1, k_noise_bins_setup, 1, NT_MAX, 0, ctl);
    if (!L.record) fy_prof_mark(st, "noise.lohi");
    // 2bw. per-bin flat_pct percentile of the variance through the bins' window: sample,
    // bounds, one counting pass over mean and variance, then four digit passes over the
    // candidates. The sample lives in the candidate region until the counting pass refills it.
    {
        long long m2 = n < kBinSampleMax ? n : kBinSampleMax;
        const long long m2cap = (Lay.cap - 64) * 4 / 5;    // keys, then labels 256-byte aligned
        if (m2 > m2cap) m2 = m2cap;
        uint32_t* skey = reinterpret_cast<uint32_t*>(cval);
        uint8_t* slab = reinterpret_cast<uint8_t*>(cval + round64((size_t)m2));
        RUN(256, 1, k_bwin_sample, 64, 256, 0, mean, var, ctl, skey, slab, m2, wa, (unsigned long long)n / 5);
        RUN(kBoundThreads, 1, k_bwin_bounds, NB, kBoundThreads, smem_keys, skey, slab, ctl, m2);
        RUN(256, 4, k_bwin_count, g, 256, 0, mean, var, ctl, cval, clab, Lay.cap);
        RUN(256, 1, k_bwin_arm, 1, 256, 0, ctl, cc, Lay.cap);
        for (int sh = 24; sh >= 0; sh -= 8) {
            // the first digit's histogram gives the inside counts (k_bwin_targets) before its
            // scan; the later digits' scans run in each pass's last CTA
            RUN(256, 1, (k_sel_hist<8, 1>), gcl, 256, smem_bin, nullptr, cval, clab, cc, sh, nullptr, nullptr, 0LL,
                sh == 24 ? -1 : (sh == 0 ? 1 : 0));
            if (sh == 24) {
                RUN(256, 1, k_bwin_targets, NB, 256, 0, ctl, cc);
                RUN(256, 1, k_sel_scan, NB, 256, 0, cc, 8, 1, 0);
            }
        }
        RUN(256, 1, k_sel_next, gcl, 256, 0, nullptr, cval, clab, cc, 1);
        RUN(32, 1, k_bwin_finish, 1, 32, 0, ctl, cc);
    }
    // 2b. (when the bins' window missed) per-bin flat_pct percentile of the variance by radix
    // passes over the whole field: 4 x 8 bits, then the k+1 neighbours;
    // the first pass also labels the voxels with their bins and yields the bin counts. The
    // third pass also lists the voxels that match their bin's 16-bit prefix (~1% of them),
    // and the last digit runs over that list (falling back to the whole field if it overflows).
    RUN(256, 1, (k_sel_hist<8, 1, true>), g, 256, smem_bin, mean, var, bin, ctl, 24, nullptr, nullptr, 0LL, -1);
    RUN(256, 1, k_bin_targets, NB, 256, 0, ctl);
    RUN(256, 1, k_sel_scan, NB, 256, 0, ctl, 8, 1, 0);
    RUN(256, 1, (k_sel_hist<8, 1>), g, 256, smem_bin, mean, var, bin, ctl, 16, nullptr, nullptr, 0LL, 0);
    RUN(32, 1, k_bin_cand_reset, 1, 1, 0, ctl);
    RUN(256, 1, (k_sel_hist<8, 1, false, true>), g, 256, smem_bin_c, mean, var, bin, ctl, 8, cval, clab, Lay.cap, 0);
    RUN(256, 1, k_bin_arm, 1, 256, 0, ctl, cc, Lay.cap);
    RUN(256, 1, (k_sel_hist<8, 1>), gs, 256, smem_bin, mean, var, bin, ctl, 0, nullptr, nullptr, 0LL, 1);       // overflow only
    RUN(256, 1, (k_sel_hist<8, 1>), gcl, 256, smem_bin, nullptr, cval, clab, cc, 0, nullptr, nullptr, 0LL, 1);  // the list
    // k+1 past the selected key's 24-bit prefix: the list holds every key of the bin that shares
    // its 16-bit prefix, so when it holds a larger key, its smallest larger key is the next one
    // (a key in between would share the prefix and be listed too). Only targets whose next key
    // leaves the 16-bit prefix are left to the whole-field scan below.
    RUN(256, 1, k_sel_next, gcl, 256, 0, nullptr, cval, clab, cc, 1);
    RUN(32, 1, k_bin_finish, 1, 1, 0, ctl, cc);
    RUN(256, 1, k_sel_next, gs, 256, 0, mean, var, bin, ctl, 1);
    RUN(32, 1, k_noise_fit, 1, 32, 0, ctl, 0);
    if (!L.record) fy_prof_mark(st, "noise.bin_select");
    // 2c. fallback (mode 2 only): flat_pct percentile over all voxels' variance
    for (int i = 0; i < 3; ++i) {
        if (all_digits[i][1] == 11) RUN(256, 1, (k_sel_hist<11, 2>), gs, 256, smem_all, mean, var, bin, ctl, all_digits[i][0], nullptr, nullptr, 0LL, i == 2 ? 1 : 0);
        else RUN(256, 1, (k_sel_hist<10, 2>), gs, 256, smem_all, mean, var, bin, ctl, all_digits[i][0], nullptr, nullptr, 0LL, i == 2 ? 1 : 0);
    }
    RUN(256, 1, k_sel_next, gs, 256, 0, mean, var, bin, ctl, 2);
    RUN(32, 1, k_noise_fit, 1, 32, 0, ctl, 1);
    return cudaSuccess;
}

}  // namespace

// Enqueue the whole estimate. scratch: fy_noise_scratch_floats(n) floats; ctl:
// fy_noise_ctl_bytes(). Supports win in {3..9} (r = win/2 <= 4). guided_mv (optional,
// 2n floats): the statistics pass also writes the guided filter's (mean, var) pairs of the
// same window, for fy_launch_guided_apply_mv with r = win/2.
// Every kernel runs as a programmatic dependent launch; the first failed launch is returned.
cudaError_t fy_launch_estimate_noise(const float* in, int nz, int ny, int nx, int win, double flat_pct,
                                     double ref_intensity, float* scratch, void* ctl_mem, int sms,
                                     cudaStream_t st, int& launches, float* guided_mv) {
    NoiseLaunch L;
    L.st = st;
    cudaError_t e = noise_sequence(L, in, nz, ny, nx, win, flat_pct, ref_intensity, scratch, ctl_mem, sms, launches,
                                   guided_mv, true);
    return e != cudaSuccess ? e : cudaGetLastError();
}

// ---------------------------------------------------------------- a batch of volumes
// The selection sequences of many volumes, recorded (no launch) for one replay: each step of
// the sequence becomes one launch over all volumes' CTAs. The statistics pass
// is not part of it (the caller runs it for every volume first: fy_noise_stats_params).
struct NoiseBatch {
    NoiseLaunch L;
    int launches = 0;                      // per volume
};
NoiseBatch* fy_noise_batch_record(const float* const* in, const int* dims, float* const* scratch,
                                  void* const* ctl_mem, int nvol, int win, double flat_pct, double ref_intensity,
                                  int sms, cudaError_t* err) {
    NoiseBatch* b = new NoiseBatch();
    b->L.record = true;
    *err = cudaSuccess;
    for (int i = 0; i < nvol && *err == cudaSuccess; ++i) {
        int launches = 0;
        b->L.si = 0;
        *err = noise_sequence(b->L, in[i], dims[3 * i], dims[3 * i + 1], dims[3 * i + 2], win, flat_pct, ref_intensity,
                              scratch[i], ctl_mem[i], sms, launches, nullptr, false);
        if (*err == cudaSuccess && b->L.si != b->L.steps.size()) *err = cudaErrorInvalidValue;
        b->L.cubes = i + 1;
        b->launches = launches;
    }
    if (*err != cudaSuccess) {
        delete b;
        return nullptr;
    }
    return b;
}
// Bytes of the packed steps: per step its volumes' arguments, then its table of first CTAs per
// volume (nvol + 1 entries), each 256-byte aligned.
static size_t al256n(size_t v) { return (v + 255) & ~(size_t)255; }
size_t fy_noise_batch_bytes(const NoiseBatch* b) {
    size_t t = 0;
    for (const auto& s : b->L.steps) t += al256n(s.packs.size()) + al256n((s.gx.size() + 1) * sizeof(unsigned));
    return t;
}
void fy_noise_batch_pack(const NoiseBatch* b, void* host) {
    unsigned char* h = (unsigned char*)host;
    for (const auto& s : b->L.steps) {
        memcpy(h, s.packs.data(), s.packs.size());
        h += al256n(s.packs.size());
        unsigned* pre = reinterpret_cast<unsigned*>(h);
        pre[0] = 0;
        for (size_t v = 0; v < s.gx.size(); ++v) pre[v + 1] = pre[v] + s.gx[v];
        h += al256n((s.gx.size() + 1) * sizeof(unsigned));
    }
}
int fy_noise_batch_steps(const NoiseBatch* b) { return (int)b->L.steps.size(); }
// One launch per step on st, its volumes' arguments read from dev (fy_noise_batch_pack's
// layout, already in device memory by stream order).
cudaError_t fy_noise_batch_launch(const NoiseBatch* b, const void* dev, cudaStream_t st) {
    const unsigned char* d = (const unsigned char*)dev;
    for (const auto& s : b->L.steps) {
        unsigned total = 0;
        for (unsigned g : s.gx) total += g;
        const void* packs = d;
        d += al256n(s.packs.size());
        const void* prefix = d;
        d += al256n((s.gx.size() + 1) * sizeof(unsigned));
        int nvol = b->L.cubes;
        cudaLaunchConfig_t c = {};
        c.gridDim = dim3(total, s.grid.y, 1);
        c.blockDim = s.block;
        c.dynamicSmemBytes = s.smem;
        c.stream = st;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        at[0].val.programmaticStreamSerializationAllowed = 1;
        c.attrs = at;
        c.numAttrs = 1;
        void* args[3] = {(void*)&packs, (void*)&prefix, (void*)&nvol};
        cudaError_t e = cudaLaunchKernelExC(&c, s.kern, args);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}
void fy_noise_batch_free(NoiseBatch* b) { delete b; }
// The statistics pass's parameters for one volume (box pass ZB_NOISE writing the guided
// (mean, var) pairs too), as noise_sequence forms them.
fyzb::Params fy_noise_stats_params(const float* in, int nz, int ny, int nx, int win, float* scratch, float* guided_mv) {
    const NoiseLayout Lay = noise_layout((size_t)nz * ny * nx);
    fyzb::Params sp{};
    sp.nz = nz; sp.ny = ny; sp.nx = nx;
    sp.f0 = in; sp.o0 = scratch + Lay.mean; sp.o1 = scratch + Lay.var; sp.o2 = guided_mv;
    sp.inv_wc = (float)(1.0 / ((double)win * win * win));
    sp.wci = win * win * win;
    return sp;
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

namespace {
// One thread copies a finished model into caller device memory laid out as fy_noise_model.
__global__ void k_noise_store(const NoiseCtl* __restrict__ ctl, fy_noise_model* __restrict__ m,
                              float* __restrict__ eps) {
    m->g = ctl->out_g;
    m->b = ctl->out_b;
    m->noise_ref = ctl->out_noise_ref;
    m->ref_intensity = ctl->out_ref_intensity;
    m->n_bins_used = ctl->out_used;
    if (eps) *eps = ctl->eps;
}
}  // namespace

cudaError_t fy_noise_store(const void* ctl_mem, void* d_model, float* d_eps, cudaStream_t st) {
    k_noise_store<<<1, 1, 0, st>>>((const NoiseCtl*)ctl_mem, (fy_noise_model*)d_model, d_eps);
    return cudaGetLastError();
}

// Test hook of the selection paths (see noise_force_radix): sets the forcing mask and returns
// the windows used since the previous call in *used. Synchronous.
cudaError_t fy_noise_test_paths(int force_radix, int* used) {
    int u = 0, zero = 0;
    cudaError_t e = cudaMemcpyFromSymbol(&u, noise_window_used, sizeof u);
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(noise_window_used, &zero, sizeof zero);
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(noise_force_radix, &force_radix, sizeof force_radix);
    if (e == cudaSuccess && used) *used = u;
    return e;
}

// Bounded waits of this unit's box passes that expired (see fy_zbox.cuh); 0 expected.
int fy_noise_wait_timeouts() { return fyzb::timeouts(); }
cudaError_t fy_noise_set_first_wait_polls(int polls) { return fyzb::set_first_wait_polls(polls); }
