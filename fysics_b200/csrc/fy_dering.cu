// fy_dering.cu -- residual ring detection and removal (dering.c:78-248) on the GPU.
//
//   k_dering_accum   per (sector, radius) sums of nonzero u8 samples on an ss-stride
//                    (dering.c:78-116), exact integer arithmetic, summed along z per
//                    sampled column before one atomic per column and z range.
//                    The (y,x) -> sector*nr + radius map is built on the host with the
//                    reference's own double-precision sqrt/atan2 formula (dering.c:89-99)
//                    so every sample lands in the same bin.
//   k_dering_smooth  per (slab, sector): mean profile p = sum/cnt over bins with
//                    cnt >= min_cnt, radial high-pass hp = p - mean over valid bins within
//                    +-hw, in radius order because a bin with too few valid neighbours is
//                    invalidated for the bins after it (dering.c:151-170)
//   k_dering_vote    per (slab, radius): sector sign-consistency vote, median, clamp
//                    (dering.c:171-189)
//   k_dering_apply   f = max(f - scale*ring[slab][r(y,x)], 0) for f > 0 (dering.c:200-248),
//                    one thread per (y,x) column walking a chunk of 32 planes.
#include "fy_internal.h"

namespace {

// ---------------------------------------------------------------- accumulate
// The bin of a sample depends on its (y, x) only, so a thread owns one sampled column
// (yi, xi) and a range of z planes: it sums the column's samples and counts the nonzero
// ones (zero samples add nothing to either), then adds both to the column's bin with one
// pair of global atomics. Integer arithmetic throughout, so the totals equal the
// per-sample accumulation exactly. Consecutive threads take consecutive xi of a row, and
// each thread has 8 loads in flight.
__global__ void __launch_bounds__(256) k_dering_accum(const uint8_t* __restrict__ buf, const int* __restrict__ map,
                                                      unsigned long long* __restrict__ gsum,
                                                      unsigned int* __restrict__ gcnt, long dz, long dy, long dx,
                                                      int ss, long sy, long sx, long zchunk) {
    const long ncol = sy * sx;
    const long col = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= ncol) return;
    const long yi = col / sx, xi = col - yi * sx;
    const int b = __ldg(map + col);
    if (b < 0) return;
    const long z0 = (long)blockIdx.y * zchunk;
    const long z1 = z0 + zchunk < dz ? z0 + zchunk : dz;
    const size_t zs = (size_t)dy * dx;
    const uint8_t* p = buf + (size_t)z0 * zs + (size_t)(yi * ss) * dx + (size_t)xi * ss;
    unsigned int s = 0, c = 0;
    long z = z0;
    for (; z + 8 <= z1; z += 8, p += 8 * zs) {
        unsigned int v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) v[u] = __ldg(p + (size_t)u * zs);
#pragma unroll
        for (int u = 0; u < 8; ++u) { s += v[u]; c += v[u] != 0u; }
    }
    for (; z < z1; ++z, p += zs) {
        const unsigned int v = __ldg(p);
        s += v;
        c += v != 0u;
    }
    if (c) {
        atomicAdd(&gsum[b], (unsigned long long)s);
        atomicAdd(&gcnt[b], c);
    }
}

// ---------------------------------------------------------------- finalize
// sum_f/cnt: float sums and counts exactly as the reference stores them (fy_dering.sum is
// float), so p = sum/cnt is the same IEEE float division.
//
// The reference sweeps radii in order and invalidates bin r when fewer than hw valid bins
// lie within +-hw, which later bins then see (dering.c:161-169). At step r the window's bins
// below r carry their final validity and the bins from r up their original one, and only
// the COUNT of valid bins decides an invalidation. So one thread first runs the sweep on
// counts alone (a running count, O(1) per radius), and then every radius forms its window
// mean in parallel, in the reference's order (ascending j, FP64), over exactly the bins the
// sequential sweep would have seen. One block per (slab, sector).
__global__ void __launch_bounds__(256) k_dering_smooth(const float* __restrict__ sum_f,
                                                       const unsigned int* __restrict__ cnt,
                                                       float* __restrict__ p, float* __restrict__ hp,
                                                       unsigned char* __restrict__ vd, int ns, int nr, int hw,
                                                       unsigned min_cnt, unsigned long long* __restrict__ detected) {
    fy_pdl_wait();
    if (blockIdx.x == 0 && threadIdx.x == 0) *detected = 0;   // the vote counts after this kernel
    extern __shared__ float sm_f[];
    float* sp = sm_f;                                  // p, hp and validity of this row in smem
    float* shp = sp + nr;
    unsigned char* svo = reinterpret_cast<unsigned char*>(shp + nr);   // original validity
    unsigned char* svf = svo + nr;                                     // after the sweep
    const size_t off = (size_t)blockIdx.x * nr;       // (slab, sector) row
    for (int r = threadIdx.x; r < nr; r += blockDim.x) {
        const unsigned c = cnt[off + r];
        const unsigned char v = c >= min_cnt;
        svo[r] = v;
        sp[r] = v ? sum_f[off + r] / (float)c : 0.0f;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        // cf = final-valid bins in [r - hw, r - 1], co = originally valid bins in [r, r + hw]
        int cf = 0, co = 0;
        for (int j = 0; j <= hw && j < nr; ++j) co += svo[j];
        for (int r = 0; r < nr; ++r) {
            unsigned char f = 0;
            if (svo[r]) f = cf + co >= hw;
            svf[r] = f;
            cf += f;
            if (r - hw >= 0) cf -= svf[r - hw];
            co -= svo[r];
            if (r + 1 + hw < nr) co += svo[r + 1 + hw];
        }
    }
    __syncthreads();
    for (int r = threadIdx.x; r < nr; r += blockDim.x) {
        float h = 0.0f;
        if (svf[r]) {
            double acc = 0;
            int c = 0;
            const int lo = r - hw < 0 ? 0 : r - hw, hi = r + hw >= nr ? nr - 1 : r + hw;
            for (int j = lo; j <= hi; ++j)
                if (j < r ? svf[j] : svo[j]) { acc += sp[j]; ++c; }
            h = sp[r] - (float)(acc / c);
        }
        p[off + r] = sp[r];
        hp[off + r] = h;
        vd[off + r] = svf[r];
    }
}

__global__ void k_dering_vote(const float* __restrict__ hp, const unsigned char* __restrict__ vd,
                              float* __restrict__ ring, int nslab, int ns, int nr, float min_amp, float max_amp,
                              unsigned long long* __restrict__ detected) {
    fy_pdl_wait();
    const long id = (long)blockIdx.x * blockDim.x + threadIdx.x;   // (slab, radius)
    if (id >= (long)nslab * nr) return;
    const int s = (int)(id / nr), r = (int)(id % nr);
    float med[64];
    int nv = 0, pos = 0, neg = 0;
    for (int q = 0; q < ns && q < 64; ++q) {
        const size_t i = ((size_t)s * ns + q) * nr + r;
        if (!vd[i]) continue;
        const float v = hp[i];
        med[nv++] = v;
        if (v > 0) ++pos; else if (v < 0) ++neg;
    }
    float out = 0.0f;
    if (!(nv < ns - 2 || (pos && neg))) {
        for (int i = 1; i < nv; ++i) {                           // ascending sort
            const float k = med[i];
            int j = i - 1;
            while (j >= 0 && med[j] > k) { med[j + 1] = med[j]; --j; }
            med[j + 1] = k;
        }
        float m = (nv & 1) ? med[nv / 2] : 0.5f * (med[nv / 2 - 1] + med[nv / 2]);
        if (!(fabsf(m) < min_amp)) {
            if (m > max_amp) m = max_amp;
            if (m < -max_amp) m = -max_amp;
            out = m;
            atomicAdd(detected, 1ull);
        }
    }
    ring[(size_t)s * nr + r] = out;
}

// detected -> have_rings (dering.c:192)
__global__ void k_dering_flag(const unsigned long long* detected, int* have_rings) {
    fy_pdl_wait();
    *have_rings = *detected >= 2;
}

// ---------------------------------------------------------------- apply
__global__ void __launch_bounds__(256) k_dering_apply(float* __restrict__ f, const float* __restrict__ ring,
                                                      const int* __restrict__ have_rings, int nslab, int nr,
                                                      int slab_z, double cy, double cx, long z0, long y0,
                                                      long x0, long dz, long dy, long dx, float sc) {
    if (have_rings && !*have_rings) return;                    // dering.c:202
    const long x = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long y = blockIdx.y;
    const long zc = (dz + gridDim.z - 1) / gridDim.z;
    const long zb = (long)blockIdx.z * zc, zend = zb + zc < dz ? zb + zc : dz;
    if (x >= dx) return;
    const double gy = (double)(y0 + y) - cy, gx = (double)(x0 + x) - cx;
    const int ri = (int)(sqrt(gy * gy + gx * gx) + 0.5);
    if (ri >= nr) return;
    const size_t zs = (size_t)dy * dx;
    float* col = f + (size_t)y * dx + x;
    for (long z = zb; z < zend; z += 4) {
        float v[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) v[k] = (z + k < zend) ? col[(size_t)(z + k) * zs] : 0.0f;   // 4 loads in flight
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (z + k >= zend || v[k] <= 0.0f) continue;   // masked voxels untouched
            long s = (z0 + z + k) / slab_z;
            if (s < 0) s = 0;
            if (s >= nslab) s = nslab - 1;
            const float w = v[k] - sc * __ldg(ring + (size_t)s * nr + ri);
            col[(size_t)(z + k) * zs] = w > 0.0f ? w : 0.0f;
        }
    }
}

}  // namespace

cudaError_t fy_launch_dering_accum(const uint8_t* buf, const int* map, unsigned long long* sum, unsigned int* cnt,
                                   int nbins, long dz, long dy, long dx, int ss, int sms, cudaStream_t st) {
    (void)nbins;
    const long sy = (dy + ss - 1) / ss, sx = (dx + ss - 1) / ss;
    const long ncol = sy * sx;
    if (dz <= 0 || ncol <= 0) return cudaSuccess;
    // z chunks: about one full wave of threads, each column sum at most 255 * zchunk < 2^32
    long nchunk = ((long)sms * 2048 + ncol - 1) / ncol;
    if (nchunk > dz) nchunk = dz;
    if (nchunk > 65535) nchunk = 65535;
    if (nchunk < 1) nchunk = 1;
    const long zchunk = (dz + nchunk - 1) / nchunk;
    const dim3 grid((unsigned)((ncol + 255) / 256), (unsigned)((dz + zchunk - 1) / zchunk));
    k_dering_accum<<<grid, 256, 0, st>>>(buf, map, sum, cnt, dz, dy, dx, ss, sy, sx, zchunk);
    return cudaGetLastError();
}

// scratch: p, hp (floats) and vd (bytes) of nslab*ns*nr each
cudaError_t fy_launch_dering_finalize(const float* sum_f, const unsigned int* cnt, float* ring, void* scratch,
                                      unsigned long long* detected, int* have_rings, int nslab, int ns, int nr,
                                      int hp_win, unsigned min_cnt, double min_amp, double max_amp,
                                      cudaStream_t st) {
    const size_t nb = (size_t)nslab * ns * nr;
    float* p = (float*)scratch;
    float* hp = p + nb;
    unsigned char* vd = (unsigned char*)(hp + nb);
    const int hw = hp_win / 2;
    const size_t smem = (size_t)nr * (2 * sizeof(float) + 2);
    cudaError_t e = fy_smem_optin(k_dering_smooth, smem);
    if (e != cudaSuccess) return e;
    // the smoothing also zeroes the detected count (block 0), which the vote then adds to;
    // the three run as programmatic dependent launches
    if ((e = fy_launch_pdl(k_dering_smooth, dim3(nslab * ns), dim3(256), smem, st, sum_f, cnt, p, hp, vd, ns, nr, hw,
                           min_cnt, detected)) != cudaSuccess)
        return e;
    const long nv = (long)nslab * nr;
    if ((e = fy_launch_pdl(k_dering_vote, dim3((unsigned)((nv + 127) / 128)), dim3(128), 0, st, hp, vd, ring, nslab, ns,
                           nr, (float)min_amp, (float)max_amp, detected)) != cudaSuccess)
        return e;
    return fy_launch_pdl(k_dering_flag, dim3(1), dim3(1), 0, st, detected, have_rings);
}

size_t fy_dering_finalize_scratch(int nslab, int ns, int nr) {
    const size_t nb = (size_t)nslab * ns * nr;
    return nb * (2 * sizeof(float) + 1);
}

cudaError_t fy_launch_dering_apply(float* f, const float* ring, const int* have_rings, int nslab, int nr,
                                   int slab_z, double cy, double cx, long z0, long y0, long x0, long dz, long dy,
                                   long dx, double scale, cudaStream_t st) {
    if (dz <= 0 || dy <= 0 || dx <= 0) return cudaSuccess;
    dim3 grid((unsigned)((dx + 255) / 256), (unsigned)dy, (unsigned)((dz + 31) / 32));
    k_dering_apply<<<grid, 256, 0, st>>>(f, ring, have_rings, nslab, nr, slab_z, cy, cx, z0, y0, x0, dz, dy, dx,
                                         (float)scale);
    return cudaGetLastError();
}
