// fy_dering.cu -- residual ring detection and removal (dering.c:78-248) on the GPU.
//
//   k_dering_accum   per (sector, radius) sums of nonzero u8 samples on an ss-stride
//                    (dering.c:78-116), exact integer arithmetic, shared-memory privatised.
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
// Grid: (x tiles of 256 samples, sampled rows * dz). Shared-memory histograms when the
// bin count fits, else global atomics.
template <bool SMEM>
__global__ void __launch_bounds__(256) k_dering_accum(const uint8_t* __restrict__ buf, const int* __restrict__ map,
                                                      unsigned long long* __restrict__ gsum,
                                                      unsigned int* __restrict__ gcnt, int nbins, long dz,
                                                      long dy, long dx, int ss, long sy, long sx,
                                                      int rows_per_cta) {
    extern __shared__ unsigned int sh[];
    unsigned int* ssum = sh;
    unsigned int* scnt = sh + nbins;
    if (SMEM) {
        for (int i = threadIdx.x; i < 2 * nbins; i += blockDim.x) sh[i] = 0;
        __syncthreads();
    }
    const long nrows = dz * sy;
    const long r0 = (long)blockIdx.y * rows_per_cta;
    for (long rr = r0; rr < r0 + rows_per_cta && rr < nrows; ++rr) {
        const long z = rr / sy, yi = rr - z * sy;
        const uint8_t* row = buf + ((size_t)z * dy + (size_t)(yi * ss)) * dx;
        const int* mrow = map + yi * sx;
        for (long xi = (long)blockIdx.x * blockDim.x + threadIdx.x; xi < sx; xi += (long)gridDim.x * blockDim.x) {
            const unsigned v = __ldg(row + xi * ss);
            if (!v) continue;                                   // masked voxels skipped
            const int b = __ldg(mrow + xi);
            if (b < 0) continue;
            if (SMEM) { atomicAdd(&ssum[b], v); atomicAdd(&scnt[b], 1u); }
            else { atomicAdd(&gsum[b], (unsigned long long)v); atomicAdd(&gcnt[b], 1u); }
        }
    }
    if (SMEM) {
        __syncthreads();
        for (int i = threadIdx.x; i < nbins; i += blockDim.x) {
            if (scnt[i]) {
                atomicAdd(&gsum[i], (unsigned long long)ssum[i]);
                atomicAdd(&gcnt[i], scnt[i]);
            }
        }
    }
}

// ---------------------------------------------------------------- finalize
// sum_f/cnt: float sums and counts exactly as the reference stores them (fy_dering.sum is
// float), so p = sum/cnt is the same IEEE float division.
//
// The reference sweeps radii in order and invalidates bin r when fewer than hw valid bins
// lie within +-hw, which later bins then see (dering.c:161-169). One block per (slab,
// sector): all radii are evaluated in parallel against the original validity; if no bin
// would be invalidated, that IS the sequential result (the first invalidation in the sweep
// would have been seen with unmodified validity). Otherwise one thread resumes the sweep
// sequentially from the first invalidated radius, which reproduces it exactly.
__global__ void __launch_bounds__(256) k_dering_smooth(const float* __restrict__ sum_f,
                                                       const unsigned int* __restrict__ cnt,
                                                       float* __restrict__ p, float* __restrict__ hp,
                                                       unsigned char* __restrict__ vd, int ns, int nr, int hw,
                                                       unsigned min_cnt) {
    extern __shared__ float sm_f[];
    float* sp = sm_f;                                  // p, hp and validity of this row in smem
    float* shp = sp + nr;
    unsigned char* svd = reinterpret_cast<unsigned char*>(shp + nr);
    __shared__ int s_first;
    const size_t off = (size_t)blockIdx.x * nr;       // (slab, sector) row
    if (threadIdx.x == 0) s_first = nr;
    for (int r = threadIdx.x; r < nr; r += blockDim.x) {
        const unsigned c = cnt[off + r];
        const unsigned char v = c >= min_cnt;
        svd[r] = v;
        sp[r] = v ? sum_f[off + r] / (float)c : 0.0f;
    }
    __syncthreads();
    for (int r = threadIdx.x; r < nr; r += blockDim.x) {
        shp[r] = 0.0f;
        if (!svd[r]) continue;
        double acc = 0;
        int c = 0;
        const int lo = r - hw < 0 ? 0 : r - hw, hi = r + hw >= nr ? nr - 1 : r + hw;
        for (int j = lo; j <= hi; ++j)
            if (svd[j]) { acc += sp[j]; ++c; }
        if (c >= hw) shp[r] = sp[r] - (float)(acc / c);
        else atomicMin(&s_first, r);
    }
    __syncthreads();
    if (threadIdx.x == 0 && s_first < nr) {           // sequential from the first change
        if (hw <= 8) {
            // the window's values are loaded together (independent loads), then summed in
            // the reference's order (ascending j)
            for (int r = s_first; r < nr; ++r) {
                if (!svd[r]) { shp[r] = 0.0f; continue; }
                const int lo = r - hw < 0 ? 0 : r - hw, hi = r + hw >= nr ? nr - 1 : r + hw;
                float wv[17];
                unsigned char wk[17];
#pragma unroll
                for (int q = 0; q < 17; ++q) {
                    const int j = lo + q;
                    const bool in = j <= hi;
                    wv[q] = in ? sp[j] : 0.0f;
                    wk[q] = in ? svd[j] : 0;
                }
                double acc = 0;
                int c = 0;
#pragma unroll
                for (int q = 0; q < 17; ++q)
                    if (wk[q]) { acc += wv[q]; ++c; }
                if (c >= hw) shp[r] = sp[r] - (float)(acc / c);
                else { shp[r] = 0.0f; svd[r] = 0; }
            }
        } else {
            for (int r = s_first; r < nr; ++r) {
                if (!svd[r]) { shp[r] = 0.0f; continue; }
                double acc = 0;
                int c = 0;
                const int lo = r - hw < 0 ? 0 : r - hw, hi = r + hw >= nr ? nr - 1 : r + hw;
                for (int j = lo; j <= hi; ++j)
                    if (svd[j]) { acc += sp[j]; ++c; }
                if (c >= hw) shp[r] = sp[r] - (float)(acc / c);
                else { shp[r] = 0.0f; svd[r] = 0; }
            }
        }
    }
    __syncthreads();
    for (int r = threadIdx.x; r < nr; r += blockDim.x) {
        p[off + r] = sp[r];
        hp[off + r] = shp[r];
        vd[off + r] = svd[r];
    }
}

__global__ void k_dering_vote(const float* __restrict__ hp, const unsigned char* __restrict__ vd,
                              float* __restrict__ ring, int nslab, int ns, int nr, float min_amp, float max_amp,
                              unsigned long long* __restrict__ detected) {
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
    const long sy = (dy + ss - 1) / ss, sx = (dx + ss - 1) / ss;
    const long nrows = dz * sy;
    if (nrows <= 0 || sx <= 0) return cudaSuccess;
    const int gx = (int)((sx + 255) / 256 < 4 ? (sx + 255) / 256 : 4);
    long want_ctas = (long)sms * 8 / gx;
    if (want_ctas < 1) want_ctas = 1;
    int rows_per_cta = (int)((nrows + want_ctas - 1) / want_ctas);
    if (rows_per_cta < 1) rows_per_cta = 1;
    dim3 grid(gx, (unsigned)((nrows + rows_per_cta - 1) / rows_per_cta));
    const size_t smem = 2 * (size_t)nbins * sizeof(unsigned int);
    if (smem <= 96 * 1024) {
        cudaError_t e = fy_smem_optin(k_dering_accum<true>, smem);
        if (e != cudaSuccess) return e;
        k_dering_accum<true><<<grid, 256, smem, st>>>(buf, map, sum, cnt, nbins, dz, dy, dx, ss, sy, sx, rows_per_cta);
    } else {
        k_dering_accum<false><<<grid, 256, 0, st>>>(buf, map, sum, cnt, nbins, dz, dy, dx, ss, sy, sx, rows_per_cta);
    }
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
    cudaError_t e = cudaMemsetAsync(detected, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
    const int hw = hp_win / 2;
    const size_t smem = (size_t)nr * (2 * sizeof(float) + 1);
    e = fy_smem_optin(k_dering_smooth, smem);
    if (e != cudaSuccess) return e;
    k_dering_smooth<<<nslab * ns, 256, smem, st>>>(sum_f, cnt, p, hp, vd, ns, nr, hw, min_cnt);
    const long nv = (long)nslab * nr;
    k_dering_vote<<<(unsigned)((nv + 127) / 128), 128, 0, st>>>(hp, vd, ring, nslab, ns, nr, (float)min_amp,
                                                                (float)max_amp, detected);
    k_dering_flag<<<1, 1, 0, st>>>(detected, have_rings);
    return cudaGetLastError();
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
