// fy_radial.cu -- the radial guided-eps model in FP64 on the device.
//
// The reference fits the flat-noise floor of its calibration sub-blocks against their
// distance from the rotation axis (pipeline.c:851-877): least squares fn(r) = a + b*r over
// up to 256 (r, floor) samples, kept only when n >= 8, b > 0, corr >= 0.5, fn(0) > 0 and
// fn(rmax)/fn(0) >= 1.3. The global eps is (k * median floor)^2 (pipeline.c:878-891), and a
// tile's eps is that times clamp((fn(r_tile)/median)^2, 0.4, 8) (pipeline.c:445-456).
// One CTA does the fit: the five sums run on one thread in the reference's order, and the
// median comes from a rank sort of the floors in shared memory.
#include "fy_context.h"

using fy::ctx;
using fy::fail;
using fy::fail_cuda;

namespace {

constexpr int kMaxSamples = 256;           // CMAX, pipeline.c:591

__global__ void __launch_bounds__(kMaxSamples) k_radial_fit(const double* __restrict__ rads,
                                                             const double* __restrict__ floors, int n,
                                                             double denoise_k, fy_radial_eps* __restrict__ out) {
    __shared__ double sf[kMaxSamples], sorted[kMaxSamples];
    const int t = threadIdx.x;
    if (t < n) sf[t] = floors[t];
    __syncthreads();
    if (t < n) {                            // rank sort: ties keep index order
        const double v = sf[t];
        int rank = 0;
        for (int j = 0; j < n; ++j) rank += (sf[j] < v) || (sf[j] == v && j < t);
        sorted[rank] = v;
    }
    __syncthreads();
    if (t != 0) return;
    fy_radial_eps r{};
    r.n = n;
    if (n >= 8) {                                                  // pipeline.c:857-876
        double sr = 0, sf2 = 0, srr = 0, srf = 0, sff = 0;
        for (int i = 0; i < n; ++i) {
            const double ri = rads[i], fi = sf[i];
            sr += ri; sf2 += fi;
            srr += ri * ri; srf += ri * fi; sff += fi * fi;
        }
        const double nn = n;
        const double den = nn * srr - sr * sr;
        if (den > 1e-9) {
            const double b = (nn * srf - sr * sf2) / den;
            const double a = (sf2 - b * sr) / nn;
            const double cden = sqrt((nn * srr - sr * sr) * (nn * sff - sf2 * sf2));
            const double corr = cden > 1e-12 ? (nn * srf - sr * sf2) / cden : 0;
            double rmax = 0;
            for (int i = 0; i < n; ++i) if (rads[i] > rmax) rmax = rads[i];
            const double f0 = a, f1 = a + b * rmax;
            r.a = a; r.b = b; r.corr = corr;
            r.have = (b > 0 && corr >= 0.5 && f0 > 0 && f1 / f0 >= 1.3) ? 1 : 0;
        }
    }
    // median_sorted (pipeline.c:74-78); 0.015 without samples (pipeline.c:878)
    r.median = n <= 0 ? 0.015 : ((n & 1) ? sorted[n / 2] : 0.5 * (sorted[n / 2 - 1] + sorted[n / 2]));
    if (denoise_k >= 0) {                                          // pipeline.c:888-891
        const double k = denoise_k > 0 ? denoise_k : 4.2;
        r.guided_eps = (k * r.median) * (k * r.median);
    }
    *out = r;
}

// Scale of a tile's eps (pipeline.c:447-456); 0 when the radial model is off.
FY_HD double radial_scale(const fy_radial_eps& f, double ecy, double ecx, long y0, long x0, long ty, long tx) {
    if (!f.have || f.median <= 0) return 0.0;
    const double ry = y0 + ty / 2.0 - ecy, rx = x0 + tx / 2.0 - ecx;
    const double fn = f.a + f.b * sqrt(ry * ry + rx * rx);
    const double s = fn / f.median;
    double s2 = s * s;
    if (s2 < 0.4) s2 = 0.4;
    if (s2 > 8.0) s2 = 8.0;
    return s2;
}

// eps for one cube: base (device float from the noise model, or the fixed host value) times
// the radial scale when the model is on (pipeline.c:292-293 takes the tile eps when > 0).
__global__ void k_radial_tile_eps(const fy_radial_eps* __restrict__ fit, const float* __restrict__ base_dev,
                                  float base_host, double ecy, double ecx, long y0, long x0, long ty, long tx,
                                  float* __restrict__ out) {
    const double base = base_dev ? (double)*base_dev : (double)base_host;
    const double s2 = radial_scale(*fit, ecy, ecx, y0, x0, ty, tx);
    *out = (float)(s2 > 0 ? base * s2 : base);
}

}  // namespace

cudaError_t fy_launch_radial_tile_eps(const fy_radial_eps* d_fit, const float* base_dev, float base_host, double ecy,
                                      double ecx, long y0, long x0, long ty, long tx, float* d_out, cudaStream_t st) {
    k_radial_tile_eps<<<1, 1, 0, st>>>(d_fit, base_dev, base_host, ecy, ecx, y0, x0, ty, tx, d_out);
    return cudaGetLastError();
}

extern "C" int fy_gpu_fit_radial_eps(const double* d_rads, const double* d_floors, int n, double denoise_k,
                                     fy_radial_eps* d_fit, void* stream) {
    fy::enter();
    const char* what = "fy_gpu_fit_radial_eps";
    if (!d_fit || (n > 0 && (!d_rads || !d_floors))) return fail(FY_EINVAL, "%s: null pointer", what);
    if (n < 0 || n > kMaxSamples) return fail(FY_EINVAL, "%s: n = %d outside [0, %d]", what, n, kMaxSamples);
    int rc = fy::ensure_ctx();
    if (rc) return rc;
    k_radial_fit<<<1, kMaxSamples, 0, (cudaStream_t)stream>>>(d_rads, d_floors, n, denoise_k, d_fit);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail_cuda(e, what);
    fy::count_launch(1);
    return FY_OK;
}

// Host form: stages the samples, fits on the device, returns the model (synchronous).
extern "C" int fy_fit_radial_eps(const double* rads, const double* floors, int n, double denoise_k,
                                 fy_radial_eps* out) {
    fy::enter();
    const char* what = "fy_fit_radial_eps";
    if (!out || (n > 0 && (!rads || !floors))) return fail(FY_EINVAL, "%s: null pointer", what);
    if (n < 0 || n > kMaxSamples) return fail(FY_EINVAL, "%s: n = %d outside [0, %d]", what, n, kMaxSamples);
    int rc = fy::ensure_ctx();
    if (rc) return rc;
    fy::ThreadCtx& c = ctx();
    cudaStream_t st = c.st;
    const size_t in_bytes = 2 * kMaxSamples * sizeof(double);
    cudaError_t e;
    fy::ws_acquire(st);
    if ((e = c.small.ensure(in_bytes + sizeof(fy_radial_eps) + 256)) != cudaSuccess) return fail_cuda(e, what);
    if ((e = c.pin.ensure(sizeof(fy_radial_eps))) != cudaSuccess) return fail_cuda(e, what);
    double* d_r = (double*)c.small.p;
    double* d_f = d_r + kMaxSamples;
    fy_radial_eps* d_fit = (fy_radial_eps*)((char*)c.small.p + in_bytes);
    if (n > 0) {
        if ((e = cudaMemcpyAsync(d_r, rads, n * sizeof(double), cudaMemcpyHostToDevice, st)) != cudaSuccess)
            return fail_cuda(e, what);
        if ((e = cudaMemcpyAsync(d_f, floors, n * sizeof(double), cudaMemcpyHostToDevice, st)) != cudaSuccess)
            return fail_cuda(e, what);
    }
    k_radial_fit<<<1, kMaxSamples, 0, st>>>(d_r, d_f, n, denoise_k, d_fit);
    if ((e = cudaGetLastError()) != cudaSuccess) return fail_cuda(e, what);
    fy::count_launch(1);
    if ((e = cudaMemcpyAsync(c.pin.p, d_fit, sizeof(fy_radial_eps), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return fail_cuda(e, what);
    fy::ws_release(st);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return fail_cuda(e, what);
    *out = *(const fy_radial_eps*)c.pin.p;
    return FY_OK;
}

// Host scalar form of the per-tile eps (pipeline.c:447-456): 0 means "use the global eps".
extern "C" double fy_radial_tile_eps(const fy_radial_eps* fit, double guided_eps, double ecy, double ecx, long y0,
                                     long x0, long ty, long tx) {
    if (!fit || guided_eps <= 0) return 0.0;
    const double s2 = radial_scale(*fit, ecy, ecx, y0, x0, ty, tx);
    return s2 > 0 ? guided_eps * s2 : 0.0;
}
