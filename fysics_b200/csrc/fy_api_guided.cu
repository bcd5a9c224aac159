// fy_api_guided.cu -- C-ABI guided filter and box mean (guided.c:100-241) plus the
// fy_gpu_guided device form.
#include "fy_context.h"

using fy::ctx;
using fy::fail;
using fy::fail_cuda;

namespace {

// Enqueue an exact (s <= 1) or fast (s >= 2) guided filter on device buffers. `scratch`
// must hold guided_scratch_floats(); in == out is allowed.
size_t guided_scratch_floats(int nz, int ny, int nx, int radius, int s) {
    const size_t n = (size_t)nz * ny * nx;
    if (radius < 1) radius = 2;
    if (s > 1) {
        const int lz = (nz + s - 1) / s, ly = (ny + s - 1) / s, lx = (nx + s - 1) / s;
        if (lz >= 2 && ly >= 2 && lx >= 2) {
            int rl = radius / s; if (rl < 1) rl = 1;
            if (rl <= 4) return fy_guided_fast_scratch_floats(lz, ly, lx);
            return 3 * (size_t)lz * ly * lx + 4 * (size_t)lz * ly * lx;
        }
    }
    return radius <= 4 ? fy_guided_fused_scratch_floats(n) : 4 * n;   // exact: a, b fields; generic: 4n
}

int enqueue_guided(const float* in, float* out, float* scratch, int nz, int ny, int nx, int radius,
                   double eps, int s, cudaStream_t st, const char* what) {
    fy::ThreadCtx& c = ctx();
    if (radius < 1) radius = 2;                                    // guided.c:115
    const float epsf = (float)eps;
    int launches = 0;
    cudaError_t e = cudaSuccess;
    bool fast = false;
    int lz = 0, ly = 0, lx = 0;
    if (s > 1) {                                                   // guided.c:155-158
        lz = (nz + s - 1) / s; ly = (ny + s - 1) / s; lx = (nx + s - 1) / s;
        fast = lz >= 2 && ly >= 2 && lx >= 2;
    }
    if (fast) {
        int rl = radius / s; if (rl < 1) rl = 1;
        if (rl <= 4) {
            e = fy_launch_guided_fast(in, out, scratch, nz, ny, nx, radius, epsf, s, c.sms, st, launches);
        } else {
            return fail(FY_EUNSUPPORTED, "%s: fast path low-grid radius %d > 4", what, rl);
        }
    } else if (radius <= 4) {
        e = fy_launch_guided_fused(in, out, nullptr, scratch, nz, ny, nx, radius, epsf, 0, c.sms, st);
        launches = 2;
    } else {
        e = fy_launch_guided_generic(in, out, scratch, nz, ny, nx, radius, epsf, st, launches);
    }
    if (e != cudaSuccess) return fail_cuda(e, what);
    fy::count_launch(launches);
    return FY_OK;
}

int host_guided(const float* in, float* out, int nz, int ny, int nx, int radius, double eps, int s,
                const char* what) {
    if (!in || !out) return fail(FY_EINVAL, "%s: null pointer", what);
    if (nz < 1 || ny < 1 || nx < 1) return fail(FY_EINVAL, "%s: bad dims", what);
    int rc = fy::ensure_ctx();
    if (rc) return rc;
    fy::ThreadCtx& c = ctx();
    cudaStream_t st = c.st;
    const size_t n = (size_t)nz * ny * nx;
    fy::ws_acquire(st);
    cudaError_t e;
    if ((e = c.vin.ensure(n * sizeof(float))) != cudaSuccess) return fail_cuda(e, what);
    if ((e = c.vout.ensure(n * sizeof(float))) != cudaSuccess) return fail_cuda(e, what);
    if ((e = c.aux.ensure(guided_scratch_floats(nz, ny, nx, radius, s) * sizeof(float))) != cudaSuccess)
        return fail_cuda(e, what);
    if ((e = cudaMemcpyAsync(c.vin.p, in, n * sizeof(float), cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return fail_cuda(e, what);
    if ((rc = enqueue_guided(c.vin.as<float>(), c.vout.as<float>(), c.aux.as<float>(), nz, ny, nx, radius, eps,
                             s, st, what)))
        return rc;
    if ((e = cudaMemcpyAsync(out, c.vout.p, n * sizeof(float), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return fail_cuda(e, what);
    fy::ws_release(st);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return fail_cuda(e, what);
    return FY_OK;
}
}  // namespace

extern "C" size_t fy_guided_ws_floats(int nz, int ny, int nx) { return (size_t)4 * nz * ny * nx; }

// The caller's ws (a host buffer of fy_guided_ws_floats floats, guided.c:140) is accepted
// for signature compatibility; the GPU path keeps its own device workspace.
extern "C" int fy_guided_denoise_ws(const float* in, float* out, int nz, int ny, int nx, int radius,
                                    double eps, float* ws) {
    fy::enter();
    (void)ws;
    return host_guided(in, out, nz, ny, nx, radius, eps, 1, "fy_guided_denoise_ws");
}
extern "C" int fy_guided_denoise(const float* in, float* out, int nz, int ny, int nx, int radius, double eps) {
    fy::enter();
    return host_guided(in, out, nz, ny, nx, radius, eps, 1, "fy_guided_denoise");
}
extern "C" int fy_guided_denoise_fast_ws(const float* in, float* out, int nz, int ny, int nx, int radius,
                                         double eps, int s, float* ws) {
    fy::enter();
    (void)ws;
    return host_guided(in, out, nz, ny, nx, radius, eps, s, "fy_guided_denoise_fast_ws");
}

// noise.c:197-202 (plan-time scalar)
extern "C" double fy_guided_eps_for_noise(double noise_ref) {
    const double k = 3.0;
    double eps = (k * noise_ref) * (k * noise_ref);
    if (!(eps > 1e-8)) eps = 1e-8;
    return eps;
}

// guided.c:104-106: one separable box mean; tmp is the caller's n-float host scratch
// (accepted for compatibility); in/out may alias.
extern "C" void fy_box_smooth(const float* in, float* out, float* tmp, int nz, int ny, int nx, int r) {
    fy::enter();
    (void)tmp;
    const char* what = "fy_box_smooth";
    if (!in || !out) { fail(FY_EINVAL, "%s: null pointer", what); return; }
    if (nz < 1 || ny < 1 || nx < 1) { fail(FY_EINVAL, "%s: bad dims", what); return; }
    if (fy::ensure_ctx()) return;
    fy::ThreadCtx& c = ctx();
    cudaStream_t st = c.st;
    const size_t n = (size_t)nz * ny * nx;
    fy::ws_acquire(st);
    cudaError_t e;
    if ((e = c.vin.ensure(n * sizeof(float))) != cudaSuccess) { fail_cuda(e, what); return; }
    if ((e = c.vout.ensure(n * sizeof(float))) != cudaSuccess) { fail_cuda(e, what); return; }
    if ((e = c.aux.ensure(n * sizeof(float))) != cudaSuccess) { fail_cuda(e, what); return; }
    if ((e = cudaMemcpyAsync(c.vin.p, in, n * sizeof(float), cudaMemcpyHostToDevice, st)) != cudaSuccess) {
        fail_cuda(e, what); return;
    }
    int launches = 0;
    if ((e = fy_launch_box_mean(c.vin.as<float>(), c.vout.as<float>(), c.aux.as<float>(), nz, ny, nx, r, st,
                                launches)) != cudaSuccess) { fail_cuda(e, what); return; }
    fy::count_launch(launches);
    if ((e = cudaMemcpyAsync(out, c.vout.p, n * sizeof(float), cudaMemcpyDeviceToHost, st)) != cudaSuccess) {
        fail_cuda(e, what); return;
    }
    fy::ws_release(st);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) fail_cuda(e, what);
}

// Device form: s <= 1 exact (fy_guided_denoise_ws), s >= 2 fast (fy_guided_denoise_fast_ws).
extern "C" size_t fy_gpu_guided_scratch_bytes(int nz, int ny, int nx, int radius, int s) {
    return guided_scratch_floats(nz, ny, nx, radius, s) * sizeof(float);
}
extern "C" int fy_gpu_guided(const float* d_in, float* d_out, int nz, int ny, int nx, int radius, double eps,
                             int s, void* stream) {
    fy::enter();
    const char* what = "fy_gpu_guided";
    if (!d_in || !d_out) return fail(FY_EINVAL, "%s: null pointer", what);
    if (nz < 1 || ny < 1 || nx < 1) return fail(FY_EINVAL, "%s: bad dims", what);
    int rc = fy::ensure_ctx();
    if (rc) return rc;
    fy::ThreadCtx& c = ctx();
    cudaStream_t st = (cudaStream_t)stream;
    fy::ws_acquire(st);
    cudaError_t e = c.aux.ensure(guided_scratch_floats(nz, ny, nx, radius, s) * sizeof(float));
    if (e != cudaSuccess) return fail_cuda(e, what);
    rc = enqueue_guided(d_in, d_out, c.aux.as<float>(), nz, ny, nx, radius, eps, s, st, what);
    fy::ws_release(st);
    return rc;
}
