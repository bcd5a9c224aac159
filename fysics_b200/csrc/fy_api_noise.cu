// fy_api_noise.cu -- C-ABI fy_estimate_noise (noise.c:75-192) and its device form.
#include "fy_context.h"

using fy::ctx;
using fy::fail;
using fy::fail_cuda;

namespace {
int check_args(int nz, int ny, int nx, int& win, double& flat_pct, const char* what) {
    if (nz < 1 || ny < 1 || nx < 1) return fail(FY_EINVAL, "%s: bad dims", what);
    if (win < 3) win = 5;                                       // noise.c:79-80
    if (flat_pct <= 0) flat_pct = 10.0;
    if (win / 2 > 4) return fail(FY_EUNSUPPORTED, "%s: win %d > 9 not supported", what, win);
    return FY_OK;
}

// Pinned staging for the 40-byte model readback.
struct ModelHost { double g, b, noise_ref, ref_intensity; int used; };
}  // namespace

extern "C" int fy_estimate_noise(const float* in, int nz, int ny, int nx, int win, double flat_pct,
                                 double ref_intensity, fy_noise_model* out) {
    fy::enter();
    const char* what = "fy_estimate_noise";
    if (!out) return fail(FY_EINVAL, "%s: null model", what);     // noise.c:78
    if (!in) return fail(FY_EINVAL, "%s: null input", what);
    int rc = check_args(nz, ny, nx, win, flat_pct, what);
    if (rc) return rc;
    if ((rc = fy::ensure_ctx())) return rc;
    fy::ThreadCtx& c = ctx();
    cudaStream_t st = c.st;
    const size_t n = (size_t)nz * ny * nx;
    fy::ws_acquire(st);
    cudaError_t e;
    if ((e = c.vin.ensure(n * sizeof(float))) != cudaSuccess) return fail_cuda(e, what);
    if ((e = c.aux.ensure(fy_noise_scratch_floats(n) * sizeof(float))) != cudaSuccess) return fail_cuda(e, what);
    if ((e = c.small.ensure(fy_noise_ctl_bytes())) != cudaSuccess) return fail_cuda(e, what);
    if ((e = c.pin.ensure(sizeof(ModelHost))) != cudaSuccess) return fail_cuda(e, what);
    if ((e = cudaMemcpyAsync(c.vin.p, in, n * sizeof(float), cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return fail_cuda(e, what);
    int launches = 0;
    if ((e = fy_launch_estimate_noise(c.vin.as<float>(), nz, ny, nx, win, flat_pct, ref_intensity,
                                      c.aux.as<float>(), c.small.p, c.sms, st, launches)) != cudaSuccess)
        return fail_cuda(e, what);
    fy::count_launch(launches);
    ModelHost* mh = (ModelHost*)c.pin.p;
    if ((e = fy_noise_read(c.small.p, &mh->g, &mh->b, &mh->noise_ref, &mh->ref_intensity, &mh->used, st)) !=
        cudaSuccess)
        return fail_cuda(e, what);
    fy::ws_release(st);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return fail_cuda(e, what);
    out->g = mh->g;
    out->b = mh->b;
    out->noise_ref = mh->noise_ref;
    out->ref_intensity = mh->ref_intensity;
    out->n_bins_used = mh->used;
    return FY_OK;
}

// Device form. Scratch: fy_gpu_noise_scratch_bytes(). The model stays in device memory
// (d_ctl); fy_gpu_noise_model() copies it out, fy_gpu_noise_eps() gives the device address
// of the guided eps float so a chained filter needs no host round trip.
extern "C" size_t fy_gpu_noise_scratch_bytes(int nz, int ny, int nx) {
    return fy_noise_scratch_floats((size_t)nz * ny * nx) * sizeof(float) + fy_noise_ctl_bytes();
}
extern "C" int fy_gpu_estimate_noise(const float* d_in, int nz, int ny, int nx, int win, double flat_pct,
                                     double ref_intensity, void* d_scratch, void* stream) {
    fy::enter();
    const char* what = "fy_gpu_estimate_noise";
    if (!d_in || !d_scratch) return fail(FY_EINVAL, "%s: null pointer", what);
    int rc = check_args(nz, ny, nx, win, flat_pct, what);
    if (rc) return rc;
    if ((rc = fy::ensure_ctx())) return rc;
    const size_t n = (size_t)nz * ny * nx;
    float* stats = (float*)d_scratch;
    void* ctl = (char*)d_scratch + fy_noise_scratch_floats(n) * sizeof(float);
    int launches = 0;
    cudaError_t e = fy_launch_estimate_noise(d_in, nz, ny, nx, win, flat_pct, ref_intensity, stats, ctl,
                                             ctx().sms, (cudaStream_t)stream, launches);
    if (e != cudaSuccess) return fail_cuda(e, what);
    fy::count_launch(launches);
    return FY_OK;
}
extern "C" int fy_gpu_noise_model(const void* d_scratch, int nz, int ny, int nx, fy_noise_model* out,
                                  void* stream) {
    fy::enter();
    if (!d_scratch || !out) return fail(FY_EINVAL, "fy_gpu_noise_model: null pointer");
    int rc = fy::ensure_ctx();
    if (rc) return rc;
    fy::ThreadCtx& c = ctx();
    cudaError_t e = c.pin.ensure(sizeof(ModelHost));
    if (e != cudaSuccess) return fail_cuda(e, "fy_gpu_noise_model");
    const void* ctl = (const char*)d_scratch + fy_noise_scratch_floats((size_t)nz * ny * nx) * sizeof(float);
    ModelHost* mh = (ModelHost*)c.pin.p;
    cudaStream_t st = (cudaStream_t)stream;
    if ((e = fy_noise_read(ctl, &mh->g, &mh->b, &mh->noise_ref, &mh->ref_intensity, &mh->used, st)) != cudaSuccess)
        return fail_cuda(e, "fy_gpu_noise_model");
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return fail_cuda(e, "fy_gpu_noise_model");
    out->g = mh->g; out->b = mh->b; out->noise_ref = mh->noise_ref;
    out->ref_intensity = mh->ref_intensity; out->n_bins_used = mh->used;
    return FY_OK;
}
extern "C" const float* fy_gpu_noise_eps(const void* d_scratch, int nz, int ny, int nx) {
    return fy_noise_eps_ptr((const char*)d_scratch + fy_noise_scratch_floats((size_t)nz * ny * nx) * sizeof(float));
}
