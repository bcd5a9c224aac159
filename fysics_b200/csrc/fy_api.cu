// fy_api.cu -- C-ABI drop-in entry points (fysics.h signatures) for sizes, windowing,
// transfer functions and the Wiener deconvolution, plus their fy_gpu_* device forms.
//
// Host-pointer entry points copy the caller's buffers to the thread's device workspace,
// run the kernels on the thread's stream and copy the result back before returning, so
// their contract is the reference's synchronous one.
#include <math.h>
#include <string.h>
#include <vector>

#include "fy_context.h"

using fy::ctx;
using fy::fail;
using fy::fail_cuda;

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

// ============================================================== sizes (fft.c:25-38)
extern "C" int fy_is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }
extern "C" int fy_next_pow2(int n) {
    int p = 1;
    while (p < n) p <<= 1;
    return p;
}
extern "C" int fy_next_fft_size(int n) {
    const int p2 = fy_next_pow2(n);
    const int p3 = 3 * fy_next_pow2((n + 2) / 3);
    return (p3 >= n && p3 < p2) ? p3 : p2;
}

// ============================================================== transfers (paganin.c:15-91)
extern "C" double fy_paganin_transfer(double f, const fy_physics* p) {
    const double lam = 1.23984199e-3 / p->energy_kev;       // micron
    const double dist = p->distance_mm * 1000.0;             // micron
    double px = p->pixel_um;
    if (px > 0.0 && px < 0.1) px *= 1000.0;                  // mm passed by mistake
    const double fu = f / px;
    return 1.0 / (1.0 + p->delta_beta * lam * dist * M_PI * (fu * fu));
}
extern "C" double fy_unsharp_transfer(double f, const fy_physics* p) {
    if (p->unsharp_coeff == 0.0 || p->unsharp_sigma == 0.0) return 1.0;
    const double s = p->unsharp_sigma;
    return 1.0 + p->unsharp_coeff * (1.0 - exp(-2.0 * M_PI * M_PI * s * s * f * f));
}
extern "C" double fy_recon_transfer(double f, const fy_physics* p) {
    const double h = fy_paganin_transfer(f, p) * fy_unsharp_transfer(f, p);
    return h < 1e-4 ? 1e-4 : h;
}
extern "C" double fy_auto_reg(const fy_physics* p, double base) {
    (void)p;
    return base > 0.0 ? base : 0.015;
}
extern "C" double fy_auto_deltabeta_scale(const fy_physics* p) {
    const double h = fy_paganin_transfer(0.5, p);
    if (!isfinite(h) || h <= 0) return 1.0;
    const double lo = 0.0025, hi = 0.0070, s_lo = 0.35;
    if (h <= lo) return s_lo;
    if (h >= hi) return 1.0;
    return s_lo + (h - lo) / (hi - lo) * (1.0 - s_lo);
}

// ============================================================== windowing (stream.c:27-63)
namespace {

// Run an elementwise host->host conversion on the GPU: H2D, kernel, D2H, sync.
template <class Tin, class Tout, class Launch>
int host_elementwise(const Tin* in, Tout* out, size_t n, Launch launch, const char* what) {
    if (!n) return FY_OK;
    if (!in || !out) return fail(FY_EINVAL, "%s: null pointer", what);
    int rc = fy::ensure_ctx();
    if (rc) return rc;
    fy::ThreadCtx& c = ctx();
    cudaStream_t st = c.st;
    fy::ws_acquire(st);
    cudaError_t e;
    if ((e = c.vin.ensure(n * sizeof(Tin))) != cudaSuccess) return fail_cuda(e, what);
    if ((e = c.vout.ensure(n * sizeof(Tout))) != cudaSuccess) return fail_cuda(e, what);
    if ((e = cudaMemcpyAsync(c.vin.p, in, n * sizeof(Tin), cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return fail_cuda(e, what);
    if ((e = launch(c.vin.as<Tin>(), c.vout.as<Tout>(), st)) != cudaSuccess) return fail_cuda(e, what);
    fy::count_launch();
    if ((e = cudaMemcpyAsync(out, c.vout.p, n * sizeof(Tout), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return fail_cuda(e, what);
    fy::ws_release(st);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return fail_cuda(e, what);
    return FY_OK;
}

inline void dewindow_params(double f32_min, double f32_max, float& lo, float& scale) {
    lo = (float)f32_min;                                  // stream.c:43-44
    scale = (float)((f32_max - f32_min) / 255.0);
}
inline void rewindow_params(double f32_min, double f32_max, float& lo, float& inv) {
    const double span = f32_max - f32_min;               // stream.c:50-52
    inv = (span != 0.0) ? (float)(255.0 / span) : 0.0f;
    lo = (float)f32_min;
}
}  // namespace

extern "C" void fy_u8_to_float(const unsigned char* in, float* out, size_t n) {
    fy::enter();
    host_elementwise(in, out, n, [&](const uint8_t* di, float* dout, cudaStream_t st) {
        return fy_launch_u8_to_float(di, dout, n, st);
    }, "fy_u8_to_float");
}
extern "C" void fy_float_to_u8(const float* in, unsigned char* out, size_t n) {
    fy::enter();
    host_elementwise(in, out, n, [&](const float* di, uint8_t* dout, cudaStream_t st) {
        return fy_launch_float_to_u8(di, dout, n, st);
    }, "fy_float_to_u8");
}
extern "C" void fy_u8_to_phys(const unsigned char* in, float* out, size_t n, double f32_min,
                              double f32_max) {
    fy::enter();
    float lo, scale;
    dewindow_params(f32_min, f32_max, lo, scale);
    host_elementwise(in, out, n, [&](const uint8_t* di, float* dout, cudaStream_t st) {
        return fy_launch_u8_to_phys(di, dout, n, lo, scale, st);
    }, "fy_u8_to_phys");
}
extern "C" void fy_phys_to_u8(const float* in, unsigned char* out, size_t n, double f32_min,
                              double f32_max) {
    fy::enter();
    float lo, inv;
    rewindow_params(f32_min, f32_max, lo, inv);
    host_elementwise(in, out, n, [&](const float* di, uint8_t* dout, cudaStream_t st) {
        return fy_launch_phys_to_u8(di, dout, n, lo, inv, st);
    }, "fy_phys_to_u8");
}
// scalar plan-time helper (stream.c:59-63)
extern "C" float fy_phys_to_u8_level(double phys, double f32_min, double f32_max) {
    const double span = f32_max - f32_min;
    if (span == 0.0) return 0.0f;
    return (float)((phys - f32_min) / span * 255.0);
}

extern "C" int fy_gpu_u8_to_phys(const unsigned char* d_in, float* d_out, size_t n, double f32_min,
                                 double f32_max, void* stream) {
    fy::enter();
    if (n && (!d_in || !d_out)) return fail(FY_EINVAL, "fy_gpu_u8_to_phys: null pointer");
    int rc = fy::ensure_ctx();
    if (rc) return rc;
    float lo, scale;
    dewindow_params(f32_min, f32_max, lo, scale);
    cudaError_t e = fy_launch_u8_to_phys(d_in, d_out, n, lo, scale, (cudaStream_t)stream);
    if (e != cudaSuccess) return fail_cuda(e, "fy_gpu_u8_to_phys");
    fy::count_launch();
    return FY_OK;
}
extern "C" int fy_gpu_phys_to_u8(const float* d_in, unsigned char* d_out, size_t n, double f32_min,
                                 double f32_max, void* stream) {
    fy::enter();
    if (n && (!d_in || !d_out)) return fail(FY_EINVAL, "fy_gpu_phys_to_u8: null pointer");
    int rc = fy::ensure_ctx();
    if (rc) return rc;
    float lo, inv;
    rewindow_params(f32_min, f32_max, lo, inv);
    cudaError_t e = fy_launch_phys_to_u8(d_in, d_out, n, lo, inv, (cudaStream_t)stream);
    if (e != cudaSuccess) return fail_cuda(e, "fy_gpu_phys_to_u8");
    fy::count_launch();
    return FY_OK;
}

// ============================================================== deconvolution
namespace {

#define FY_MAX_DECONV_GAIN 8.0   // paganin.c:50

// wiener_weight, paganin.c:296-299
double wiener_w(double fr, const fy_physics* p, double reg) {
    const double h = fy_recon_transfer(fr, p);
    return h / (h * h + reg);
}
// matched_transfer, paganin.c:321-328
double matched_w(double fr, const fy_physics* p, double gamma) {
    const double sigma = p->psf_sigma_vox > 0 ? p->psf_sigma_vox : 1.0;
    const double g = exp(-2.0 * M_PI * M_PI * sigma * sigma * (fr * fr));
    const double hf = g * fy_unsharp_transfer(fr, p);
    return hf / (hf * hf + gamma);
}

struct DeconvKey {
    int nz, ny, nx, kind;
    double param, fz2s;
    fy_physics p;
};

}  // namespace

// Plan-time tables of deconv_radial (paganin.c:213-230) into host memory of
// fy_deconv_table_bytes(g) bytes: the 4097-entry float LUT of the capped weight over u = f^2
// (padded to 16 bytes), then fz2, fy2 and fx2 in double. Returns the LUT index scale us.
size_t fy_deconv_table_bytes(const SpecGeom& g) {
    const size_t lut_bytes = ((FY_LUT_N + 1) * sizeof(float) + 15) & ~(size_t)15;
    return lut_bytes + sizeof(double) * ((size_t)g.pz + g.py + g.hx);
}
double fy_deconv_fill_tables(const SpecGeom& g, const fy_physics* p, double param, int kind, double fz2s,
                             void* host) {
    const size_t lut_bytes = ((FY_LUT_N + 1) * sizeof(float) + 15) & ~(size_t)15;
    unsigned char* h = (unsigned char*)host;
    float* lut = (float*)h;
    double* fz2 = (double*)(h + lut_bytes);
    double* fy2 = fz2 + g.pz;
    double* fx2 = fy2 + g.py;
    double mz = 0, my = 0, mx = 0;
    for (int i = 0; i < g.pz; i++) {
        const double f = (i <= g.pz / 2) ? (double)i / g.pz : (double)(i - g.pz) / g.pz;
        fz2[i] = f * f * fz2s; if (fz2[i] > mz) mz = fz2[i];
    }
    for (int i = 0; i < g.py; i++) {
        const double f = (i <= g.py / 2) ? (double)i / g.py : (double)(i - g.py) / g.py;
        fy2[i] = f * f; if (fy2[i] > my) my = fy2[i];
    }
    for (int i = 0; i < g.hx; i++) {
        const double f = (double)i / g.px;
        fx2[i] = f * f; if (fx2[i] > mx) mx = fx2[i];
    }
    const double umax = mz + my + mx;
    // A 1x1x1 volume has umax = 0; every sample then sits at u = 0 (us = 0 -> t = 0).
    const double us = umax > 0 ? FY_LUT_N / umax : 0.0;
    const double cap = kind == 1 ? 0.0 : FY_MAX_DECONV_GAIN;
    for (int i = 0; i <= FY_LUT_N; i++) {
        const double fr = us > 0 ? sqrt((double)i / us) : 0.0;
        double w = kind == 1 ? matched_w(fr, p, param) : wiener_w(fr, p, param);
        if (cap > 0 && w > cap) w = cap;
        lut[i] = (float)w;
    }
    return us;
}

namespace {
// The same tables, cached per thread and uploaded once per parameter set.
int deconv_tables(const SpecGeom& g, const fy_physics* p, double param, int kind, double fz2s,
                  cudaStream_t st, DeconvLaunch& d) {
    fy::ThreadCtx& c = ctx();
    DeconvKey key;
    memset(&key, 0, sizeof key);
    key.nz = g.nz; key.ny = g.ny; key.nx = g.nx; key.kind = kind;
    key.param = param; key.fz2s = fz2s; key.p = *p;
    const size_t lut_bytes = ((FY_LUT_N + 1) * sizeof(float) + 15) & ~(size_t)15;
    const size_t bytes = fy_deconv_table_bytes(g);
    if (!(c.tab.valid && c.tab.keylen == sizeof key && !memcmp(c.tab.key, &key, sizeof key))) {
        std::vector<unsigned char> h(bytes);
        const double us = fy_deconv_fill_tables(g, p, param, kind, fz2s, h.data());
        cudaError_t e = c.tab.buf.ensure(bytes);
        if (e != cudaSuccess) return fail_cuda(e, "deconv tables");
        // Stage through pinned memory so the upload is an ordinary asynchronous copy (a
        // pageable one waits for the stream and shares the driver's staging path); the
        // staging buffer is reused only once the previous upload has been read.
        if (c.tab_pending && (e = cudaEventSynchronize(c.tab_done)) != cudaSuccess)
            return fail_cuda(e, "deconv tables upload");
        c.tab_pending = false;
        if ((e = c.tab_pin.ensure(bytes)) != cudaSuccess) return fail_cuda(e, "deconv tables");
        if (!c.tab_done && (e = cudaEventCreateWithFlags(&c.tab_done, cudaEventDisableTiming)) != cudaSuccess)
            return fail_cuda(e, "deconv tables");
        memcpy(c.tab_pin.p, h.data(), bytes);
        if ((e = cudaMemcpyAsync(c.tab.buf.p, c.tab_pin.p, bytes, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
            (e = cudaEventRecord(c.tab_done, st)) != cudaSuccess)
            return fail_cuda(e, "deconv tables upload");
        c.tab_pending = true;
        memcpy(c.tab.key, &key, sizeof key);
        c.tab.keylen = sizeof key;
        c.tab.us = us;
        c.tab.valid = true;
    }
    unsigned char* base = (unsigned char*)c.tab.buf.p;
    d.lut = (const float*)base;
    d.fz2 = (const double*)(base + lut_bytes);
    d.fy2 = d.fz2 + g.pz;
    d.fx2 = d.fy2 + g.py;
    d.us = c.tab.us;
    return FY_OK;
}

int make_geom(int nz, int ny, int nx, SpecGeom& g, const char* what) {
    if (nz < 1 || ny < 1 || nx < 1) return fail(FY_EINVAL, "%s: bad dims %dx%dx%d", what, nz, ny, nx);
    g.nz = nz; g.ny = ny; g.nx = nx;
    g.pz = fy_next_fft_size(nz); g.py = fy_next_fft_size(ny); g.px = fy_next_fft_size(nx);
    if (!fy_fft_len_ok(g.pz) || !fy_fft_len_ok(g.py) || !fy_fft_len_ok(g.px))
        return fail(FY_EUNSUPPORTED, "%s: padded size %dx%dx%d exceeds %d per axis", what, g.pz, g.py,
                    g.px, FY_FFT_MAXN);
    g.hx = g.px / 2 + 1;
    g.hxp = (g.hx + 15) & ~15;
    g.zero_pad = 0;
    return FY_OK;
}

// Resolve kind defaults exactly as fy_deconvolve / fy_deconvolve_matched do.
void deconv_defaults(const fy_physics* p, int kind, double& param, double& fz2s) {
    if (kind == 0) { if (param <= 0.0) param = fy_auto_reg(p, 0.015); fz2s = 1.0; }   // paganin.c:305
    else if (kind == 1) {                                                            // paganin.c:333-340
        if (param <= 0) param = 0.05;
        fz2s = 1.0;
        const double sxy = p->psf_sigma_vox > 0 ? p->psf_sigma_vox : 1.0;
        if (p->psf_sigma_z_vox > 0 && sxy > 0) { const double rr = p->psf_sigma_z_vox / sxy; fz2s = rr * rr; }
    } else {
        if (param <= 0.0) param = fy_auto_reg(p, 0.015);
        if (fz2s <= 0) fz2s = 1.0;                                                  // paganin.c:218
    }
}

// Enqueue the full deconvolution on st. src is device memory (u8 or f32), dst device f32.
int enqueue_deconv(const void* src, int src_u8, double fmin, double fmax, float* dst, int nz, int ny,
                   int nx, const fy_physics* p, double param, int kind, double fz2s, cudaStream_t st,
                   const char* what) {
    fy::ThreadCtx& c = ctx();
    DeconvLaunch d{};
    int rc = make_geom(nz, ny, nx, d.g, what);
    if (rc) return rc;
    deconv_defaults(p, kind, param, fz2s);
    d.plx = fy_make_plan(d.g.px); d.ply = fy_make_plan(d.g.py); d.plz = fy_make_plan(d.g.pz);
    d.twx = fy::twiddles(d.g.px); d.twy = fy::twiddles(d.g.py); d.twz = fy::twiddles(d.g.pz);
    if (!d.twx || !d.twy || !d.twz) return fail(FY_ENOMEM, "%s: twiddle tables", what);
    cudaError_t e = c.spec.ensure(fy_deconv_spec_elems(d.g) * sizeof(float2));
    if (e != cudaSuccess) return fail_cuda(e, what);
    d.spec = c.spec.as<float2>();
    if ((rc = deconv_tables(d.g, p, param, kind, fz2s, st, d))) return rc;
    d.src = src; d.src_u8 = src_u8; d.dst = dst;
    dewindow_params(fmin, fmax, d.lo, d.scale);
    if ((e = fy_launch_deconv(d, st)) != cudaSuccess) return fail_cuda(e, what);
    fy::count_launch(5);
    return FY_OK;
}

int host_deconv(const float* in, float* out, int nz, int ny, int nx, const fy_physics* p, double param,
                int kind, double fz2s, const char* what) {
    if (!in || !out || !p) return fail(FY_EINVAL, "%s: null pointer", what);
    SpecGeom g;
    int rc = make_geom(nz, ny, nx, g, what);
    if (rc) return rc;
    if ((rc = fy::ensure_ctx())) return rc;
    fy::ThreadCtx& c = ctx();
    cudaStream_t st = c.st;
    const size_t n = (size_t)nz * ny * nx;
    fy::ws_acquire(st);
    cudaError_t e = c.vin.ensure(n * sizeof(float));
    if (e != cudaSuccess) return fail_cuda(e, what);
    if ((e = cudaMemcpyAsync(c.vin.p, in, n * sizeof(float), cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return fail_cuda(e, what);
    // dst aliases the device copy of src: P1 consumes src before P5 writes dst
    if ((rc = enqueue_deconv(c.vin.p, 0, 0.0, 0.0, c.vin.as<float>(), nz, ny, nx, p, param, kind, fz2s, st,
                             what)))
        return rc;
    if ((e = cudaMemcpyAsync(out, c.vin.p, n * sizeof(float), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return fail_cuda(e, what);
    fy::ws_release(st);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return fail_cuda(e, what);
    return FY_OK;
}
}  // namespace

// Everything of a deconvolution launch but its buffers (spectrum, tables, source, output): the
// geometry, the kind's defaults (param and fz2 scale, as fy_deconvolve* resolve them), the
// plans, the twiddle tables and the dewindow scalars.
int fy_deconv_setup(int nz, int ny, int nx, const fy_physics* p, double& param, int kind, double& fz2s,
                    double fmin, double fmax, DeconvLaunch& d, const char* what) {
    int rc = make_geom(nz, ny, nx, d.g, what);
    if (rc) return rc;
    deconv_defaults(p, kind, param, fz2s);
    d.plx = fy_make_plan(d.g.px); d.ply = fy_make_plan(d.g.py); d.plz = fy_make_plan(d.g.pz);
    d.twx = fy::twiddles(d.g.px); d.twy = fy::twiddles(d.g.py); d.twz = fy::twiddles(d.g.pz);
    if (!d.twx || !d.twy || !d.twz) return fail(FY_ENOMEM, "%s: twiddle tables", what);
    dewindow_params(fmin, fmax, d.lo, d.scale);
    return FY_OK;
}

// Size the calling thread's deconvolution workspaces (half spectrum, tables) for a cube shape,
// so later calls up to that shape allocate nothing.
int fy_deconv_reserve(int nz, int ny, int nx) {
    SpecGeom g;
    int rc = make_geom(nz, ny, nx, g, "fy_deconv_reserve");
    if (rc) return rc;
    if ((rc = fy::ensure_ctx())) return rc;
    fy::ThreadCtx& c = ctx();
    const size_t lut_bytes = ((FY_LUT_N + 1) * sizeof(float) + 15) & ~(size_t)15;
    cudaError_t e;
    if ((e = c.spec.ensure(fy_deconv_spec_elems(g) * sizeof(float2))) != cudaSuccess ||
        (e = c.tab.buf.ensure(lut_bytes + sizeof(double) * ((size_t)g.pz + g.py + g.hx))) != cudaSuccess ||
        (e = c.tab_pin.ensure(lut_bytes + sizeof(double) * ((size_t)g.pz + g.py + g.hx))) != cudaSuccess)
        return fail_cuda(e, "fy_deconv_reserve");
    if (!fy::twiddles(g.px) || !fy::twiddles(g.py) || !fy::twiddles(g.pz))
        return fail(FY_ENOMEM, "fy_deconv_reserve: twiddle tables");
    return FY_OK;
}

extern "C" int fy_deconvolve(const float* in, float* out, int nz, int ny, int nx, const fy_physics* p,
                             double reg) {
    fy::enter();
    return host_deconv(in, out, nz, ny, nx, p, reg, 0, 1.0, "fy_deconvolve");
}
extern "C" int fy_deconvolve_matched(const float* in, float* out, int nz, int ny, int nx,
                                     const fy_physics* p, double tikhonov) {
    fy::enter();
    return host_deconv(in, out, nz, ny, nx, p, tikhonov, 1, 1.0, "fy_deconvolve_matched");
}

extern "C" int fy_gpu_deconvolve_ex(const void* d_in, int src_u8, double f32_min, double f32_max,
                                    float* d_out, int nz, int ny, int nx, const fy_physics* p,
                                    double param, int kind, double fz2_scale, void* stream) {
    fy::enter();
    if (!d_in || !d_out || !p) return fail(FY_EINVAL, "fy_gpu_deconvolve_ex: null pointer");
    if (kind < 0 || kind > 2) return fail(FY_EINVAL, "fy_gpu_deconvolve_ex: kind %d", kind);
    int rc = fy::ensure_ctx();
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    fy::ws_acquire(st);
    rc = enqueue_deconv(d_in, src_u8 ? 1 : 0, f32_min, f32_max, d_out, nz, ny, nx, p, param, kind,
                        fz2_scale, st, "fy_gpu_deconvolve_ex");
    fy::ws_release(st);
    return rc;
}
