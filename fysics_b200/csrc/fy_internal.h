// fy_internal.h -- host-side declarations shared between the kernel files and the C-ABI
// layer (fy_api.cu). Not part of the public interface.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>
#include <type_traits>
#include "fy_spectral.cuh"

#define FY_LUT_N 4096   // paganin.c:138, radial weight LUT over u = f^2

// Everything the five deconvolution passes need, all device pointers.
struct DeconvLaunch {
    const void* src;          // f32 or u8 volume (nz,ny,nx)
    int src_u8;               // 1: u8 source dewindowed as lo + u8*scale (stream.c:41-46)
    float lo, scale;
    float* dst;               // f32 (nz,ny,nx); may alias src when src is f32
    float2* spec;             // nz * py * hxp complex workspace
    SpecGeom g;
    FftPlan plx, ply, plz;
    const float2 *twx, *twy, *twz;
    const float* lut;         // FY_LUT_N+1 floats
    const double *fz2, *fy2, *fx2;
    double us;                // LUT index scale FY_LUT_N / umax
};
cudaError_t fy_launch_deconv(const DeconvLaunch& d, cudaStream_t st);
// Compile-time-plan pass `pass` (1..5) for axis length n; cudaErrorNotSupported when n has no
// instantiation in that unit (a: 512, 96, 1024; b: 256, 384, 64; c: 128, 192, 768).
cudaError_t fy_deconv_pass_ct_a(int pass, int n, const DeconvLaunch& d, cudaStream_t st);
cudaError_t fy_deconv_pass_ct_b(int pass, int n, const DeconvLaunch& d, cudaStream_t st);
cudaError_t fy_deconv_pass_ct_c(int pass, int n, const DeconvLaunch& d, cudaStream_t st);
size_t fy_deconv_spec_elems(const SpecGeom& g);
// Host side of a deconvolution (fy_api.cu): the plan-time tables into host memory (returns the
// LUT index scale), their size, and the launch fields other than its buffers.
size_t fy_deconv_table_bytes(const SpecGeom& g);
double fy_deconv_fill_tables(const SpecGeom& g, const fy_physics* p, double param, int kind, double fz2s, void* host);
int fy_deconv_setup(int nz, int ny, int nx, const fy_physics* p, double& param, int kind, double& fz2s,
                    double fmin, double fmax, DeconvLaunch& d, const char* what);
cudaError_t fy_launch_spec_y(float2* spec, const SpecGeom& g, const FftPlan& ply, const float2* twy, int nplanes,
                             int sign, int keep_rows, cudaStream_t st);
cudaError_t fy_launch_cfft3d(float2* c, int nz, int ny, int nx, int nxp, int sign, cudaStream_t st);

// Elementwise stream ops (stream.c)
cudaError_t fy_launch_u8_to_phys(const uint8_t* in, float* out, size_t n, float lo, float scale,
                                 cudaStream_t st);
cudaError_t fy_launch_phys_to_u8(const float* in, uint8_t* out, size_t n, float lo, float inv,
                                 cudaStream_t st);
cudaError_t fy_launch_float_to_u8(const float* in, uint8_t* out, size_t n, cudaStream_t st);
cudaError_t fy_launch_u8_to_float(const uint8_t* in, float* out, size_t n, cudaStream_t st);

// Guided filter / box mean (fy_guided.cu)
// Ring subtraction folded into a producer's store (dering.c:200-248, the same arithmetic as
// fy_dering_apply): ring == nullptr means none.
struct RingApply {
    const float* ring = nullptr;      // [nslab][nr] device ring profile
    const int* have = nullptr;        // device have_rings flag (nullptr: apply unconditionally)
    int nslab = 0, nr = 0, slab_z = 1;
    double cy = 0.0, cx = 0.0;        // ring centre (global y, x)
    long z0 = 0, y0 = 0, x0 = 0;      // global offset of the volume
    float sc = 0.f;                   // ring units -> volume units
};
// Fill `ra` from a device ring handle (fy_api_dering.cu).
void fy_dering_ring_args(const fy_gpu_dering* h, long z0, long y0, long x0, double scale, RingApply* ra);

// exact r <= 4: ab_ws holds fy_guided_fused_scratch_floats(n); out may alias in
size_t fy_guided_fused_scratch_floats(size_t n);
size_t fy_guided_fast_scratch_floats(int lz, int ly, int lx);
cudaError_t fy_launch_guided_fused(const float* in, float* out, float* out_b, float* ab_ws, int nz, int ny, int nx,
                                   int r, float eps, int mode, int sms, cudaStream_t st,
                                   const float* eps_ptr = nullptr, const RingApply* rings = nullptr);
cudaError_t fy_launch_guided_generic(const float* in, float* out, float* ws, int nz, int ny, int nx, int r,
                                     float eps, cudaStream_t st, int& launches);
cudaError_t fy_launch_guided_fast(const float* in, float* out, float* ws, int nz, int ny, int nx, int r,
                                  float eps, int s, int sms, cudaStream_t st, int& launches,
                                  const float* eps_ptr = nullptr);
cudaError_t fy_launch_box_mean(const float* in, float* out, float* tmp, int nz, int ny, int nx, int r,
                               cudaStream_t st, int& launches);
// output pass from guided (mean, var) pairs written by the noise statistics pass (r = win/2)
cudaError_t fy_launch_guided_apply_mv(const float* mv, const float* in, float* out, int nz, int ny, int nx, int r,
                                      float eps, int sms, cudaStream_t st, const float* eps_ptr,
                                      const RingApply* rings);

// Noise model (fy_noise.cu)
size_t fy_noise_ctl_bytes();
size_t fy_noise_scratch_floats(size_t n);
cudaError_t fy_launch_estimate_noise(const float* in, int nz, int ny, int nx, int win, double flat_pct,
                                     double ref_intensity, float* scratch, void* ctl_mem, int sms,
                                     cudaStream_t st, int& launches, float* guided_mv = nullptr);
cudaError_t fy_noise_read(const void* ctl_mem, double* g, double* b, double* noise_ref, double* ref_intensity,
                          int* used, cudaStream_t st);
const float* fy_noise_eps_ptr(const void* ctl_mem);
// Copy a finished model into caller device memory (an fy_noise_model; d_eps may be null).
cudaError_t fy_noise_store(const void* ctl_mem, void* d_model, float* d_eps, cudaStream_t st);

// Ring removal (fy_dering.cu)
cudaError_t fy_launch_dering_accum(const uint8_t* buf, const int* map, unsigned long long* sum, unsigned int* cnt,
                                   int nbins, long dz, long dy, long dx, int ss, int sms, cudaStream_t st);
cudaError_t fy_launch_dering_finalize(const float* sum_f, const unsigned int* cnt, float* ring, void* scratch,
                                      unsigned long long* detected, int* have_rings, int nslab, int ns, int nr,
                                      int hp_win, unsigned min_cnt, double min_amp, double max_amp,
                                      cudaStream_t st);
size_t fy_dering_finalize_scratch(int nslab, int ns, int nr);
cudaError_t fy_launch_dering_apply(float* f, const float* ring, const int* have_rings, int nslab, int nr,
                                   int slab_z, double cy, double cx, long z0, long y0, long x0, long dz, long dy,
                                   long dx, double scale, cudaStream_t st);

// Per-kernel profiling marks (fy_context.cu): records a CUDA event on st after a launch
// when profiling is enabled on the calling thread; no-op otherwise.
void fy_prof_mark(cudaStream_t st, const char* name);

// Opt a kernel into a large dynamic shared-memory carve-out. Above 32 KB of dynamic smem
// (the default limit is 48 KB including static smem), raise the kernel's limit once per
// device and size; cached so launches pay the driver call only when the size grows.
cudaError_t fy_smem_optin_raw(const void* kernel, size_t bytes);
template <class K>
inline cudaError_t fy_smem_optin(K kernel, size_t bytes) {
    if (bytes <= 32 * 1024) return cudaSuccess;
    return fy_smem_optin_raw((const void*)kernel, bytes);
}

// Launch with programmatic stream serialization: the kernel (which starts with fy_pdl_wait())
// may be scheduled before the previous kernel on `st` has finished, hiding the launch gap
// between a chain of small dependent kernels.
template <class... KArgs, class... Args>
inline cudaError_t fy_launch_pdl(void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                                 Args... args) {
    cudaLaunchConfig_t c = {};
    c.gridDim = grid;
    c.blockDim = block;
    c.dynamicSmemBytes = smem;
    c.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    c.attrs = at;
    c.numAttrs = 1;
    return cudaLaunchKernelEx(&c, k, ((KArgs)args)...);
}

// Runtime elements-per-thread (fy_fft_e) -> compile-time E for kernel instantiation.
template <class F>
inline cudaError_t fy_with_e(int e, F&& f) {
    switch (e) {
        case 24: return f(std::integral_constant<int, 24>{});
        case 16: return f(std::integral_constant<int, 16>{});
        case 12: return f(std::integral_constant<int, 12>{});
        case 8: return f(std::integral_constant<int, 8>{});
        case 6: return f(std::integral_constant<int, 6>{});
        case 4: return f(std::integral_constant<int, 4>{});
        case 3: return f(std::integral_constant<int, 3>{});
        case 2: return f(std::integral_constant<int, 2>{});
        default: return f(std::integral_constant<int, 1>{});
    }
}

// Launch shape of a tile of lines of length n: W lines, NT = W*n/E threads.
struct TileShape {
    int W, wlog, E, NT;
};
inline TileShape fy_tile_shape(int n) {
    TileShape t;
    t.W = fy_tile_lines(n);
    t.wlog = fy_log2i(t.W);
    t.E = fy_fft_e(n);
    t.NT = t.W * n / t.E;
    return t;
}

// Autotuned launch shapes (fy_autotune.cu), per device. A lookup returns 0 when nothing is
// tuned for the key (the caller keeps its default). Tuned shapes change how work is split
// over CTAs, never the arithmetic, so results are bit-identical to the defaults.
//   fy_tuned_x_wlog   log2 of the lines per CTA of a deconvolution X pass (pass 1 or 5) of
//                     axis length n (line-major tiles: any W <= the default fits)
int fy_tuned_x_wlog(int pass, int n);
// Default z-chunk count of a box pass (64 x 16 column tiles, `per_sm` CTAs resident per SM,
// so a launch runs in waves of per_sm*sms CTAs): among chunk counts with chunks of >= 8r
// planes and at least ~3 waves of work, the one whose CTAs best fill their last wave, net of
// the 2r-plane warm-up each chunk repeats: score = (waves / ceil(waves)) * zchunk / (zchunk + 2r).
inline int fy_box_default_chunks(int nz, int ny, int nx, int r, int sms, int per_sm = 2) {
    const long txy = (long)((nx + 63) / 64) * ((ny + 15) / 16), slots = (long)per_sm * sms;
    int hi = nz / (8 * r);
    if (hi < 1) hi = 1;
    int lo = (int)((3 * slots + txy - 1) / txy);
    if (lo > hi) lo = hi;
    if (lo < 1) lo = 1;
    int best = lo;
    double best_score = -1.0;
    for (int nc = lo; nc <= hi && nc <= 4 * lo; ++nc) {
        const int zc = (nz + nc - 1) / nc;
        const long ctas = txy * ((nz + zc - 1) / zc);
        const double waves = (double)ctas / (double)slots;
        const long whole = (long)waves + ((double)(long)waves < waves ? 1 : 0);
        const double score = waves / (double)whole * (double)zc / (double)(zc + 2 * r);
        if (score > best_score + 1e-9) { best_score = score; best = nc; }
    }
    return best;
}
// TileShape of an X pass: the tuned lines per CTA when there is one, else the default.
inline TileShape fy_x_tile_shape(int pass, int n) {
    TileShape t = fy_tile_shape(n);
    const int wl = fy_tuned_x_wlog(pass, n);
    if (wl > 0 && wl < t.wlog && (n << wl) / t.E >= 32) {
        t.wlog = wl;
        t.W = 1 << wl;
        t.NT = t.W * n / t.E;
    }
    return t;
}

// Radial guided-eps model (fy_radial.cu): cube eps = base * radial scale, on the device.
cudaError_t fy_launch_radial_tile_eps(const fy_radial_eps* d_fit, const float* base_dev, float base_host, double ecy,
                                      double ecx, long y0, long x0, long ty, long tx, float* d_out, cudaStream_t st);

// Workspace reservation for a cube shape on the calling thread (fy_api.cu, fy_restore.cu).
int fy_deconv_reserve(int nz, int ny, int nx);
int fy_restore_reserve(int nz, int ny, int nx);
// Free the calling thread's per-tile chain workspaces (fy_tile.cu); part of fy_gpu_release.
void fy_tile_release();
int fy_guided_wait_timeouts();
int fy_batch_wait_timeouts();
int fy_deconv_wait_timeouts();
int fy_deconv_ct_a_timeouts();
int fy_deconv_ct_b_timeouts();
int fy_deconv_ct_c_timeouts();
cudaError_t fy_batch_set_first_wait_polls(int polls);
int fy_noise_wait_timeouts();
cudaError_t fy_guided_set_first_wait_polls(int polls);
cudaError_t fy_noise_set_first_wait_polls(int polls);
cudaError_t fy_noise_test_paths(int force_radix, int* used);
