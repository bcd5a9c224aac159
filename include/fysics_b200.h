/* fysics_b200.h -- B200 (sm_100a) drop-in for the fysics per-cube restoration hot path.
 *
 * Part 1 declares the SAME C symbols, signatures and struct layouts as the reference's
 * public header (fysics.h), for exactly the functions on the restoration path. A C caller
 * of fysics links libfysics_b200.so ahead of libfysics and gets these entry points on the
 * GPU with unchanged semantics: caller-owned HOST buffers, synchronous calls, outputs
 * valid on return, int 0 = success. Each declaration cites the fysics.h line it replaces.
 * Every call runs on the GPU; there is no CPU fallback. Without a usable CUDA device an
 * int entry point returns FY_ENODEV (4) and a void entry point leaves its outputs
 * untouched and records the error, readable through fy_gpu_last_error().
 *
 * Part 2 is the fy_gpu_* extension: device pointers, CUDA streams (passed as void*),
 * fused chains, batches and the serving loop. Nothing in it has a reference counterpart
 * except where stated.
 */
#ifndef FYSICS_B200_H
#define FYSICS_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ====================================================================== part 1: drop-in */

/* fysics.h:23-35 -- 8 doubles, layout-identical */
typedef struct {
    double delta_beta;
    double energy_kev;
    double distance_mm;
    double pixel_um;
    double unsharp_sigma;
    double unsharp_coeff;
    double psf_sigma_vox;
    double psf_sigma_z_vox;
} fy_physics;

/* fysics.h:191-197 */
typedef struct {
    double g;
    double b;
    double noise_ref;
    double ref_intensity;
    int    n_bins_used;
} fy_noise_model;

/* fysics.h:406-415 -- callers read ring[] and have_rings directly; fwrite-serialisable */
typedef struct {
    long Z, Y, X;
    double cy, cx;
    int slab_z, nslab;
    int ns, nr;
    float *sum;
    unsigned int *cnt;
    float *ring;
    int have_rings;
} fy_dering;

/* FFT sizes, fysics.h:38-40 */
int  fy_is_pow2(int n);
int  fy_next_pow2(int n);
int  fy_next_fft_size(int n);
/* fysics.h:41-43: in-place split re/im transforms (sizes 2^k, 3*2^k up to 4096 per axis) */
void fy_fft1d(float *re, float *im, int n, int sign);
void fy_fft3d(float *re, float *im, int nz, int ny, int nx, int sign);
void fy_fft3d_normalize(float *re, float *im, int nz, int ny, int nx);

/* u8 <-> float windowing, fysics.h:56-57, 70-76 */
void  fy_u8_to_float(const unsigned char *in, float *out, size_t n);
void  fy_float_to_u8(const float *in, unsigned char *out, size_t n);
void  fy_u8_to_phys(const unsigned char *in, float *out, size_t n, double f32_min, double f32_max);
void  fy_phys_to_u8(const float *in, unsigned char *out, size_t n, double f32_min, double f32_max);
float fy_phys_to_u8_level(double phys, double f32_min, double f32_max);

/* transfer functions and plan-time helpers, fysics.h:98-117, 146 */
double fy_paganin_transfer(double f_cyc_per_voxel, const fy_physics *p);
double fy_unsharp_transfer(double f_cyc_per_voxel, const fy_physics *p);
double fy_recon_transfer(double f_cyc_per_voxel, const fy_physics *p);
double fy_auto_reg(const fy_physics *p, double base);
double fy_auto_deltabeta_scale(const fy_physics *p);
int    fy_kernel_halo(const fy_physics *p);

/* Wiener deconvolution, fysics.h:131-142 (in/out may alias) */
int fy_deconvolve(const float *in, float *out, int nz, int ny, int nx,
                  const fy_physics *p, double reg);
int fy_deconvolve_matched(const float *in, float *out, int nz, int ny, int nx,
                          const fy_physics *p, double tikhonov);

/* guided filter, fysics.h:152-167 */
int    fy_guided_denoise(const float *in, float *out, int nz, int ny, int nx,
                         int radius, double eps);
int    fy_guided_denoise_ws(const float *in, float *out, int nz, int ny, int nx,
                            int radius, double eps, float *ws);
size_t fy_guided_ws_floats(int nz, int ny, int nx);
int    fy_guided_denoise_fast_ws(const float *in, float *out, int nz, int ny, int nx,
                                 int radius, double eps, int s, float *ws);
void   fy_box_smooth(const float *in, float *out, float *tmp, int nz, int ny, int nx, int r);
double fy_guided_eps_for_noise(double noise_ref);

/* noise model, fysics.h:203-205 */
int fy_estimate_noise(const float *in, int nz, int ny, int nx, int win, double flat_pct,
                      double ref_intensity, fy_noise_model *out);

/* ring removal, fysics.h:417-433 */
int  fy_dering_init(fy_dering *d, long Z, long Y, long X, double cy, double cx,
                    int slab_z, int ns);
void fy_dering_free(fy_dering *d);
int  fy_dering_tile_init(fy_dering *t, const fy_dering *d);
void fy_dering_tile_reset(fy_dering *t);
void fy_dering_accumulate_u8(fy_dering *t, const unsigned char *buf, long y0, long x0,
                             long dz, long dy, long dx, int ss);
void fy_dering_merge_tile(fy_dering *d, int slab, const fy_dering *t);
long fy_dering_finalize(fy_dering *d, int hp_win, unsigned int min_cnt, double min_amp,
                        double max_amp);
void fy_dering_apply(const fy_dering *d, float *f, long z0, long y0, long x0, long dz,
                     long dy, long dx, double scale);

/* phase correlation, fysics.h:311-313 */
int fy_phase_correlate(const float *fixed, const float *moving, int nz, int ny, int nx,
                       double *shift, double *peak, int window);

/* calibration statistics (pass 1), fysics.h:54, 78-82, 95, 214-215. The histogram state is
 * layout-identical; fy_hist_init/merge/percentile* are O(256) host bookkeeping on it, the
 * per-voxel counting of fy_hist_accumulate_u8 runs on the GPU. fy_flat_noise returns NaN
 * (reason in fy_gpu_last_error) when it cannot run; fy_noise_aniso returns 1 as the
 * reference does for too few blocks, and an FY_E* code above 1 when it cannot run. */
typedef struct { long hist[256]; long total; } fy_hist_state;
void   fy_hist_init(fy_hist_state *s);
void   fy_hist_accumulate_u8(fy_hist_state *s, const unsigned char *chunk, size_t n);
void   fy_hist_merge(fy_hist_state *dst, const fy_hist_state *src);
int    fy_hist_percentile_u8(const fy_hist_state *s, double pct);
int    fy_hist_percentile_u8_inner(const fy_hist_state *s, double pct);
double fy_flat_noise(const float *v, int nz, int ny, int nx, int blk);
int    fy_noise_aniso(const float *v, int nz, int ny, int nx, double *rho_z, double *rho_xy);

/* PSF edge fit of pass-1 calibration (pipeline.c:107-196, static there and called by
 * fy_calibrate): sigma in voxels of the effective PSF from up to 400 air/papyrus edge
 * profiles of a u8 tile, or -1 with fewer than 30 (or a fit outside (0.3, 5)). *nprof (may
 * be NULL) receives the number of profiles used. Returns NaN when it cannot run (reason in
 * fy_gpu_last_error). */
double fy_measure_psf_sigma(const unsigned char *vol, int Z, int Y, int X, int *nprof);

/* histogram valley (fysics.h:92, stream.c:138-168): O(256) host arithmetic on counts */
double fy_valley_depth(const long hist[256], int *dark_out, int *light_out, int *valley_out);

/* ---- the per-tile chain of the export tool (fysics.h:436-511, pipeline.c:252-510).
 * fy_pipeline_cfg is layout-identical to the reference's; fy_process_buffer reads the
 * fields the tile chain uses (physics, window, do_deconv/use_matched_deconv/psf/tikhonov,
 * dec range, guided_eps/subsample and the radial eps fit, air-zero settings, norm, dither,
 * rings through `dering`, z drift through `zdrift_factor`) and ignores the rest. */
typedef struct {
    double delta_beta, energy_kev, distance_mm, pixel_um, unsharp_sigma, unsharp_coeff;
    double machine_current_start, machine_current_stop;
    double window_lo, window_hi;
    int    do_deconv;
    int    use_matched_deconv;
    double psf_sigma_vox, deconv_tikhonov;
    double guided_eps;
    int    do_air_zero; int air_cut_u8, air_cut_band; double air_thresh;
    double air_cut_aggr;
    int    air_min_component;
    double denoise_k;
    int    scratch_passes;
    int    do_normalize; int norm_lo, norm_hi;
    int    do_zdrift; float *zdrift_factor;
    int    do_dering;
    double calib_budget_gb;
    double dering_cy, dering_cx;
    double psf_p5, psf_med;
    int    do_musica; double musica_p; int musica_levels; double musica_core;
    int    guided_subsample;
    int    no_dither;
    int    halo;
    int    have_norm, have_zdrift, have_dec_range;
    int    have_dering; fy_dering *dering;
    double psf_z_ratio;
    int    have_eps_r; double eps_fn_a, eps_fn_b, eps_fn_med;
    double dec_lo, dec_hi;
    long   vol_z;
    double noise_floor;
    const unsigned char *occ;
    long   occ_ncz, occ_ncy, occ_ncx;
    long   occ_cz, occ_cy, occ_cx;
} fy_pipeline_cfg;
/* One inner tile from a haloed u8 buffer (fysics.h:507-511): u8buf is hz*hy*hx at global
 * origin (rz0, ry0, rx0); the inner tile (z0, y0, x0, tz, ty, tx) lies inside it; vol_y and
 * vol_x are the full volume's (rotation axis default). Writes tz*ty*tx u8 to out and sets
 * *all_air. Runs on the GPU and returns when out is written; thread-safe (each host thread
 * has its own stream and workspaces). Returns 0, or an FY_E* code: FY_EINVAL for a
 * tile outside the buffer, FY_EUNSUPPORTED for do_musica (not on this path). */
int    fy_process_buffer(const fy_pipeline_cfg *cfg, const unsigned char *u8buf,
                         long rz0, long ry0, long rx0, long hz, long hy, long hx,
                         long z0, long y0, long x0, long tz, long ty, long tx,
                         long vol_y, long vol_x, unsigned char *out, int *all_air);

/* ---- local zarr v2 raw-u8 input (fysics.h:375-386, zarr_io.c:133-331), staged into the GPU.
 * fy_zarr is layout-identical to the reference's. fy_zarr_open reads <root>/0/.zarray with the
 * reference's header grammar; returns 0, or 1 for a missing or bad header or an "s3://" root
 * (S3 is not supported). fy_zarr_read assembles the region [z0,z0+dz) x [y0,..) x [x0,..) into
 * out (dz*dy*dx, C order) with the reference's semantics: chunk files hold their true extent,
 * a missing or empty chunk reads as fill_value, a short file's tail as fill_value, voxels
 * outside the volume are left untouched. The chunk files are read whole into pinned memory,
 * kept in a device chunk cache and assembled on the GPU; thread-safe. Returns 0, or FY_EINVAL
 * (negative origin or size), FY_EIO (unreadable chunk file), FY_ENOMEM (the chunk cache cannot
 * hold the region's chunks). */
typedef struct {
    char root[1024];
    long shape[3];
    long chunk[3];
    unsigned char fill;
} fy_zarr;
int    fy_zarr_open(fy_zarr *z, const char *root);
int    fy_zarr_read(const fy_zarr *z, long z0, long y0, long x0, long dz, long dy, long dx,
                    unsigned char *out);
/* One inner tile of `tile`^3 at (z0,y0,x0) straight from the zarr (fysics.h:500-502,
 * pipeline.c:512-537): the haloed region (halo = cfg->halo, or 8) is assembled on the GPU from
 * the chunk cache and fed to the per-tile chain without a host round trip; writes the inner
 * tile (*out_tz x *out_ty x *out_tx u8) to out and sets *all_air. Thread-safe. */
int    fy_process_chunk(const fy_zarr *zin, const fy_pipeline_cfg *cfg, long z0, long y0, long x0,
                        int tile, unsigned char *out, int *out_tz, int *out_ty, int *out_tx,
                        int *all_air);

/* ================================================================== part 2: fy_gpu_* */

/* status codes (0 = success; 1 is the reference's generic failure) */
#define FY_OK 0
#define FY_EINVAL 1
#define FY_ENOMEM 2
#define FY_ECUDA 3
#define FY_ENODEV 4
#define FY_EUNSUPPORTED 5
#define FY_ETIMEDOUT 6
#define FY_EBUSY 7
#define FY_EDEGENERATE 8
#define FY_EIO 9          /* a chunk file could not be read */

/* Select the CUDA device for the calling thread (default 0). No reference counterpart. */
int         fy_gpu_init(int device);
/* Status and message of the calling thread's last failed call. */
int         fy_gpu_last_status(void);
const char *fy_gpu_last_error(void);
/* Release the calling thread's stream and cached device/pinned buffers. */
void        fy_gpu_release(void);
/* Launch counter: number of kernels this thread has launched (for measurement). */
unsigned long long fy_gpu_kernel_launches(void);
/* Number of bounded in-kernel waits (tensor-copy completions of the box passes, bulk row
 * copies of the deconvolution's first pass) that gave up since the library loaded on this
 * device; the kernel then returned without finishing.
 * 0 in normal operation; -1 without a device. */
int fy_gpu_kernel_timeouts(void);
/* Failure-detection hook for tests; no reference counterpart. Sets the polls that each box
 * pass CTA may spend on its FIRST tensor-copy wait (0 makes that wait expire at once, so the
 * CTA raises the timeout flag, drains its copies under the normal bound and returns with its
 * output unfinished); polls < 0 restores the normal bound. Also clears the timeout count.
 * Synchronous; call it only while no kernel of this library is in flight. */
int fy_gpu_test_box_first_wait(int polls);
/* Test hook of the noise model's order-statistic paths; no reference counterpart. The 1st/
 * 99th percentiles of the local means and the per-bin percentiles of the local variances
 * come from sample-guided key windows over one pass each, with exact radix passes over the
 * whole field when a window misses. force_radix bit 0 sends the means, bit 1 the bins, to
 * the radix passes every time (0 restores the windows). *window_used (optional) receives
 * which windows produced their result (bit 0 means, bit 1 bins) since the previous call.
 * Both paths give the same exact order statistics. Synchronises the device. */
int fy_gpu_test_noise_paths(int force_radix, int *window_used);

/* Device-pointer forms of the drop-in calls, enqueued on `stream` (a cudaStream_t, NULL =
 * legacy default stream) and NOT synchronised: results are valid once the stream reaches
 * them. Same argument meaning as part 1 (fysics.h lines cited there). */
int fy_gpu_u8_to_phys(const unsigned char *d_in, float *d_out, size_t n,
                      double f32_min, double f32_max, void *stream);
int fy_gpu_phys_to_u8(const float *d_in, unsigned char *d_out, size_t n,
                      double f32_min, double f32_max, void *stream);

/* kind: 0 = fy_deconvolve (Wiener of Paganin x unsharp, gain cap 8, param = reg),
 *       1 = fy_deconvolve_matched (PSF x unsharp, param = tikhonov),
 *       2 = Paganin x unsharp Wiener with anisotropic z: fz^2 scaled by fz2_scale
 *           (= (sigma_z/sigma_xy)^2), cap 8, param = reg -- deconv_radial's fz2_scale
 *           (paganin.c:140-154), which fysics reaches only through the matched weight.
 * src_u8 != 0: d_in is u8 and is dewindowed on load as fy_u8_to_phys(f32_min, f32_max). */
int fy_gpu_deconvolve_ex(const void *d_in, int src_u8, double f32_min, double f32_max,
                         float *d_out, int nz, int ny, int nx, const fy_physics *p,
                         double param, int kind, double fz2_scale, void *stream);

/* Guided filter on device buffers: s <= 1 exact (fy_guided_denoise_ws), s >= 2 the
 * s-decimated fast variant (fy_guided_denoise_fast_ws). d_in may equal d_out. */
int    fy_gpu_guided(const float *d_in, float *d_out, int nz, int ny, int nx, int radius,
                     double eps, int s, void *stream);
size_t fy_gpu_guided_scratch_bytes(int nz, int ny, int nx, int radius, int s);

/* Noise model on a device volume (fy_estimate_noise, fysics.h:203-205). d_scratch holds
 * fy_gpu_noise_scratch_bytes(): local mean/variance fields plus a control block in which
 * the model stays on the device. fy_gpu_noise_model copies it to the host (synchronises
 * `stream`); fy_gpu_noise_eps returns the device address of the float guided eps
 * fy_guided_eps_for_noise(noise_ref) for chaining without a host round trip. */
size_t fy_gpu_noise_scratch_bytes(int nz, int ny, int nx);
int    fy_gpu_estimate_noise(const float *d_in, int nz, int ny, int nx, int win, double flat_pct,
                             double ref_intensity, void *d_scratch, void *stream);
int    fy_gpu_noise_model(const void *d_scratch, int nz, int ny, int nx, fy_noise_model *out,
                          void *stream);
const float *fy_gpu_noise_eps(const void *d_scratch, int nz, int ny, int nx);

/* Noise model without any allocation; it has no counterpart in the reference. It is for
 * callers that may not allocate device memory while they run, e.g. a serving loop whose
 * HBM is already committed to its own pool, where a cudaMalloc can fail or stall the
 * device. Scratch is one static device array inside the library, sized for
 * FY_NOISE_NOALLOC_MAX_VOXELS voxels (128^3): FY_NOISE_NOALLOC_SCRATCH_BYTES =
 * 20,533,248 bytes (19.6 MiB). Every GPU that loads the library holds it until the
 * process exits. Larger volumes return FY_EUNSUPPORTED.
 * Runs on the calling thread's current device and enqueues on `stream`. The model goes to
 * d_model, caller device memory laid out as fy_noise_model (8-byte aligned). d_eps, which
 * may be NULL, receives the float fy_guided_eps_for_noise(noise_ref) (4-byte aligned).
 * Misaligned pointers return FY_EINVAL before anything is enqueued.
 * Every call that is not being captured resolves the array's device address afresh, so a
 * device reset between calls is harmless. The first call on each device must come before
 * any stream capture: a call made while `stream` captures reuses the address that the
 * latest uncaptured call resolved. All calls on a device share the array, which keeps
 * the previous call's contents. Calls whose GPU work can overlap race on it, e.g. calls
 * on unordered streams or from several host threads, so serialise them. */
#define FY_NOISE_NOALLOC_MAX_VOXELS 2097152
#define FY_NOISE_NOALLOC_SCRATCH_BYTES 20533248
int    fy_gpu_estimate_noise_noalloc(const float *d_in, int nz, int ny, int nx, int win,
                                     double flat_pct, double ref_intensity,
                                     fy_noise_model *d_model, float *d_eps, void *stream);

/* Calibration statistics on device data (fy_hist_accumulate_u8, fy_flat_noise,
 * fy_noise_aniso; fysics.h:79, 95, 214-215). fy_gpu_hist_accumulate_u8 adds the counts of a
 * device u8 chunk to d_hist, 256 unsigned 64-bit counters in device memory. The other two
 * take d_scratch of fy_gpu_calib_scratch_bytes(nz, ny, nx, blk) bytes (blk: the noise
 * floor's block size; the anisotropy uses 8) and leave their result in device memory: the
 * noise floor as one double, the anisotropy as an fy_aniso_result whose status is
 * fy_noise_aniso's return value. All enqueue on `stream` without synchronising, except
 * fy_gpu_noise_aniso on a volume of fewer than 64 blocks, which writes status 1 and
 * waits for that copy. */
typedef struct { double rho_z, rho_xy; int status; } fy_aniso_result;
int    fy_gpu_hist_accumulate_u8(const unsigned char *d_chunk, size_t n, unsigned long long *d_hist,
                                 void *stream);
size_t fy_gpu_calib_scratch_bytes(int nz, int ny, int nx, int blk);
int    fy_gpu_flat_noise(const float *d_v, int nz, int ny, int nx, int blk, double *d_floor,
                         void *d_scratch, void *stream);
int    fy_gpu_noise_aniso(const float *d_v, int nz, int ny, int nx, fy_aniso_result *d_out,
                          void *d_scratch, void *stream);

/* Device-resident ring state for chains (fy_dering's arrays live on the GPU). accumulate
 * adds a device u8 region at global (z0,y0,x0) into slab z0/slab_z (accumulate + merge);
 * finalize runs the sector vote on the device; apply subtracts on a device f32 region and
 * is a no-op when fewer than 2 radii were detected; download copies the state into a host
 * fy_dering created with fy_dering_init on the same geometry. */
typedef struct fy_gpu_dering fy_gpu_dering;
int  fy_gpu_dering_create(fy_gpu_dering **out, long Z, long Y, long X, double cy, double cx,
                          int slab_z, int ns);
void fy_gpu_dering_destroy(fy_gpu_dering *h);
int  fy_gpu_dering_reset(fy_gpu_dering *h, void *stream);
int  fy_gpu_dering_accumulate_u8(fy_gpu_dering *h, const unsigned char *d_buf, long z0, long y0,
                                 long x0, long dz, long dy, long dx, int ss, void *stream);
int  fy_gpu_dering_finalize(fy_gpu_dering *h, int hp_win, unsigned int min_cnt, double min_amp,
                            double max_amp, void *stream);
int  fy_gpu_dering_apply(const fy_gpu_dering *h, float *d_f, long z0, long y0, long x0, long dz,
                         long dy, long dx, double scale, void *stream);
int  fy_gpu_dering_download(const fy_gpu_dering *h, fy_dering *d, long *detected, void *stream);

/* Device form of fy_zarr_read (no reference counterpart): assembles the region into d_out
 * (device memory, dz*dy*dx) on `stream`, with the same semantics; returns once the copies and
 * the gather are enqueued. The chunks it reads stay in the device chunk cache until that work
 * has run. fy_gpu_zarr_cache_limit sets the cache's device-memory limit per GPU (default
 * 4 GiB, at least 16 MiB); fy_gpu_zarr_cache_stats reports chunk hits, chunk loads and the
 * bytes loaded from chunk files since the library loaded. */
int    fy_gpu_zarr_read(const fy_zarr *z, long z0, long y0, long x0, long dz, long dy, long dx,
                        unsigned char *d_out, void *stream);
int    fy_gpu_zarr_cache_limit(size_t bytes);
void   fy_gpu_zarr_cache_stats(unsigned long long *hits, unsigned long long *loads,
                               unsigned long long *bytes_loaded);

/* Autotuner (no reference counterpart). fy_gpu_autotune times the restoration chain
 * (fy_gpu_restore_u8 with the matched anisotropic deconvolution, noise window 5, exact guided
 * filter r 2) on a scratch cube of this shape on the calling thread's device, varies one
 * launch-shape knob at a time -- the lines per CTA of the forward and inverse deconvolution X
 * passes -- keeps each change that is faster, and writes the winners to the tuning cache, one
 * JSON object per line, keyed by GPU model, SM count, driver and runtime versions and the
 * knob (pass and padded axis length). Every knob only splits the work
 * differently, so results stay bit-identical. The cache file is $FY_TUNE_CACHE, else
 * $XDG_CACHE_HOME/fysics_b200/tune.json, else ~/.cache/fysics_b200/tune.json; later calls
 * and processes read it on first use. It allocates scratch (about 5 bytes per voxel) and
 * synchronises the device: call it at set-up. flags bit 0 re-measures shapes already in the
 * cache. fy_gpu_tune_load replaces the in-memory table with a cache file's entries (NULL:
 * the default path) and returns how many it read; fy_gpu_tune_value returns the tuned value
 * of a knob on the current device ("x1.512", "x5.512"), 0 when untuned.
 * FY_TUNE=0 in the environment makes every lookup use the defaults. */
int    fy_gpu_autotune(int nz, int ny, int nx, int flags);
int    fy_gpu_tune_load(const char *path);
int    fy_gpu_tune_value(const char *knob);

/* Phase correlation of `npairs` device volume pairs (fixed[i], moving[i] at a stride of
 * nz*ny*nx floats) with fy_phase_correlate's semantics (fysics.h:311-313). d_scratch holds
 * fy_gpu_phase_correlate_scratch_bytes(). Results go to host arrays: shift[3*npairs],
 * peak[npairs] and peak_index[npairs] (nullable; flat index of the integer peak in the
 * power-of-two padded surface), status[npairs] (0 ok, 1 degenerate input). Synchronises
 * `stream` before returning. */
size_t fy_gpu_phase_correlate_scratch_bytes(int nz, int ny, int nx);
int    fy_gpu_phase_correlate_batch(const float *d_fixed, const float *d_moving, int npairs,
                                    int nz, int ny, int nx, int window, void *d_scratch,
                                    double *shift, double *peak, long long *peak_index,
                                    int *status, void *stream);

/* Radial guided-eps model. The reference computes it inside fy_run_pipeline
 * (pipeline.c:851-891, 445-456) and has no public function for it. Least squares
 * fn(r) = a + b*r of the calibration noise floors against their distance from the rotation
 * axis, in FP64. have = 1 when the reference's gate passes: n >= 8, b > 0, corr >= 0.5,
 * fn(0) > 0 and fn(rmax)/fn(0) >= 1.3. median is the median floor (0.015 without samples).
 * guided_eps = (k*median)^2 with k = denoise_k (0 -> 4.2); 0 when denoise_k < 0. */
typedef struct {
    double a, b, corr;
    double median;
    double guided_eps;
    int    have;
    int    n;
} fy_radial_eps;
/* n <= 256 samples on the device; the model is written to d_fit (device memory). */
int    fy_gpu_fit_radial_eps(const double *d_rads, const double *d_floors, int n, double denoise_k,
                             fy_radial_eps *d_fit, void *stream);
/* Host form of the same fit (runs on the device, synchronous). */
int    fy_fit_radial_eps(const double *rads, const double *floors, int n, double denoise_k,
                         fy_radial_eps *out);
/* eps of the tile (y0, x0, ty, tx) around the axis (ecy, ecx): guided_eps times
 * clamp((fn(r)/median)^2, 0.4, 8), or 0 when the model is off (pipeline.c:447-456).
 * Host arithmetic only: no device is needed. */
double fy_radial_tile_eps(const fy_radial_eps *fit, double guided_eps, double ecy, double ecx,
                          long y0, long x0, long ty, long tx);

/* The per-cube restoration chain on device buffers: dewindow (fused into the
 * deconvolution) -> Wiener deconvolution -> noise model -> guided filter with
 * eps = fy_guided_eps_for_noise(noise_ref) taken on the device -> ring subtraction.
 * No host round trip inside. Workspaces are the calling thread's. */
typedef struct {
    int    deconv_kind;          /* 0 fy_deconvolve, 1 fy_deconvolve_matched, 2 anisotropic Paganin */
    double deconv_param;         /* reg / tikhonov; <= 0 takes the entry point's default */
    double fz2_scale;            /* kind 2: (sigma_z/sigma_xy)^2 */
    int    noise_win;            /* fy_estimate_noise arguments */
    double noise_flat_pct;
    double noise_ref_intensity;
    double guided_eps;           /* > 0: fixed eps instead of the noise model */
    int    guided_radius;
    int    guided_s;             /* <= 1 exact, >= 2 decimated fast variant */
    fy_gpu_dering *dering;       /* NULL: no ring removal */
    int    dering_accumulate;    /* 1: accumulate this cube's u8 input and vote before applying */
    int    dering_ss;
    int    dering_hp_win;
    unsigned int dering_min_cnt;
    double dering_min_amp, dering_max_amp;
    double dering_scale;         /* ring u8 units -> output units */
    long   z0, y0, x0;           /* global offset of the cube (ring and radial geometry) */
    const fy_radial_eps *radial; /* device model from fy_gpu_fit_radial_eps, or NULL: when it is
                                    on, the guided eps is scaled for the cube centre's distance
                                    from (radial_cy, radial_cx), as pipeline.c:447-456 */
    double radial_cy, radial_cx;
} fy_restore_cfg;
void fy_restore_cfg_default(fy_restore_cfg *cfg);
int  fy_gpu_restore_u8(const unsigned char *d_u8, float *d_out, int nz, int ny, int nx,
                       double f32_min, double f32_max, const fy_physics *p,
                       const fy_restore_cfg *cfg, void *stream);

/* A batch of device-resident volumes of any sizes through the same chain in one call (no
 * reference counterpart; the reference runs its tiles in an OpenMP loop, pipeline.c:1008-1020).
 * Each volume has its own dewindow range and physics; cfg is shared. The deconvolutions
 * run on several streams, the two box passes (noise statistics, guided output) run as one
 * work-queue launch each over every volume's (tile, z chunk) items, and the noise model's
 * selection as one launch per step over all volumes. Each output equals fy_gpu_restore_u8's
 * for that volume bit for bit. The batched form covers the model's eps with the shared
 * noise/guided window (noise_win = 2*guided_radius + 1, guided_s <= 1) without rings or a
 * radial model, for volumes whose x extent is a multiple of 4; other configurations run the
 * volumes one by one through fy_gpu_restore_u8. Enqueued on `stream` (NULL: legacy
 * default stream), not synchronised; the thread's batch buffers grow to the batch's need
 * (about 24 bytes per voxel plus eight half spectra of the largest volume). */
typedef struct {
    const unsigned char *u8;    /* device, nz*ny*nx */
    float *out;                 /* device, nz*ny*nx floats (may not alias u8) */
    int nz, ny, nx;
    double f32_min, f32_max;    /* dewindow range (fy_u8_to_phys) */
    fy_physics phys;
} fy_batch_cube;
int  fy_gpu_restore_u8_batch(const fy_batch_cube *cubes, int n, const fy_restore_cfg *cfg, void *stream);

/* fy_process_buffer on device buffers: d_u8 (hz*hy*hx) in, d_out (tz*ty*tx) out, on
 * `stream`. Synchronises the stream twice: after the all-air test (an empty buffer skips
 * the chain, as the reference does) and at the end, so that *all_air and the status are
 * final on return. */
int    fy_gpu_process_buffer(const fy_pipeline_cfg *cfg, const unsigned char *d_u8,
                             long rz0, long ry0, long rx0, long hz, long hy, long hx,
                             long z0, long y0, long x0, long tz, long ty, long tx,
                             long vol_y, long vol_x, unsigned char *d_out, int *all_air, void *stream);
/* fy_measure_psf_sigma on a device u8 tile; d_out (16 bytes of device memory) receives
 * { double sigma; int nprof; }. Enqueued on `stream`, no synchronisation. */
int    fy_gpu_measure_psf_sigma(const unsigned char *d_vol, int Z, int Y, int X, void *d_out, void *stream);
/* Air-cut state of the calling thread's last fy_process_buffer / fy_gpu_process_buffer:
 * the 256-bin histogram of the scratch smooth and (cut, uniform cut, textured cut) in u8
 * levels. Returns 0, or 1 when that call ran no air cut. */
int    fy_process_buffer_air_state(long hist[256], int cuts[3]);

/* Request loop (continuous batching) on one GPU; no reference counterpart. Callers submit
 * cubes from any thread as they need them. A pool of worker threads, each with its own CUDA
 * stream and device workspaces, runs the restoration chain of several requests at once, so
 * their kernels and their host<->device copies overlap on the device. A request is
 * admitted in arrival order when a worker is free and the estimated device memory of the
 * requests in flight stays within hbm_budget_bytes (reserved small-request workers may take
 * a small request out of order); a request larger than the whole budget
 * is refused at submission. Each result equals the single-cube fy_gpu_restore_u8 call. */
typedef struct fy_server fy_server;
typedef struct {
    size_t hbm_budget_bytes;     /* device memory admitted at once (default 150 GB) */
    int    workers;              /* requests executing at once (default 8) */
    int    device;
    size_t priority_voxels;      /* requests up to this size run on high-priority streams
                                    (default 256^3), so small cubes keep low latency beside
                                    large ones; copies move in 32 MB chunks for the same reason */
    int    small_workers;        /* workers reserved for requests up to priority_voxels (default
                                    2); they may take a small request from behind a large one */
    int    reserve_nz, reserve_ny, reserve_nx;  /* > 0: every worker sizes its device workspaces for
                                    this cube at start, so serving up to that size allocates
                                    nothing (a workspace that grows frees its old buffer, and a
                                    free synchronises the device); 0: grow on demand */
} fy_server_cfg;
typedef struct {
    const unsigned char *u8;     /* input, nz*ny*nx: host (pinned avoids a staging copy) or, together
                                    with out, device memory (the chain then runs in place, no copies) */
    float *out;                  /* output, nz*ny*nx floats: host, or device when u8 is */
    int    nz, ny, nx;
    double f32_min, f32_max;     /* dewindow range (fy_u8_to_phys) */
    fy_physics phys;
    fy_restore_cfg cfg;          /* dering: a finalised handle, applied only (no accumulation) */
} fy_request;
typedef struct {
    int    status;
    double queue_ms, run_ms, latency_ms;   /* submit -> start, start -> done, submit -> done */
    /* device-side phases from CUDA events on the worker's stream: input copy, the chain
     * (including time its kernels waited for other requests' work), output copy */
    double h2d_ms, chain_ms, d2h_ms;
} fy_request_result;
typedef struct {
    long long completed;
    double voxels, mvox_per_s;   /* over completed requests, first start to last completion */
    double p50_ms, p99_ms;       /* nearest-rank latency percentiles, submit -> done */
    int    inflight, queued;
} fy_server_stats;
void fy_server_cfg_default(fy_server_cfg *cfg);
int  fy_server_create(fy_server **out, const fy_server_cfg *cfg);
/* The request's buffers must stay valid until fy_server_wait returns for its ticket. */
int  fy_server_submit(fy_server *s, const fy_request *req, long long *ticket);
/* timeout_ms < 0 waits without limit; FY_ETIMEDOUT leaves the ticket pending. */
int  fy_server_wait(fy_server *s, long long ticket, double timeout_ms, fy_request_result *res);
int  fy_server_get_stats(fy_server *s, fy_server_stats *out);
void fy_server_reset_stats(fy_server *s);
/* Finishes running requests, cancels queued ones (FY_EBUSY) and joins the workers. */
void fy_server_destroy(fy_server *s);

/* Per-kernel timing: CUDA events recorded on the launching stream after every launch of
 * the instrumented kernels. read(i) gives mark i's name and the ms since mark i-1, once
 * the stream has been synchronised. */
int fy_gpu_profile_start(int capacity, void *stream);
int fy_gpu_profile_stop(void);
int fy_gpu_profile_read(int i, const char **name, float *ms);
/* Record only the marks named in `names` (comma-separated, e.g. "noise,guided"; each mark's
 * span then runs from the previous recorded mark); NULL or "" records every mark. Each event
 * between two launches costs the pair its overlap, so a timed loop records few. */
int fy_gpu_profile_select(const char *names);

#ifdef __cplusplus
}
#endif
#endif /* FYSICS_B200_H */
