/* fy_oracle64.h -- FP64 CPU restatement of the fysics restoration hot path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker): tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg may call it; the product library never links or loads it.
 *
 * Every routine restates the reference algorithm in double precision with the reference's
 * index conventions (row-major, x fastest, idx = (z*ny+y)*nx+x), citing the fysics source
 * line it follows. Differences from the reference are deliberate and listed per function:
 * the Wiener weight is evaluated directly (no 4096-entry LUT), FFTs and box sums are double.
 * Parity pin: tests/test_oracle_pins.py checks this file against the reference's own
 * known-answer tests and against the reference library compiled from source.
 */
#ifndef FY_ORACLE64_H
#define FY_ORACLE64_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* same layout as fysics.h:23-35 (8 doubles) */
typedef struct {
    double delta_beta, energy_kev, distance_mm, pixel_um;
    double unsharp_sigma, unsharp_coeff, psf_sigma_vox, psf_sigma_z_vox;
} o64_physics;

int    o64_next_fft_size(int n);
int    o64_next_pow2(int n);
/* in-place complex FFT of interleaved (re,im) doubles, any n = 2^a 3^b; sign -1 fwd */
void   o64_fft1d(double *x, int n, int sign);
void   o64_fft3d(double *x, int nz, int ny, int nx, int sign);

void   o64_u8_to_phys(const uint8_t *in, double *out, size_t n, double f32_min, double f32_max);

double o64_paganin_transfer(double f, const o64_physics *p);
double o64_unsharp_transfer(double f, const o64_physics *p);
double o64_recon_transfer(double f, const o64_physics *p);
double o64_auto_deltabeta_scale(const o64_physics *p);

/* kind 0 = fy_deconvolve Wiener (param=reg, cap 8), kind 1 = fy_deconvolve_matched
 * (param=tikhonov), kind 2 = Paganin Wiener with an anisotropic z scale (param=reg,
 * cap 8, fz2_scale given). use_lut: 1 = the reference's weight LUT (in double), 0 = the
 * weight evaluated directly. Returns 0. */
int    o64_deconvolve(const double *in, double *out, int nz, int ny, int nx,
                      const o64_physics *p, double param, int kind, double fz2_scale, int use_lut);

void   o64_box_mean(const double *in, double *out, int nz, int ny, int nx, int r);
int    o64_guided(const double *in, double *out, int nz, int ny, int nx, int r, double eps);
int    o64_guided_fast(const double *in, double *out, int nz, int ny, int nx,
                       int r, double eps, int s);

typedef struct { double g, b, noise_ref, ref_intensity; int n_bins_used; } o64_noise_model;
int    o64_estimate_noise(const float *in, int nz, int ny, int nx, int win, double flat_pct,
                          double ref_intensity, o64_noise_model *out);
/* the same on a double volume (the FP64 chain's deconvolved output) */
int    o64_estimate_noise64(const double *in, int nz, int ny, int nx, int win, double flat_pct,
                            double ref_intensity, o64_noise_model *out);
double o64_guided_eps_for_noise(double noise_ref);

/* dering: exact 64-bit integer sums; geometry identical to fy_dering_init. */
int    o64_dering_nr(long Y, long X, double cy, double cx);
void   o64_dering_accumulate_u8(const uint8_t *buf, long y0, long x0, long dz, long dy, long dx,
                                int ss, double cy, double cx, int ns, int nr,
                                uint64_t *sum, uint64_t *cnt);
long   o64_dering_finalize(const uint64_t *sum, const uint64_t *cnt, int nslab, int ns, int nr,
                           int hp_win, unsigned min_cnt, double min_amp, double max_amp,
                           double *ring, int *have_rings);
void   o64_dering_apply(const double *ring, int nslab, int nr, int slab_z, double cy, double cx,
                        double *f, long z0, long y0, long x0, long dz, long dy, long dx,
                        double scale);

int    o64_phase_correlate(const double *fixed, const double *moving, int nz, int ny, int nx,
                           double *shift, double *peak, int window, long *peak_index);

/* radial eps fit (pipeline.c:856-877): returns 1 and fills a,b when the gate passes */
int    o64_fit_radial_eps(const double *rads, const double *floors, int n,
                          double *a, double *b, double *corr);
/* median of the noise floors, pipeline.c:74-78 and :878 (0.015 when n == 0) */
double o64_median_floor(const double *v, int n);
/* per-tile eps, pipeline.c:447-456 (0 = use the global eps) */
double o64_radial_tile_eps(int have, double a, double b, double median, double guided_eps,
                           double ecy, double ecx, long y0, long x0, long ty, long tx);

/* calibration statistics (pass 1 of the pipeline) */
/* counts of every u8 value of v[0, n) added to hist[256] (stream.c:76-86) */
void   o64_hist_u8(const uint8_t *v, size_t n, long long *hist);
/* 10th-percentile std over the bright (mean > 0.1) non-overlapping blk^3 blocks
 * (stream.c:174-200); blk < 4 means 8; 0 without blocks */
double o64_flat_noise(const float *v, int nz, int ny, int nx, int blk);
/* lag-1 noise autocorrelation per axis in flat 8^3 blocks (noise.c:210-269); 0 on success */
int    o64_noise_aniso(const float *v, int nz, int ny, int nx, double *rho_z, double *rho_xy);

#ifdef __cplusplus
}
#endif
#endif
