/* fy_oracle_tile.h -- CPU restatement of the reference's per-tile chain
 * (fy_process_buffer, pipeline.c:252-510). Test infrastructure only; see fy_oracle_tile.c
 * for the precision contract.
 */
#ifndef FY_ORACLE_TILE_H
#define FY_ORACLE_TILE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* The fields of fy_pipeline_cfg (fysics.h:436-491) the tile chain reads, resolved: the
 * ring table and z-drift factors are plain arrays and tile_eps is eps_for_tile's value. */
typedef struct {
    double delta_beta, energy_kev, distance_mm, pixel_um, unsharp_sigma, unsharp_coeff;
    double window_lo, window_hi;
    int do_deconv, use_matched_deconv;
    double psf_sigma_vox, deconv_tikhonov, psf_z_ratio;
    int have_dec_range;
    double dec_lo, dec_hi;
    double guided_eps;
    int guided_subsample;
    double tile_eps;                 /* > 0 overrides guided_eps (radial fit) */
    int do_air_zero, air_cut_u8, air_cut_band;
    double air_thresh, air_cut_aggr;
    int air_min_component, scratch_passes;
    int have_norm, norm_lo, norm_hi;
    int do_musica, no_dither;
    const float *ring;               /* [nslab][nr] ring profile in u8 units, NULL = none */
    int nslab, nr, slab_z;
    double ring_cy, ring_cx;
    const float *zdrift;             /* per global z, NULL = none */
} ot_tile_cfg;

double  ot_valley_depth(const long hist[256], int *dark_out, int *light_out, int *valley_out);
void    ot_box_smooth(const float *in, float *out, int nz, int ny, int nx, int r);
long    ot_cc_despeckle(float *f, int nz, int ny, int nx, int min_size);
float   ot_dither01(long z, long y, long x);
uint8_t ot_quant_u8(float v, long gz, long gy, long gx, int no_dither);
void    ot_air_cuts(const long hist[256], int air_cut_u8, int air_cut_band, double air_thresh,
                    double air_cut_aggr, int *cut, int *cut_uni, int *cut_tex);
/* Returns 0, or 2 when do_musica is set (MUSICA is not restated). hist_out (256 longs) and
 * cuts_out (cut, uniform cut, textured cut) receive the air-cut state when non-NULL. */
int     ot_process_buffer(const ot_tile_cfg *c, const uint8_t *u8buf, long rz0, long ry0, long rx0,
                          long hz, long hy, long hx, long z0, long y0, long x0, long tz, long ty,
                          long tx, uint8_t *out, int *all_air, long *hist_out, int *cuts_out);

/* measure_tile_psf_sigma (pipeline.c:107-196): sigma or -1; *nprof_out = edge profiles used */
double  ot_measure_psf_sigma(const uint8_t *vol, int Z, int Y, int X, int *nprof_out);

#ifdef __cplusplus
}
#endif
#endif
