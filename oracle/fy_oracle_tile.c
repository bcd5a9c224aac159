/* fy_oracle_tile.c -- CPU restatement of the reference's per-tile chain
 * (fy_process_buffer / process_tile, pipeline.c:252-510).
 *
 * TEST INFRASTRUCTURE ONLY (the checker): tests/, __graft_entry__.smoke() and bench.py's
 * CPU legs may call it; the product library never links or loads it.
 *
 * Precision contract. The chain's decisions are float comparisons (air cut, texture split,
 * material > 0) and a float quantiser, so this file restates them in float with the
 * reference source's operation order, and with a*b+c forms fused (fmaf) as the reference
 * build (-Ofast, FMA target) contracts them. Two stages are FP64: the deconvolution and the
 * guided filter go through o64_deconvolve / o64_guided_fast and are rounded to float on
 * the way back. A division by a constant is a multiplication by the constant's rounded
 * reciprocal (x / 255.0f -> x * (1.0f / 255.0f)), as the reference build folds it
 * (-freciprocal-math); divisions by variables are IEEE. Deliberate differences from the
 * compiled reference:
 *   - the box smooth's 1/count is IEEE. The reference build vectorises box_recip
 *     (guided.c:22-28) with an rcpps + Newton sequence whose last bit depends on the host
 *     CPU, so its scratch smooth is not reproducible across machines;
 *   - connected components are found by union-find, not breadth-first search; the set of
 *     zeroed voxels is the same by construction (it depends on component membership only).
 * The GPU chain follows this file operation for operation; where the deconvolution and
 * guided filter are off, the two agree bit for bit.
 * Parity pin: tests/test_tile_oracle.py checks this file against the reference library
 * compiled from source (u8 outputs within a mismatch bound, integer stages exactly).
 */
#include "fy_oracle_tile.h"
#include "fy_oracle64.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* stream.c:138-168 */
double ot_valley_depth(const long hist[256], int *dark_out, int *light_out, int *valley_out) {
    double hf[256];
    for (int i = 0; i < 256; i++) {
        long s = 0;
        int cnt = 0;
        for (int j = i - 2; j <= i + 2; j++)
            if (j >= 0 && j < 256) { s += hist[j]; cnt++; }
        hf[i] = (double)s / cnt;
    }
    hf[0] = 0; hf[254] = 0; hf[255] = 0;
    double mx = 0;
    for (int i = 0; i < 256; i++) mx = hf[i] > mx ? hf[i] : mx;
    if (mx <= 0) return -1;
    int pk[256], np = 0;                       /* local maxima above 5% of max, 10-bin merge */
    for (int u = 3; u < 253; u++) {
        if (!(hf[u] >= hf[u - 1] && hf[u] >= hf[u + 1] && hf[u] > 0.05 * mx)) continue;
        if (np > 0 && u - pk[np - 1] <= 10) {
            if (hf[u] > hf[pk[np - 1]]) pk[np - 1] = u;
        } else {
            pk[np++] = u;
        }
    }
    if (np < 2) return -1;
    int p1 = pk[0], p2 = pk[1];                /* the two tallest */
    for (int i = 0; i < np; i++) {
        const int u = pk[i];
        if (hf[u] > hf[p1]) { p2 = p1; p1 = u; }
        else if (hf[u] > hf[p2] && u != p1) p2 = u;
    }
    const int a = p1 < p2 ? p1 : p2, b = p1 < p2 ? p2 : p1;
    int v = a;
    double vmin = hf[a];
    for (int u = a; u <= b; u++)
        if (hf[u] < vmin) { vmin = hf[u]; v = u; }
    if (dark_out) *dark_out = a;
    if (light_out) *light_out = b;
    if (valley_out) *valley_out = v;
    const double mn = hf[a] < hf[b] ? hf[a] : hf[b];
    return 1.0 - vmin / (mn + 1e-12);
}

/* One line of guided.c:34-98's sliding sum: prime with [0, r], then emit s * recip and
 * slide (add the entering sample, then subtract the leaving one). */
static void box_line(const float *in, long st, int L, int r, float *out, long ost) {
    float s = 0.0f;
    for (int i = 0; i <= r && i < L; i++) s += in[i * st];
    for (int i = 0; i < L; i++) {
        const int lo = i - r < 0 ? 0 : i - r, hi = i + r > L - 1 ? L - 1 : i + r;
        out[i * ost] = s * (1.0f / (float)(hi - lo + 1));
        if (i + r + 1 < L) s += in[(i + r + 1) * st];
        if (i - r >= 0) s -= in[(i - r) * st];
    }
}

/* fy_box_smooth (guided.c:104-106): X, then Y, then Z sliding means; in/out may alias */
void ot_box_smooth(const float *in, float *out, int nz, int ny, int nx, int r) {
    const size_t n = (size_t)nz * ny * nx;
    float *t1 = malloc(sizeof(float) * n), *t2 = malloc(sizeof(float) * n);
    for (long z = 0; z < nz; z++)
        for (long y = 0; y < ny; y++) box_line(in + (z * ny + y) * nx, 1, nx, r, t1 + (z * ny + y) * nx, 1);
    for (long z = 0; z < nz; z++)
        for (long x = 0; x < nx; x++) box_line(t1 + z * ny * nx + x, nx, ny, r, t2 + z * ny * nx + x, nx);
    for (long y = 0; y < ny; y++)
        for (long x = 0; x < nx; x++)
            box_line(t2 + y * nx + x, (long)ny * nx, nz, r, out + y * nx + x, (long)ny * nx);
    free(t1);
    free(t2);
}

static long uf_find(long *p, long i) {
    while (p[i] != i) { p[i] = p[p[i]]; i = p[i]; }
    return i;
}

/* pipeline.c:223-250: zero every 6-connected component of f > 0 that touches no face of
 * the buffer and has fewer than min_size voxels. Returns the number of voxels zeroed. */
long ot_cc_despeckle(float *f, int nz, int ny, int nx, int min_size) {
    const long n = (long)nz * ny * nx, plane = (long)ny * nx;
    long *p = malloc(sizeof(long) * n), *size = calloc(n, sizeof(long));
    unsigned char *edge = calloc(n, 1);
    for (long i = 0; i < n; i++) p[i] = i;
    for (long z = 0; z < nz; z++)
        for (long y = 0; y < ny; y++)
            for (long x = 0; x < nx; x++) {
                const long i = (z * ny + y) * nx + x;
                if (!(f[i] > 0.0f)) continue;
                const long nb[3] = {x > 0 ? i - 1 : -1, y > 0 ? i - nx : -1, z > 0 ? i - plane : -1};
                for (int k = 0; k < 3; k++) {
                    if (nb[k] < 0 || !(f[nb[k]] > 0.0f)) continue;
                    const long a = uf_find(p, i), b = uf_find(p, nb[k]);
                    if (a != b) p[a > b ? a : b] = a < b ? a : b;
                }
            }
    for (long z = 0; z < nz; z++)
        for (long y = 0; y < ny; y++)
            for (long x = 0; x < nx; x++) {
                const long i = (z * ny + y) * nx + x;
                if (!(f[i] > 0.0f)) continue;
                const long root = uf_find(p, i);
                size[root]++;
                if (z == 0 || z == nz - 1 || y == 0 || y == ny - 1 || x == 0 || x == nx - 1) edge[root] = 1;
            }
    long zeroed = 0;
    for (long i = 0; i < n; i++) {
        if (!(f[i] > 0.0f)) continue;
        const long root = uf_find(p, i);
        if (!edge[root] && size[root] < min_size) { f[i] = 0.0f; zeroed++; }
    }
    free(p);
    free(size);
    free(edge);
    return zeroed;
}

/* pipeline.c:53-58: integer hash of the global voxel coordinate -> [0, 1) */
float ot_dither01(long z, long y, long x) {
    unsigned h = (unsigned)z * 73856093u ^ (unsigned)y * 19349663u ^ (unsigned)x * 83492791u;
    h ^= h >> 16;
    h *= 0x7feb352du;
    h ^= h >> 15;
    h *= 0x846ca68bu;
    h ^= h >> 16;
    return (float)(h >> 8) * (1.0f / 16777216.0f);
}

/* pipeline.c:60-65 */
uint8_t ot_quant_u8(float v, long gz, long gy, long gx, int no_dither) {
    const float t = fmaf(v, 255.0f, no_dither ? 0.5f : ot_dither01(gz, gy, gx));
    if (t <= 0.0f) return 0;
    const int q = (int)t;
    return q > 255 ? 255 : (uint8_t)q;
}

/* The air-cut decision of pipeline.c:336-368 from the scratch histogram. Writes the
 * value cut and the texture-split cuts (uniform, textured), all in u8 levels. */
void ot_air_cuts(const long hist[256], int air_cut_u8, int air_cut_band, double air_thresh, double air_cut_aggr,
                 int *cut_out, int *cut_uni, int *cut_tex) {
    int dark = 0, light = 0, valley = 0;
    const double d = ot_valley_depth(hist, &dark, &light, &valley);
    const int pf = air_thresh > 0 ? (int)fma(air_thresh, 255.0, 0.5) : 39;
    int cut;
    if (air_cut_u8 >= 0) {
        const int gg = air_cut_u8, band = air_cut_band;
        if (d >= 0) {
            double a = air_cut_aggr;
            a = a < 0 ? 0 : (a > 2 ? 2 : a);
            int local;
            if (valley <= pf) local = pf;
            else if (a <= 1.0) local = (int)(fma(a, (double)(valley - pf), (double)pf) + 0.5);
            else local = (int)(fma(a - 1.0, (double)(light > valley ? light - valley : 0), (double)valley) + 0.5);
            cut = local < gg - band ? gg - band : (local > gg + band ? gg + band : local);
        } else {
            cut = gg;
        }
    } else if (d >= 0) {
        const int mid = (dark + valley) / 2;
        cut = dark + 8 < mid ? dark + 8 : mid;
    } else {
        cut = (int)((air_thresh > 0 ? air_thresh : 0.05) * 255);
    }
    const int spread = valley > pf ? (valley - pf) / 2 : 8;          /* pipeline.c:373-378 */
    int cu = cut + spread;
    if (valley > cut && cu > valley) cu = valley;
    int ct = cut - spread;
    if (ct < pf) ct = pf;
    *cut_out = cut;
    *cut_uni = cu;
    *cut_tex = ct;
}

static int hist_bin(float v) {
    int b = (int)fmaf(v, 255.0f, 0.5f);
    return b < 0 ? 0 : (b > 255 ? 255 : b);
}

/* pipeline.c:252-443 for one haloed tile in f (in/out); orig = the pre-deconvolution copy */
static int tile_chain(const ot_tile_cfg *c, float *f, const float *orig, int nz, int ny, int nx, long *hist_out,
                      int *cuts_out) {
    const size_t N = (size_t)nz * ny * nx;
    if (c->do_deconv) {                                               /* (b) */
        o64_physics ph = {c->delta_beta, c->energy_kev, c->distance_mm, c->pixel_um, c->unsharp_sigma,
                          c->unsharp_coeff, c->psf_sigma_vox,
                          (c->psf_z_ratio > 1.0 && c->psf_sigma_vox > 0) ? c->psf_z_ratio * c->psf_sigma_vox : 0.0};
        ph.delta_beta *= o64_auto_deltabeta_scale(&ph);
        const int windowed = c->window_hi > c->window_lo;
        const float wlo = (float)c->window_lo, wspan = (float)(c->window_hi - c->window_lo);
        double *a = malloc(sizeof(double) * N), *b = malloc(sizeof(double) * N);
        for (size_t i = 0; i < N; i++) a[i] = windowed ? fmaf(f[i], wspan, wlo) : f[i];
        const int matched = c->use_matched_deconv && c->psf_sigma_vox > 0;
        o64_deconvolve(a, b, nz, ny, nx, &ph, matched ? c->deconv_tikhonov : -1.0, matched ? 1 : 0, 1.0, 1);
        const float inv = windowed ? 1.0f / wspan : 1.0f;
        const int rescale = c->have_dec_range && c->dec_hi - c->dec_lo > 1e-6;
        const float lo = (float)c->dec_lo, dinv = rescale ? 1.0f / (float)(c->dec_hi - c->dec_lo) : 1.0f;
        for (size_t i = 0; i < N; i++) {
            float v = (float)b[i];
            if (windowed) v = (v - wlo) * inv;
            if (rescale) v = (v - lo) * dinv;
            f[i] = v < 0.0f ? 0.0f : (v > 1.0f ? 1.0f : v);
        }
        free(a);
        free(b);
    }
    if (c->guided_eps > 0 || c->tile_eps > 0) {                      /* (c) */
        const double eps = c->tile_eps > 0 ? c->tile_eps : c->guided_eps;
        const int gs = c->guided_subsample == 0 ? 2 : c->guided_subsample;
        double *a = malloc(sizeof(double) * N), *b = malloc(sizeof(double) * N);
        for (size_t i = 0; i < N; i++) a[i] = f[i];
        /* eps reaches the filter as a float (the reference's guided filter is float) */
        o64_guided_fast(a, b, nz, ny, nx, 2, (double)(float)eps, gs);
        for (size_t i = 0; i < N; i++) f[i] = (float)b[i];
        free(a);
        free(b);
    }
    if (c->do_air_zero) {                                             /* (d) */
        const int sr = c->scratch_passes > 0 ? c->scratch_passes : 5;
        long hist[256];
        memset(hist, 0, sizeof hist);
        const int lz = (nz + 1) / 2, ly = (ny + 1) / 2, lx = (nx + 1) / 2;
        const size_t nl = (size_t)lz * ly * lx;
        const int lowres = lz >= 2 && ly >= 2 && lx >= 2;
        float *sm = malloc(sizeof(float) * (lowres ? nl : N));
        if (lowres) {
            float *dec = malloc(sizeof(float) * nl);
            for (long z = 0; z < lz; z++)
                for (long y = 0; y < ly; y++)
                    for (long x = 0; x < lx; x++)
                        dec[(z * ly + y) * lx + x] = orig[((2 * z) * ny + 2 * y) * nx + 2 * x];
            int rl = (sr + 1) / 2;
            if (rl < 1) rl = 1;
            ot_box_smooth(dec, sm, lz, ly, lx, rl);
            free(dec);
            for (size_t i = 0; i < nl; i++) hist[hist_bin(sm[i])]++;
        } else {
            ot_box_smooth(orig, sm, nz, ny, nx, sr);
            for (size_t i = 0; i < N; i++) hist[hist_bin(sm[i])]++;
        }
        int cut, cu, ct;
        ot_air_cuts(hist, c->air_cut_u8, c->air_cut_band, c->air_thresh, c->air_cut_aggr, &cut, &cu, &ct);
        if (hist_out) memcpy(hist_out, hist, sizeof hist);
        if (cuts_out) { cuts_out[0] = cut; cuts_out[1] = cu; cuts_out[2] = ct; }
        const float cutf_uni = (float)cu * (1.0f / 255.0f), cutf_tex = (float)ct * (1.0f / 255.0f);
        const float AIR_TEX = 0.03f;
        if (lowres) {
            for (long z = 0; z < nz; z++) {
                long z0 = z >> 1;
                if (z0 > lz - 2) z0 = lz - 2;
                float zf = 0.5f * (float)z - (float)z0;
                if (zf > 1.0f) zf = 1.0f;
                for (long y = 0; y < ny; y++) {
                    long y0 = y >> 1;
                    if (y0 > ly - 2) y0 = ly - 2;
                    float yf = 0.5f * (float)y - (float)y0;
                    if (yf > 1.0f) yf = 1.0f;
                    const size_t r00 = ((size_t)z0 * ly + y0) * lx, r01 = r00 + lx;
                    const size_t r10 = r00 + (size_t)ly * lx, r11 = r10 + lx;
                    const float w00 = (1 - zf) * (1 - yf), w01 = (1 - zf) * yf, w10 = zf * (1 - yf), w11 = zf * yf;
                    for (long x = 0; x < nx; x++) {
                        long x0 = x >> 1;
                        if (x0 > lx - 2) x0 = lx - 2;
                        float fx = 0.5f * (float)x - (float)x0;
                        if (fx > 1.0f) fx = 1.0f;
                        /* the row blend at x0 and x0 + 1 (pipeline.c:397-399); every weight is
                         * a product of 0, 1/2 and 1, so each product is exact */
                        const float a0 = w00 * sm[r00 + x0] + w01 * sm[r01 + x0] + w10 * sm[r10 + x0] +
                                         w11 * sm[r11 + x0];
                        const float a1 = w00 * sm[r00 + x0 + 1] + w01 * sm[r01 + x0 + 1] +
                                         w10 * sm[r10 + x0 + 1] + w11 * sm[r11 + x0 + 1];
                        const float v = fmaf(a1 - a0, fx, a0);
                        const size_t i = ((size_t)z * ny + y) * nx + x;
                        const float tex = fabsf(orig[i] - v);
                        if (v < (tex < AIR_TEX ? cutf_uni : cutf_tex)) f[i] = 0.0f;
                    }
                }
            }
        } else {
            for (size_t i = 0; i < N; i++) {
                const float tex = fabsf(orig[i] - sm[i]);
                if (sm[i] < (tex < AIR_TEX ? cutf_uni : cutf_tex)) f[i] = 0.0f;
            }
        }
        free(sm);
        if (c->air_min_component > 0) ot_cc_despeckle(f, nz, ny, nx, c->air_min_component);
    }
    if (c->have_norm && c->norm_hi > c->norm_lo) {                  /* (d.5) */
        const float midf = 0.5f * (float)(c->norm_lo + c->norm_hi) * (1.0f / 255.0f);
        const float k = (2.0f * 0.375f) * 255.0f / (float)(c->norm_hi - c->norm_lo);
        for (size_t i = 0; i < N; i++) {
            if (f[i] <= 0.0f) { f[i] = 0.0f; continue; }
            const float v = 0.5f + (f[i] - midf) * k;     /* not fused in the reference build */
            f[i] = v < 0.0f ? 0.0f : (v > 1.0f ? 1.0f : v);
        }
    }
    return 0;
}

int ot_process_buffer(const ot_tile_cfg *c, const uint8_t *u8buf, long rz0, long ry0, long rx0, long hz, long hy,
                      long hx, long z0, long y0, long x0, long tz, long ty, long tx, uint8_t *out, int *all_air,
                      long *hist_out, int *cuts_out) {
    const size_t hn = (size_t)hz * hy * hx;
    int any = 0;
    for (size_t i = 0; i < hn && !any; i++) any = u8buf[i] != 0;
    if (!any) {                                                       /* pipeline.c:472-476 */
        memset(out, 0, (size_t)tz * ty * tx);
        if (all_air) *all_air = 1;
        return 0;
    }
    if (c->do_musica) return 2;                                       /* not restated */
    float *f = malloc(sizeof(float) * hn), *orig = malloc(sizeof(float) * hn);
    for (size_t i = 0; i < hn; i++) f[i] = (float)u8buf[i] * (1.0f / 255.0f);
    if (c->ring && c->nr > 0 && c->nslab > 0) {                       /* dering.c:200-248, scale 1/255 */
        const float sc = (float)(1.0 / 255.0);
        for (long z = 0; z < hz; z++) {
            long s = (rz0 + z) / c->slab_z;
            s = s < 0 ? 0 : (s >= c->nslab ? c->nslab - 1 : s);
            const float *ring = c->ring + (size_t)s * c->nr;
            for (long y = 0; y < hy; y++) {
                const double gy = (double)(ry0 + y) - c->ring_cy;
                for (long x = 0; x < hx; x++) {
                    const double gx = (double)(rx0 + x) - c->ring_cx;
                    const int ri = (int)(sqrt(gy * gy + gx * gx) + 0.5);
                    float *v = f + ((size_t)z * hy + y) * hx + x;
                    if (ri >= c->nr || *v <= 0.0f) continue;
                    const float w = fmaf(-sc, ring[ri], *v);
                    *v = w > 0.0f ? w : 0.0f;
                }
            }
        }
    }
    if (c->zdrift)                                                    /* zdrift.c:64-71 */
        for (long z = 0; z < hz; z++) {
            const float fz = c->zdrift[rz0 + z];
            for (size_t i = 0; i < (size_t)hy * hx; i++) f[(size_t)z * hy * hx + i] *= fz;
        }
    memcpy(orig, f, sizeof(float) * hn);
    tile_chain(c, f, orig, (int)hz, (int)hy, (int)hx, hist_out, cuts_out);
    size_t oi = 0;                                                    /* pipeline.c:500-505 */
    for (long zz = z0 - rz0; zz < z0 - rz0 + tz; zz++)
        for (long yy = y0 - ry0; yy < y0 - ry0 + ty; yy++)
            for (long xx = x0 - rx0; xx < x0 - rx0 + tx; xx++)
                out[oi++] = ot_quant_u8(f[((size_t)zz * hy + yy) * hx + xx], rz0 + zz, ry0 + yy, rx0 + xx,
                                        c->no_dither);
    if (all_air) *all_air = 0;
    free(f);
    free(orig);
    return 0;
}

/* ---------------------------------------------------------------- PSF edge fit
 * measure_tile_psf_sigma (pipeline.c:107-196): effective PSF sigma (voxels) from air/papyrus
 * edge profiles of a u8 tile. Candidate lines come from the reference's LCG, reseeded to 1
 * per call (:111-112, :124); up to 2500 candidates per axis (y lines, then x lines), the
 * first 400 accepted edges kept in candidate order. The edge normalisation is a true
 * division (a reciprocal there flipped an edge decision against the compiled reference);
 * acc / nprof and lsf / lsum are multiplications by the reciprocal, and
 * e[i]*(1-f) + e[i+1]*f is fused. The final reductions (lsum, mu, var) are sequential
 * here; the reference build vectorises them, so sigma agrees to rounding (1e-15 measured),
 * and nprof and the accepted set exactly.
 * Returns sigma or -1; *nprof_out receives the number of profiles. */
static unsigned ot_psf_rand(unsigned *s) {
    *s = *s * 1103515245u + 12345u;
    return (*s >> 16) & 0x7fff;
}

/* one candidate: returns 1 and fills e[15], *cross when the line is an accepted edge */
static int ot_psf_candidate(const uint8_t *vol, int Z, int Y, int X, int ax, unsigned *rng, double *e,
                            double *cross) {
    const int half = 7, plen = 15, min_c = 40;
    int line[15];
    if (ax == 1) {
        const int z = (int)(ot_psf_rand(rng) % (unsigned)Z);
        const int y = half + (int)(ot_psf_rand(rng) % (unsigned)(Y - 2 * half));
        const int x = (int)(ot_psf_rand(rng) % (unsigned)X);
        for (int i = 0; i < plen; i++) line[i] = vol[((size_t)z * Y + (y - half + i)) * X + x];
    } else {
        const int z = (int)(ot_psf_rand(rng) % (unsigned)Z);
        const int y = (int)(ot_psf_rand(rng) % (unsigned)Y);
        const int x = half + (int)(ot_psf_rand(rng) % (unsigned)(X - 2 * half));
        for (int i = 0; i < plen; i++) line[i] = vol[((size_t)z * Y + y) * X + (x - half + i)];
    }
    const double lo = 0.5 * (line[0] + line[1]), hi = 0.5 * (line[plen - 1] + line[plen - 2]);
    if (fabs(hi - lo) < min_c) return 0;
    int s[15];
    for (int i = 0; i < plen; i++) s[i] = hi > lo ? line[i] : line[plen - 1 - i];
    double dmin = 1e9, dmax = -1e9;
    int amax = 0;
    for (int i = 0; i < plen - 1; i++) {
        const double d = (double)s[i + 1] - s[i];
        if (d < dmin) dmin = d;
        if (d > dmax) { dmax = d; amax = i; }
    }
    if (dmin < -8) return 0;
    if (!(amax == half - 1 || amax == half || amax == half + 1)) return 0;
    int smin = s[0];
    for (int i = 1; i < plen; i++) smin = s[i] < smin ? s[i] : smin;
    double emax = 0;
    for (int i = 0; i < plen; i++) { e[i] = s[i] - smin; emax = e[i] > emax ? e[i] : emax; }
    if (emax <= 0) return 0;
    for (int i = 0; i < plen; i++) e[i] /= emax;
    int idx0 = -1;
    for (int i = 0; i < plen; i++)
        if (e[i] >= 0.5) { idx0 = i; break; }
    if (idx0 <= 0) return 0;
    const double frac = (0.5 - e[idx0 - 1]) / (e[idx0] - e[idx0 - 1] + 1e-9);
    *cross = idx0 - 1 + frac;
    return 1;
}

double ot_measure_psf_sigma(const uint8_t *vol, int Z, int Y, int X, int *nprof_out) {
    enum { HALF = 7, SUP = 8, PLEN = 15, GLEN = 2 * HALF * SUP + 1, MAXE = 400 };
    static double esf_p[MAXE][PLEN], cross_p[MAXE];
    double grid[GLEN], acc[GLEN], esf[GLEN], lsf[GLEN];
    for (int i = 0; i < GLEN; i++) { grid[i] = -HALF + (double)i * (2.0 * HALF) / (GLEN - 1); acc[i] = 0; }
    unsigned rng = 1u;
    int nprof = 0;
    for (int ax = 1; ax <= 2 && nprof < MAXE; ax++) {
        if ((ax == 1 ? Y : X) - 2 * HALF <= 0) continue;      /* the reference breaks before any draw */
        for (int it = 0; it < 2500 && nprof < MAXE; it++)
            if (ot_psf_candidate(vol, Z, Y, X, ax, &rng, esf_p[nprof], &cross_p[nprof])) nprof++;
    }
    if (nprof_out) *nprof_out = nprof;
    if (nprof < 30) return -1.0;
    for (int p = 0; p < nprof; p++)
        for (int gi = 0; gi < GLEN; gi++) {
            const double xs = grid[gi] + cross_p[p];
            double v;
            if (xs <= 0) v = 0.0;
            else if (xs >= PLEN - 1) v = 1.0;
            else {
                const int i = (int)xs;
                const double f = xs - i;
                v = fma(esf_p[p][i + 1], f, esf_p[p][i] * (1.0 - f));
            }
            acc[gi] += v;
        }
    const double rn = 1.0 / nprof;
    for (int gi = 0; gi < GLEN; gi++) esf[gi] = acc[gi] * rn;
    double lsum = 0;
    for (int gi = 0; gi < GLEN; gi++) {
        double d;
        if (gi == 0) d = esf[1] - esf[0];
        else if (gi == GLEN - 1) d = esf[GLEN - 1] - esf[GLEN - 2];
        else d = 0.5 * (esf[gi + 1] - esf[gi - 1]);
        if (d < 0) d = 0;
        lsf[gi] = d;
        lsum += d;
    }
    if (!(lsum > 0)) return -1.0;
    const double rl = 1.0 / lsum;
    double mu = 0, var = 0;
    for (int gi = 0; gi < GLEN; gi++) { lsf[gi] *= rl; mu = fma(grid[gi], lsf[gi], mu); }
    for (int gi = 0; gi < GLEN; gi++) { const double g = grid[gi] - mu; var = fma(g * g, lsf[gi], var); }
    const double sig = sqrt(var);
    return (sig > 0.3 && sig < 5.0) ? sig : -1.0;
}
