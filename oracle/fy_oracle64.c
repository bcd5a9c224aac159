/* fy_oracle64.c -- FP64 CPU restatement of the fysics restoration hot path.
 *
 * TEST INFRASTRUCTURE ONLY: this is the checker. The product library (fysics_b200) never
 * links, loads or calls it; only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg do.
 *
 * Each function restates the reference algorithm (fysics, C11) in double precision and
 * cites the reference lines it follows. It is written from the algorithm, not copied:
 * FFTs are a double-precision mixed-radix Stockham transform, the Wiener weight is
 * evaluated directly per frequency instead of through the reference's LUT, and the ring
 * accumulator uses exact 64-bit integer sums.
 */
#include "fy_oracle64.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ---------------------------------------------------------------- FFT sizes
 * fft.c:25-38: 2^k, or 3*2^k when that is smaller. */
int o64_next_pow2(int n) { int p = 1; while (p < n) p <<= 1; return p; }
int o64_next_fft_size(int n) {
    int p2 = o64_next_pow2(n);
    int p3 = 3 * o64_next_pow2((n + 2) / 3);
    return (p3 >= n && p3 < p2) ? p3 : p2;
}

/* ---------------------------------------------------------------- double FFT
 * Unnormalised DFT X[k] = sum_t x[t] exp(sign*2*pi*i*k*t/n), the convention of
 * fy_fft1d (fft.c:168-173). Mixed-radix Stockham over the prime factors of n, with a
 * per-size table w[m] = exp(+2*pi*i*m/n) evaluated in double (sign applied to sin). */
typedef struct { int n; double *c, *s; } o64_tw;

static o64_tw tw_make(int n) {
    o64_tw t = {n, malloc(sizeof(double) * (size_t)n), malloc(sizeof(double) * (size_t)n)};
    for (int m = 0; m < n; m++) {
        t.c[m] = cos(2.0 * M_PI * (double)m / (double)n);
        t.s[m] = sin(2.0 * M_PI * (double)m / (double)n);
    }
    return t;
}
static void tw_free(o64_tw *t) { free(t->c); free(t->s); }

static void fft_stockham(double *a, double *b, int n, int sign, const o64_tw *tw) {
    int Ns = 1;
    double *src = a, *dst = b;
    int m = n;
    while (m > 1) {
        int R = (m % 3 == 0) ? 3 : (m % 2 == 0 ? 2 : m);
        m /= R;
        int nr = n / R;
        int step = n / (Ns * R);                 /* w_(Ns*R) = w_n^step */
        for (int j = 0; j < nr; j++) {
            int k = j % Ns;
            double vr[8], vi[8];
            for (int r = 0; r < R; r++) {
                int idx = (int)(((long)r * k * step) % n);
                double c = tw->c[idx], s = sign * tw->s[idx];
                double xr = src[2 * (j + r * nr)], xi = src[2 * (j + r * nr) + 1];
                vr[r] = xr * c - xi * s; vi[r] = xr * s + xi * c;
            }
            int base = (j / Ns) * Ns * R + k;
            for (int q = 0; q < R; q++) {
                double sr = 0, si = 0;
                for (int r = 0; r < R; r++) {
                    int idx = ((q * r) % R) * nr;        /* w_R^(qr) = w_n^(qr*n/R) */
                    double c = tw->c[idx], s = sign * tw->s[idx];
                    sr += vr[r] * c - vi[r] * s; si += vr[r] * s + vi[r] * c;
                }
                dst[2 * (base + q * Ns)] = sr; dst[2 * (base + q * Ns) + 1] = si;
            }
        }
        double *t = src; src = dst; dst = t;
        Ns *= R;
    }
    if (src != a) memcpy(a, src, sizeof(double) * 2 * (size_t)n);
}

void o64_fft1d(double *x, int n, int sign) {
    if (n <= 1) return;
    double *tmp = malloc(sizeof(double) * 2 * (size_t)n);
    o64_tw tw = tw_make(n);
    fft_stockham(x, tmp, n, sign, &tw);
    tw_free(&tw);
    free(tmp);
}

static void fft_lines(double *x, int n, int sign, size_t nlines, size_t line_stride, size_t elem_stride) {
    if (n <= 1) return;
    double *line = malloc(sizeof(double) * 2 * (size_t)n), *tmp = malloc(sizeof(double) * 2 * (size_t)n);
    o64_tw tw = tw_make(n);
    for (size_t L = 0; L < nlines; L++) {
        double *base = x + 2 * L * line_stride;
        for (int i = 0; i < n; i++) { line[2 * i] = base[2 * i * elem_stride]; line[2 * i + 1] = base[2 * i * elem_stride + 1]; }
        fft_stockham(line, tmp, n, sign, &tw);
        for (int i = 0; i < n; i++) { base[2 * i * elem_stride] = line[2 * i]; base[2 * i * elem_stride + 1] = line[2 * i + 1]; }
    }
    tw_free(&tw);
    free(line); free(tmp);
}

/* axis-by-axis 3-D transform, fy_fft3d (fft.c:178-220) */
void o64_fft3d(double *x, int nz, int ny, int nx, int sign) {
    fft_lines(x, nx, sign, (size_t)nz * ny, (size_t)nx, 1);                    /* X */
    for (int z = 0; z < nz; z++)                                               /* Y */
        fft_lines(x + 2 * (size_t)z * ny * nx, ny, sign, (size_t)nx, 1, (size_t)nx);
    fft_lines(x, nz, sign, (size_t)ny * nx, 1, (size_t)ny * nx);               /* Z */
}

/* ---------------------------------------------------------------- dewindow
 * stream.c:41-46: phys = f32_min + u8 * (f32_max - f32_min)/255, here in double. */
void o64_u8_to_phys(const uint8_t *in, double *out, size_t n, double f32_min, double f32_max) {
    double scale = (f32_max - f32_min) / 255.0;
    for (size_t i = 0; i < n; i++) out[i] = f32_min + in[i] * scale;
}

/* ---------------------------------------------------------------- transfers
 * paganin.c:15-44 (nabu form; pixel < 0.1 um is read as mm). */
double o64_paganin_transfer(double f, const o64_physics *p) {
    double lam = 1.23984199e-3 / p->energy_kev;
    double dist = p->distance_mm * 1000.0;
    double px = p->pixel_um;
    if (px > 0.0 && px < 0.1) px *= 1000.0;
    double fu = f / px;
    return 1.0 / (1.0 + p->delta_beta * lam * dist * M_PI * fu * fu);
}
double o64_unsharp_transfer(double f, const o64_physics *p) {
    if (p->unsharp_coeff == 0.0 || p->unsharp_sigma == 0.0) return 1.0;
    double s = p->unsharp_sigma;
    return 1.0 + p->unsharp_coeff * (1.0 - exp(-2.0 * M_PI * M_PI * s * s * f * f));
}
double o64_recon_transfer(double f, const o64_physics *p) {
    double h = o64_paganin_transfer(f, p) * o64_unsharp_transfer(f, p);
    return h < 1e-4 ? 1e-4 : h;
}
/* paganin.c:80-91 */
double o64_auto_deltabeta_scale(const o64_physics *p) {
    double h = o64_paganin_transfer(0.5, p);
    if (!isfinite(h) || h <= 0) return 1.0;
    if (h <= 0.0025) return 0.35;
    if (h >= 0.0070) return 1.0;
    return 0.35 + (h - 0.0025) / (0.0070 - 0.0025) * 0.65;
}

/* radial weights: wiener_weight (paganin.c:296-299, cap paganin.c:50) and
 * matched_transfer (paganin.c:321-328) */
static double weight_at(double fr, const o64_physics *p, double param, int kind) {
    if (kind == 1) {
        double sg = p->psf_sigma_vox > 0 ? p->psf_sigma_vox : 1.0;
        double g = exp(-2.0 * M_PI * M_PI * sg * sg * fr * fr);
        double hf = g * o64_unsharp_transfer(fr, p);
        return hf / (hf * hf + param);
    }
    double h = o64_recon_transfer(fr, p);
    double w = h / (h * h + param);
    return w > 8.0 ? 8.0 : w;
}

/* paganin.c:121-128 */
static int reflect_idx(int i, int n) {
    if (n == 1) return 0;
    while (i < 0 || i >= n) {
        if (i < 0) i = -i - 1;
        if (i >= n) i = 2 * n - i - 1;
    }
    return i;
}

/* deconv_radial (paganin.c:152-293) restated on the FULL complex spectrum in double:
 * reflect-pad to fy_next_fft_size per axis, forward FFT, multiply by the radial weight at
 * u = fz^2*fz2_scale + fy^2 + fx^2, inverse, 1/N, crop. use_lut = 1 follows the reference's
 * 4096-entry linear-interpolation LUT over u (paganin.c:223-244) with double entries, so the
 * comparison isolates FP32 rounding; use_lut = 0 evaluates the weight directly at sqrt(u)
 * (the exact operator; its gap to use_lut = 1 is the LUT's own approximation error). */
int o64_deconvolve(const double *in, double *out, int nz, int ny, int nx,
                   const o64_physics *p, double param, int kind, double fz2_scale, int use_lut) {
    if (kind == 0) { if (param <= 0) param = 0.015; fz2_scale = 1.0; }          /* paganin.c:305 */
    if (kind == 1) {                                                           /* paganin.c:333-340 */
        if (param <= 0) param = 0.05;
        double sxy = p->psf_sigma_vox > 0 ? p->psf_sigma_vox : 1.0;
        fz2_scale = 1.0;
        if (p->psf_sigma_z_vox > 0) { double rr = p->psf_sigma_z_vox / sxy; fz2_scale = rr * rr; }
    }
    if (kind == 2 && param <= 0) param = 0.015;
    if (fz2_scale <= 0) fz2_scale = 1.0;
    int pz = o64_next_fft_size(nz), py = o64_next_fft_size(ny), px = o64_next_fft_size(nx);
    size_t np = (size_t)pz * py * px;
    double *c = calloc(2 * np, sizeof(double));
    if (!c) return 1;
    for (int z = 0; z < pz; z++)
        for (int y = 0; y < py; y++) {
            const double *row = in + ((size_t)reflect_idx(z, nz) * ny + reflect_idx(y, ny)) * nx;
            for (int x = 0; x < px; x++) c[2 * (((size_t)z * py + y) * px + x)] = row[reflect_idx(x, nx)];
        }
    o64_fft3d(c, pz, py, px, -1);
    /* LUT over u = f^2 exactly as paganin.c:217-244 but with double entries; max f^2 per
     * axis taken over the half-spectrum x range, as the reference does. */
    enum { LUTN = 4096 };
    double lut[LUTN + 1], us = 0;
    if (use_lut) {
        double mz = 0, my = 0, mx = 0;
        for (int i = 0; i < pz; i++) { double f = (i <= pz / 2) ? (double)i / pz : (double)(i - pz) / pz; if (f * f * fz2_scale > mz) mz = f * f * fz2_scale; }
        for (int i = 0; i < py; i++) { double f = (i <= py / 2) ? (double)i / py : (double)(i - py) / py; if (f * f > my) my = f * f; }
        for (int i = 0; i <= px / 2; i++) { double f = (double)i / px; if (f * f > mx) mx = f * f; }
        double umax = mz + my + mx;
        us = umax > 0 ? LUTN / umax : 0.0;
        for (int i = 0; i <= LUTN; i++) lut[i] = weight_at(us > 0 ? sqrt((double)i / us) : 0.0, p, param, kind);
    }
    for (int z = 0; z < pz; z++) {
        double fz = (z <= pz / 2) ? (double)z / pz : (double)(z - pz) / pz;
        for (int y = 0; y < py; y++) {
            double fy = (y <= py / 2) ? (double)y / py : (double)(y - py) / py;
            for (int x = 0; x < px; x++) {
                double fx = (x <= px / 2) ? (double)x / px : (double)(x - px) / px;
                double u = fz * fz * fz2_scale + fy * fy + fx * fx, w;
                if (use_lut) {
                    double t = u * us;
                    int ti = (int)t;
                    if (ti >= LUTN) ti = LUTN - 1;
                    w = lut[ti] + (lut[ti + 1] - lut[ti]) * (t - ti);
                } else {
                    w = weight_at(sqrt(u), p, param, kind);
                }
                size_t o = ((size_t)z * py + y) * px + x;
                c[2 * o] *= w; c[2 * o + 1] *= w;
            }
        }
    }
    o64_fft3d(c, pz, py, px, +1);
    double inv = 1.0 / (double)np;
    for (int z = 0; z < nz; z++)
        for (int y = 0; y < ny; y++)
            for (int x = 0; x < nx; x++)
                out[((size_t)z * ny + y) * nx + x] = c[2 * (((size_t)z * py + y) * px + x)] * inv;
    free(c);
    return 0;
}

/* ---------------------------------------------------------------- box mean
 * guided.c:19-98: mean over the IN-BOUNDS part of the (2r+1)^3 window (each axis divides
 * by its own clamped count), here as exact double window sums. */
static void box_axis(const double *in, double *out, int nz, int ny, int nx, int r, int axis) {
    int len = axis == 0 ? nz : (axis == 1 ? ny : nx);
    size_t st = axis == 0 ? (size_t)ny * nx : (axis == 1 ? (size_t)nx : 1);
    for (int z = 0; z < nz; z++)
        for (int y = 0; y < ny; y++)
            for (int x = 0; x < nx; x++) {
                int pos = axis == 0 ? z : (axis == 1 ? y : x);
                int lo = pos - r < 0 ? 0 : pos - r, hi = pos + r > len - 1 ? len - 1 : pos + r;
                size_t i = ((size_t)z * ny + y) * nx + x;
                const double *b = in + i - (size_t)pos * st;
                double s = 0;
                for (int j = lo; j <= hi; j++) s += b[(size_t)j * st];
                out[i] = s / (double)(hi - lo + 1);
            }
}
void o64_box_mean(const double *in, double *out, int nz, int ny, int nx, int r) {
    size_t n = (size_t)nz * ny * nx;
    double *t = malloc(sizeof(double) * n);
    box_axis(in, out, nz, ny, nx, r, 2);
    box_axis(out, t, nz, ny, nx, r, 1);
    box_axis(t, out, nz, ny, nx, r, 0);
    free(t);
}

/* guided.c:113-137: mean, corr, var=max(corr-mean^2,0), a=var/(var+eps), b=mean(1-a),
 * out = box(a)*I + box(b); radius < 1 -> 2 */
int o64_guided(const double *in, double *out, int nz, int ny, int nx, int r, double eps) {
    if (r < 1) r = 2;
    size_t n = (size_t)nz * ny * nx;
    double *m = malloc(sizeof(double) * n), *c = malloc(sizeof(double) * n);
    double *a = malloc(sizeof(double) * n), *b = malloc(sizeof(double) * n);
    if (!m || !c || !a || !b) { free(m); free(c); free(a); free(b); return 1; }
    o64_box_mean(in, m, nz, ny, nx, r);
    for (size_t i = 0; i < n; i++) a[i] = in[i] * in[i];
    o64_box_mean(a, c, nz, ny, nx, r);
    for (size_t i = 0; i < n; i++) {
        double v = c[i] - m[i] * m[i];
        if (v < 0) v = 0;
        a[i] = v / (v + eps);
        b[i] = m[i] * (1.0 - a[i]);
    }
    o64_box_mean(a, m, nz, ny, nx, r);
    o64_box_mean(b, c, nz, ny, nx, r);
    for (size_t i = 0; i < n; i++) out[i] = m[i] * in[i] + c[i];
    free(m); free(c); free(a); free(b);
    return 0;
}

/* guided.c:152-231: decimated (sample, not mean) coefficients with radius max(1,r/s),
 * trilinear upsample with the same clamps (x0 <= l-2, frac <= 1). */
int o64_guided_fast(const double *in, double *out, int nz, int ny, int nx,
                    int r, double eps, int s) {
    if (r < 1) r = 2;
    if (s <= 1) return o64_guided(in, out, nz, ny, nx, r, eps);
    int lz = (nz + s - 1) / s, ly = (ny + s - 1) / s, lx = (nx + s - 1) / s;
    if (lz < 2 || ly < 2 || lx < 2) return o64_guided(in, out, nz, ny, nx, r, eps);
    size_t nl = (size_t)lz * ly * lx;
    double *il = malloc(sizeof(double) * nl), *m = malloc(sizeof(double) * nl);
    double *c = malloc(sizeof(double) * nl), *a = malloc(sizeof(double) * nl);
    double *b = malloc(sizeof(double) * nl);
    for (int z = 0; z < lz; z++)
        for (int y = 0; y < ly; y++)
            for (int x = 0; x < lx; x++)
                il[((size_t)z * ly + y) * lx + x] = in[((size_t)(z * s) * ny + (size_t)y * s) * nx + (size_t)x * s];
    int rl = r / s; if (rl < 1) rl = 1;
    o64_box_mean(il, m, lz, ly, lx, rl);
    for (size_t i = 0; i < nl; i++) a[i] = il[i] * il[i];
    o64_box_mean(a, c, lz, ly, lx, rl);
    for (size_t i = 0; i < nl; i++) {
        double v = c[i] - m[i] * m[i];
        if (v < 0) v = 0;
        a[i] = v / (v + eps);
        b[i] = m[i] * (1.0 - a[i]);
    }
    o64_box_mean(a, m, lz, ly, lx, rl);
    o64_box_mean(b, c, lz, ly, lx, rl);
    for (int z = 0; z < nz; z++) {
        double uz = (double)z / s; int z0 = (int)uz; if (z0 > lz - 2) z0 = lz - 2;
        double fz = uz - z0; if (fz > 1) fz = 1;
        for (int y = 0; y < ny; y++) {
            double uy = (double)y / s; int y0 = (int)uy; if (y0 > ly - 2) y0 = ly - 2;
            double fy = uy - y0; if (fy > 1) fy = 1;
            for (int x = 0; x < nx; x++) {
                double ux = (double)x / s; int x0 = (int)ux; if (x0 > lx - 2) x0 = lx - 2;
                double fx = ux - x0; if (fx > 1) fx = 1;
                double av = 0, bv = 0;
                for (int dz = 0; dz < 2; dz++)
                    for (int dy = 0; dy < 2; dy++)
                        for (int dx = 0; dx < 2; dx++) {
                            double w = (dz ? fz : 1 - fz) * (dy ? fy : 1 - fy) * (dx ? fx : 1 - fx);
                            size_t li = ((size_t)(z0 + dz) * ly + (y0 + dy)) * lx + (x0 + dx);
                            av += w * m[li]; bv += w * c[li];
                        }
                size_t i = ((size_t)z * ny + y) * nx + x;
                out[i] = av * in[i] + bv;
            }
        }
    }
    free(il); free(m); free(c); free(a); free(b);
    return 0;
}

/* ---------------------------------------------------------------- noise model
 * noise.c:20-59 box SUM with zero outside the volume; noise.c:66-73 interpolated
 * percentile; noise.c:75-192 binning + IRLS. */
static void box_sum_axis(const double *in, double *out, int nz, int ny, int nx, int r, int axis) {
    int len = axis == 0 ? nz : (axis == 1 ? ny : nx);
    size_t st = axis == 0 ? (size_t)ny * nx : (axis == 1 ? (size_t)nx : 1);
    for (int z = 0; z < nz; z++)
        for (int y = 0; y < ny; y++)
            for (int x = 0; x < nx; x++) {
                int pos = axis == 0 ? z : (axis == 1 ? y : x);
                int lo = pos - r < 0 ? 0 : pos - r, hi = pos + r > len - 1 ? len - 1 : pos + r;
                size_t i = ((size_t)z * ny + y) * nx + x;
                const double *b = in + i - (size_t)pos * st;
                double s = 0;
                for (int j = lo; j <= hi; j++) s += b[(size_t)j * st];
                out[i] = s;
            }
}
static void box_sum3(const double *in, double *out, double *tmp, int nz, int ny, int nx, int r) {
    box_sum_axis(in, out, nz, ny, nx, r, 2);
    box_sum_axis(out, tmp, nz, ny, nx, r, 1);
    box_sum_axis(tmp, out, nz, ny, nx, r, 0);
}
static int cmp_dbl(const void *a, const void *b) {
    double x = *(const double *)a, y = *(const double *)b;
    return (x > y) - (x < y);
}
static double pct_sorted(double *v, long n, double pct) {
    if (n <= 0) return 0.0;
    qsort(v, (size_t)n, sizeof(double), cmp_dbl);
    double idx = pct / 100.0 * (double)(n - 1);
    long lo = (long)idx; double f = idx - (double)lo;
    if (lo + 1 < n) return v[lo] * (1 - f) + v[lo + 1] * f;
    return v[lo];
}

/* The float input of the reference's API (inf), or a double volume (ind) for the FP64
 * chain, whose stages pass double data from one to the next. */
static int noise_impl(const float *inf, const double *ind, int nz, int ny, int nx, int win, double flat_pct,
                      double ref_intensity, o64_noise_model *out) {
    if (!out) return 1;
    if (win < 3) win = 5;
    if (flat_pct <= 0) flat_pct = 10.0;
    int r = win / 2;
    size_t n = (size_t)nz * ny * nx;
    double *x = malloc(sizeof(double) * n), *s1 = malloc(sizeof(double) * n);
    double *s2 = malloc(sizeof(double) * n), *t = malloc(sizeof(double) * n);
    if (!x || !s1 || !s2 || !t) { free(x); free(s1); free(s2); free(t); return 1; }
    for (size_t i = 0; i < n; i++) x[i] = inf ? (double)inf[i] : ind[i];
    box_sum3(x, s1, t, nz, ny, nx, r);
    for (size_t i = 0; i < n; i++) x[i] = x[i] * x[i];
    box_sum3(x, s2, t, nz, ny, nx, r);
    double wc = (double)win * win * win;                 /* fixed divisor, noise.c:92 */
    double *mean = t, *var = s2;
    for (size_t i = 0; i < n; i++) {
        double m = s1[i] / wc, v = s2[i] / wc - m * m;
        mean[i] = m; var[i] = v > 0 ? v : 0;
    }
    memcpy(x, mean, sizeof(double) * n);
    double lo = pct_sorted(x, (long)n, 1.0);
    double hi = pct_sorted(x, (long)n, 99.0);           /* x is sorted now; same result */
    if (hi <= lo) hi = lo + 1e-6;
    enum { NB = 24 };
    double bin_i[NB], bin_f[NB]; long bin_c[NB];
    int used = 0;
    for (int bk = 0; bk < NB; bk++) {
        double b0 = lo + (hi - lo) * bk / NB, b1 = lo + (hi - lo) * (bk + 1) / NB;
        long c = 0;
        for (size_t i = 0; i < n; i++) if (mean[i] >= b0 && mean[i] < b1) x[c++] = var[i];
        if (c < 200) continue;
        bin_f[used] = pct_sorted(x, c, flat_pct);
        bin_i[used] = 0.5 * (b0 + b1);
        bin_c[used] = c;
        used++;
    }
    out->n_bins_used = used;
    double g = 0, b = 0;
    if (used >= 3) {                                      /* IRLS, noise.c:139-161 */
        double w[NB];
        for (int i = 0; i < used; i++) w[i] = sqrt((double)bin_c[i]);
        for (int it = 0; it < 4; it++) {
            double sw = 0, swx = 0, swy = 0, swxx = 0, swxy = 0;
            for (int i = 0; i < used; i++) {
                sw += w[i]; swx += w[i] * bin_i[i]; swy += w[i] * bin_f[i];
                swxx += w[i] * bin_i[i] * bin_i[i]; swxy += w[i] * bin_i[i] * bin_f[i];
            }
            double det = sw * swxx - swx * swx;
            if (fabs(det) < 1e-20) break;
            g = (sw * swxy - swx * swy) / det;
            b = (swxx * swy - swx * swxy) / det;
            double res[NB], rc[NB];
            for (int i = 0; i < used; i++) { res[i] = fabs(bin_f[i] - (g * bin_i[i] + b)); rc[i] = res[i]; }
            double med = pct_sorted(rc, used, 50.0) + 1e-9;
            for (int i = 0; i < used; i++) {
                double rr = res[i] / (2.0 * med);
                w[i] = sqrt((double)bin_c[i]) / (1.0 + rr * rr);
            }
        }
    } else if (used > 0) {
        double s = 0; for (int i = 0; i < used; i++) s += bin_f[i];
        b = s / used; g = 0;
    } else {
        memcpy(x, var, sizeof(double) * n);
        b = pct_sorted(x, (long)n, flat_pct); g = 0;
    }
    if (!isfinite(g)) g = 0;
    if (!isfinite(b)) b = 0;
    out->g = g; out->b = b;
    double vr = g * ref_intensity + b;
    if (vr < 0) vr = b > 0 ? b : 0;
    out->noise_ref = sqrt(vr) * 1.15;                     /* noise.c:181-187 */
    out->ref_intensity = ref_intensity;
    free(x); free(s1); free(s2); free(t);
    return 0;
}

int o64_estimate_noise(const float *in, int nz, int ny, int nx, int win, double flat_pct,
                       double ref_intensity, o64_noise_model *out) {
    return noise_impl(in, NULL, nz, ny, nx, win, flat_pct, ref_intensity, out);
}

int o64_estimate_noise64(const double *in, int nz, int ny, int nx, int win, double flat_pct,
                         double ref_intensity, o64_noise_model *out) {
    return noise_impl(NULL, in, nz, ny, nx, win, flat_pct, ref_intensity, out);
}

/* noise.c:197-202 */
double o64_guided_eps_for_noise(double noise_ref) {
    double e = (3.0 * noise_ref) * (3.0 * noise_ref);
    return (e > 1e-8) ? e : 1e-8;
}

/* ---------------------------------------------------------------- dering
 * dering.c:40-42 radial bin count */
int o64_dering_nr(long Y, long X, double cy, double cx) {
    if (cy < 0) cy = (Y - 1) / 2.0;
    if (cx < 0) cx = (X - 1) / 2.0;
    double ry = cy > Y - 1 - cy ? cy : Y - 1 - cy;
    double rx = cx > X - 1 - cx ? cx : X - 1 - cx;
    return (int)sqrt(ry * ry + rx * rx) + 2;
}

/* dering.c:78-116 with exact integer sums */
void o64_dering_accumulate_u8(const uint8_t *buf, long y0, long x0, long dz, long dy, long dx,
                              int ss, double cy, double cx, int ns, int nr,
                              uint64_t *sum, uint64_t *cnt) {
    if (ss < 1) ss = 1;
    double inv_sect = ns / (2.0 * M_PI);
    for (long yi = 0; yi * ss < dy; yi++) {
        double gy = (double)(y0 + yi * ss) - cy;
        for (long xi = 0; xi * ss < dx; xi++) {
            double gx = (double)(x0 + xi * ss) - cx;
            int ri = (int)(sqrt(gy * gy + gx * gx) + 0.5);
            if (ri >= nr) continue;
            int q = (int)((atan2(gy, gx) + M_PI) * inv_sect);
            if (q >= ns) q = ns - 1;
            for (long z = 0; z < dz; z++) {
                uint8_t v = buf[((size_t)z * dy + (size_t)(yi * ss)) * dx + (size_t)(xi * ss)];
                if (!v) continue;
                sum[(size_t)q * nr + ri] += v;
                cnt[(size_t)q * nr + ri] += 1;
            }
        }
    }
}

static int cmp_d2(const void *a, const void *b) {
    double x = *(const double *)a, y = *(const double *)b;
    return (x > y) - (x < y);
}

/* dering.c:136-194 sector sign-consistency vote, in double */
long o64_dering_finalize(const uint64_t *sum, const uint64_t *cnt, int nslab, int ns, int nr,
                         int hp_win, unsigned min_cnt, double min_amp, double max_amp,
                         double *ring, int *have_rings) {
    if (hp_win < 3) hp_win = 15;
    if (min_amp <= 0) min_amp = 0.5;
    if (max_amp <= 0) max_amp = 6.0;
    int hw = hp_win / 2;
    double *p = malloc(sizeof(double) * (size_t)ns * nr), *hp = malloc(sizeof(double) * (size_t)ns * nr);
    unsigned char *vd = malloc((size_t)ns * nr);
    double med[64];
    long det = 0;
    for (int s = 0; s < nslab; s++) {
        const uint64_t *sm = sum + (size_t)s * ns * nr, *cn = cnt + (size_t)s * ns * nr;
        for (int q = 0; q < ns; q++) {
            for (int r = 0; r < nr; r++) {
                size_t i = (size_t)q * nr + r;
                vd[i] = cn[i] >= min_cnt;
                p[i] = vd[i] ? (double)sm[i] / (double)cn[i] : 0.0;
            }
            for (int r = 0; r < nr; r++) {
                size_t i = (size_t)q * nr + r;
                if (!vd[i]) { hp[i] = 0; continue; }
                double acc = 0; int c = 0;
                int lo = r - hw < 0 ? 0 : r - hw, hi = r + hw >= nr ? nr - 1 : r + hw;
                for (int j = lo; j <= hi; j++) if (vd[(size_t)q * nr + j]) { acc += p[(size_t)q * nr + j]; c++; }
                if (c >= hw) hp[i] = p[i] - acc / c;
                else { hp[i] = 0; vd[i] = 0; }
            }
        }
        double *rg = ring + (size_t)s * nr;
        for (int r = 0; r < nr; r++) {
            int nv = 0, pos = 0, neg = 0;
            for (int q = 0; q < ns; q++) {
                size_t i = (size_t)q * nr + r;
                if (!vd[i]) continue;
                med[nv++] = hp[i];
                if (hp[i] > 0) pos++; else if (hp[i] < 0) neg++;
            }
            if (nv < ns - 2 || (pos && neg)) { rg[r] = 0; continue; }
            qsort(med, (size_t)nv, sizeof(double), cmp_d2);
            double m = (nv & 1) ? med[nv / 2] : 0.5 * (med[nv / 2 - 1] + med[nv / 2]);
            if (fabs(m) < min_amp) { rg[r] = 0; continue; }
            if (m > max_amp) m = max_amp;
            if (m < -max_amp) m = -max_amp;
            rg[r] = m;
            det++;
        }
    }
    free(p); free(hp); free(vd);
    if (have_rings) *have_rings = det >= 2;
    return det;
}

/* dering.c:200-248 */
void o64_dering_apply(const double *ring, int nslab, int nr, int slab_z, double cy, double cx,
                      double *f, long z0, long y0, long x0, long dz, long dy, long dx,
                      double scale) {
    for (long z = 0; z < dz; z++) {
        long s = (z0 + z) / slab_z;
        if (s < 0) s = 0;
        if (s >= nslab) s = nslab - 1;
        const double *rg = ring + (size_t)s * nr;
        for (long y = 0; y < dy; y++) {
            double gy = (double)(y0 + y) - cy;
            for (long x = 0; x < dx; x++) {
                double gx = (double)(x0 + x) - cx;
                int ri = (int)(sqrt(gy * gy + gx * gx) + 0.5);
                size_t i = ((size_t)z * dy + y) * dx + x;
                if (ri >= nr || f[i] <= 0) continue;
                double v = f[i] - scale * rg[ri];
                f[i] = v > 0 ? v : 0;
            }
        }
    }
}

/* ---------------------------------------------------------------- phase correlation
 * phasecorr.c:38-186 in double: Hann (phasecorr.c:38-42), means of the unwindowed input,
 * zero-pad to next pow2, cross-power R = conj(F)M/|.| (|.|<=1e-12 -> 0), inverse, argmax
 * (strict >, first index), fftfreq unwrap, Foroosh per axis clamped to +-0.5. */
int o64_phase_correlate(const double *fixed, const double *moving, int nz, int ny, int nx,
                        double *shift, double *peak, int window, long *peak_index) {
    if (!fixed || !moving || !shift || nz < 2 || ny < 2 || nx < 2) return 1;
    int pz = o64_next_pow2(nz), py = o64_next_pow2(ny), px = o64_next_pow2(nx);
    size_t pn = (size_t)pz * py * px, n = (size_t)nz * ny * nx;
    double *F = calloc(2 * pn, sizeof(double)), *M = calloc(2 * pn, sizeof(double));
    double *wz = malloc(sizeof(double) * nz), *wy = malloc(sizeof(double) * ny), *wx = malloc(sizeof(double) * nx);
    int dims[3] = {nz, ny, nx}; double *ws[3] = {wz, wy, wx};
    for (int a = 0; a < 3; a++)
        for (int i = 0; i < dims[a]; i++)
            ws[a][i] = window ? 0.5 - 0.5 * cos(2.0 * M_PI * i / (double)(dims[a] - 1)) : 1.0;
    double sf = 0, sm = 0;
    for (size_t i = 0; i < n; i++) { sf += fixed[i]; sm += moving[i]; }
    double mf = sf / n, mm = sm / n;
    for (int z = 0; z < nz; z++)
        for (int y = 0; y < ny; y++)
            for (int x = 0; x < nx; x++) {
                double w = wz[z] * wy[y] * wx[x];
                size_t i = ((size_t)z * ny + y) * nx + x, o = ((size_t)z * py + y) * px + x;
                F[2 * o] = (fixed[i] - mf) * w;
                M[2 * o] = (moving[i] - mm) * w;
            }
    free(wz); free(wy); free(wx);
    o64_fft3d(F, pz, py, px, -1);
    o64_fft3d(M, pz, py, px, -1);
    double maxmag = 0;
    for (size_t i = 0; i < pn; i++) {
        double fr = F[2 * i], fi = F[2 * i + 1], mr = M[2 * i], mi = M[2 * i + 1];
        double cr = fr * mr + fi * mi, ci = fr * mi - fi * mr;
        double mag = sqrt(cr * cr + ci * ci);
        if (mag > maxmag) maxmag = mag;
        if (mag > 1e-12) { F[2 * i] = cr / mag; F[2 * i + 1] = ci / mag; }
        else { F[2 * i] = 0; F[2 * i + 1] = 0; }
    }
    free(M);
    if (maxmag < 1e-20) { free(F); shift[0] = shift[1] = shift[2] = 0; if (peak) *peak = 0; return 1; }
    o64_fft3d(F, pz, py, px, +1);
    size_t pk = 0; double best = F[0];
    for (size_t i = 1; i < pn; i++) if (F[2 * i] > best) { best = F[2 * i]; pk = i; }
    int kz = (int)(pk / ((size_t)py * px)), ky = (int)((pk / px) % py), kx = (int)(pk % px);
    int k[3] = {kz, ky, kx}, p[3] = {pz, py, px};
    double c0 = best;
    for (int a = 0; a < 3; a++) {
        int km = (k[a] - 1 + p[a]) % p[a], kp = (k[a] + 1) % p[a];
        int im[3] = {kz, ky, kx}, ip[3] = {kz, ky, kx};
        im[a] = km; ip[a] = kp;
        double cm = F[2 * (((size_t)im[0] * py + im[1]) * px + im[2])];
        double cp = F[2 * (((size_t)ip[0] * py + ip[1]) * px + ip[2])];
        double c1 = cp >= cm ? cp : cm, sg = cp >= cm ? 1.0 : -1.0, d = 0;
        if (fabs(c1 - c0) > 1e-20 && fabs(c1 + c0) > 1e-20) {
            double d1 = c1 / (c1 - c0), d2 = c1 / (c1 + c0);
            d = sg * (fabs(d1) <= fabs(d2) ? d1 : d2);
        }
        if (d > 0.5) d = 0.5;
        if (d < -0.5) d = -0.5;
        int iu = k[a] <= p[a] / 2 ? k[a] : k[a] - p[a];
        shift[a] = iu + d;
    }
    if (peak) *peak = best / (double)pn;
    if (peak_index) *peak_index = (long)pk;
    free(F);
    return 0;
}

/* ---------------------------------------------------------------- radial eps fit
 * pipeline.c:860-877: least squares fn = a + b*r, gate n>=8, den>1e-9, b>0, corr>=0.5,
 * f0=a>0 and f1/f0 >= 1.3 with f1 = a + b*max(r). */
int o64_fit_radial_eps(const double *rads, const double *floors, int n,
                       double *a, double *b, double *corr) {
    if (n < 8) return 0;
    double sr = 0, sf = 0, srr = 0, srf = 0, sff = 0;
    for (int i = 0; i < n; i++) {
        sr += rads[i]; sf += floors[i]; srr += rads[i] * rads[i];
        srf += rads[i] * floors[i]; sff += floors[i] * floors[i];
    }
    double nn = n, den = nn * srr - sr * sr;
    if (!(den > 1e-9)) return 0;
    double bb = (nn * srf - sr * sf) / den, aa = (sf - bb * sr) / nn;
    double cden = sqrt((nn * srr - sr * sr) * (nn * sff - sf * sf));
    double cc = cden > 1e-12 ? (nn * srf - sr * sf) / cden : 0;
    double rmax = 0;
    for (int i = 0; i < n; i++) if (rads[i] > rmax) rmax = rads[i];
    double f0 = aa, f1 = aa + bb * rmax;
    if (a) *a = aa;
    if (b) *b = bb;
    if (corr) *corr = cc;
    return (bb > 0 && cc >= 0.5 && f0 > 0 && f1 / f0 >= 1.3) ? 1 : 0;
}

/* median_sorted (pipeline.c:74-78) on a copy; 0.015 without samples (pipeline.c:878). */
static int o64_cmp_double(const void *a, const void *b) {
    double x = *(const double *)a, y = *(const double *)b;
    return (x > y) - (x < y);
}
double o64_median_floor(const double *v, int n) {
    if (n <= 0) return 0.015;
    double *w = (double *)malloc(sizeof(double) * (size_t)n);
    if (!w) return -1;
    memcpy(w, v, sizeof(double) * (size_t)n);
    qsort(w, (size_t)n, sizeof(double), o64_cmp_double);
    double m = (n & 1) ? w[n / 2] : 0.5 * (w[n / 2 - 1] + w[n / 2]);
    free(w);
    return m;
}

/* eps of a tile (pipeline.c:447-456): 0 when the radial model is off. */
double o64_radial_tile_eps(int have, double a, double b, double median, double guided_eps,
                           double ecy, double ecx, long y0, long x0, long ty, long tx) {
    if (!have || guided_eps <= 0 || median <= 0) return 0.0;
    double ry = y0 + ty / 2.0 - ecy, rx = x0 + tx / 2.0 - ecx;
    double fn = a + b * sqrt(ry * ry + rx * rx);
    double s = fn / median, s2 = s * s;
    if (s2 < 0.4) s2 = 0.4;
    if (s2 > 8.0) s2 = 8.0;
    return guided_eps * s2;
}

/* ---------------------------------------------------------------- calibration statistics */
/* Histogram of u8 values (stream.c:76-86): every value counted once. */
void o64_hist_u8(const uint8_t *v, size_t n, long long *hist) {
    for (size_t i = 0; i < n; ++i) hist[v[i]] += 1;
}

/* Flat-region noise floor (stream.c:174-200). Blocks of blk^3 voxels tile the volume from
 * the origin (partial blocks at the far edges are skipped). A block's sums run in voxel
 * order in double; the squares are float products, as the reference's `val*val` on a float
 * is. Blocks whose mean exceeds 0.1 contribute sqrt(max(var, 0)); the answer is the order
 * statistic m/10 (0-based) of those stds, ascending. */
double o64_flat_noise(const float *v, int nz, int ny, int nx, int blk) {
    if (blk < 4) blk = 8;
    const int bz = nz / blk, by = ny / blk, bx = nx / blk;
    const long nb = (long)bz * by * bx;
    if (nb <= 0) return 0;
    double *std_of = (double *)malloc(sizeof(double) * (size_t)nb);
    if (!std_of) return -1;
    long m = 0;
    const double cnt = (double)blk * blk * blk;
    for (long b = 0; b < nb; ++b) {
        const long z0 = (b / ((long)by * bx)) * blk, y0 = ((b / bx) % by) * blk, x0 = (b % bx) * blk;
        double s = 0, s2 = 0;
        for (int k = 0; k < blk * blk * blk; ++k) {
            const long z = z0 + k / (blk * blk), y = y0 + (k / blk) % blk, x = x0 + k % blk;
            const float t = v[((size_t)z * ny + y) * nx + x];
            const float t2 = t * t;
            s += t;
            s2 += t2;
        }
        const double mean = s / cnt, var = s2 / cnt - mean * mean;
        if (mean > 0.1) std_of[m++] = sqrt(var > 0 ? var : 0);
    }
    double out = 0;
    if (m > 0) {
        qsort(std_of, (size_t)m, sizeof(double), o64_cmp_double);
        out = std_of[m / 10];
    }
    free(std_of);
    return out;
}

/* Noise anisotropy (noise.c:210-269). 8^3 blocks from the origin; a block with any voxel
 * <= 0 is skipped (a NaN voxel does not skip it). Block variance in double from double sums of t and t^2, stored as a
 * float; the threshold is the order statistic nv/5 (0-based) of those floats. Blocks whose
 * variance (double) is at most the threshold give residuals r = (float)(t - (float)mean)
 * and add r*r to the denominator and the products of each r with its +z, +y, +x neighbour
 * inside the block to the three lag-1 sums (all double). rho = 8/7 * lag sum / denominator,
 * rho_xy the mean of the y and x ones. Returns 1 with fewer than 64 blocks, 64 non-zero
 * blocks, 32 flat blocks, or a zero denominator. */
static int o64_cmp_float(const void *a, const void *b) {
    float x = *(const float *)a, y = *(const float *)b;
    return (x > y) - (x < y);
}
int o64_noise_aniso(const float *v, int nz, int ny, int nx, double *rho_z, double *rho_xy) {
    enum { B = 8, B3 = B * B * B };
    const int bz = nz / B, by = ny / B, bx = nx / B;
    const long nb = (long)bz * by * bx;
    if (nb < 64) return 1;
    float *bvar = (float *)malloc(sizeof(float) * (size_t)nb);
    signed char *state = (signed char *)malloc((size_t)nb);       /* 0 skipped, 1 kept */
    double *mean_of = (double *)malloc(sizeof(double) * (size_t)nb);
    double *var_of = (double *)malloc(sizeof(double) * (size_t)nb);
    if (!bvar || !state || !mean_of || !var_of) { free(bvar); free(state); free(mean_of); free(var_of); return 1; }
    long nv = 0;
    for (long b = 0; b < nb; ++b) {
        const long z0 = (b / ((long)by * bx)) * B, y0 = ((b / bx) % by) * B, x0 = (b % bx) * B;
        double s = 0, s2 = 0;
        int positive = 1;
        for (int k = 0; k < B3; ++k) {
            const float t = v[((size_t)(z0 + k / (B * B)) * ny + y0 + (k / B) % B) * nx + x0 + k % B];
            if (t <= 0) positive = 0;
            s += t;
            s2 += (double)t * t;
        }
        state[b] = (signed char)positive;
        mean_of[b] = s / B3;
        var_of[b] = s2 / B3 - mean_of[b] * mean_of[b];
        if (positive) bvar[nv++] = (float)var_of[b];
    }
    int rc = 1;
    if (nv >= 64) {
        qsort(bvar, (size_t)nv, sizeof(float), o64_cmp_float);
        const float thresh = bvar[nv / 5];
        double nzs = 0, nys = 0, nxs = 0, den = 0;
        long used = 0;
        float r[B3];
        for (long b = 0; b < nb; ++b) {
            if (!state[b] || var_of[b] > thresh) continue;
            const long z0 = (b / ((long)by * bx)) * B, y0 = ((b / bx) % by) * B, x0 = (b % bx) * B;
            const float fm = (float)mean_of[b];
            for (int k = 0; k < B3; ++k)
                r[k] = v[((size_t)(z0 + k / (B * B)) * ny + y0 + (k / B) % B) * nx + x0 + k % B] - fm;
            for (int k = 0; k < B3; ++k) {
                const int dz = k / (B * B), dy = (k / B) % B, dx = k % B;
                den += (double)r[k] * r[k];
                if (dz + 1 < B) nzs += (double)r[k] * r[k + B * B];
                if (dy + 1 < B) nys += (double)r[k] * r[k + B];
                if (dx + 1 < B) nxs += (double)r[k] * r[k + 1];
            }
            ++used;
        }
        if (used >= 32 && den > 0) {
            const double corr = (double)B / (B - 1);
            *rho_z = corr * nzs / den;
            *rho_xy = corr * 0.5 * (nys + nxs) / den;
            rc = 0;
        }
    }
    free(bvar); free(state); free(mean_of); free(var_of);
    return rc;
}
