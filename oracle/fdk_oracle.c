/*
 * FP64 CPU oracle of satidev/gct's axial FDK path.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the checker that the CUDA engine is compared against;
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it. The product
 * path never calls it.
 *
 * It restates, in double precision and with plain loops, what the reference computes on the
 * GPU (paths relative to the satidev/gct project root):
 *   geometry factories   src/cpp/io/geom_reader/proj_geom_factory_params.cpp:8-108,
 *                        proj_geom_cb_factory.cpp:14-48, proj_geom_fb_factory.cpp:13-45
 *   rotation analysis    src/cpp/geom/rotation_geom.cpp:7-134, src/cpp/geom/utils.h:322-389
 *   cosine weights       src/cuda/recon/cos_weighting.cuh:16-153
 *   Parker weights       src/cuda/recon/parker_weighting.cuh:19-200
 *   ramp taps            src/cpp/recon/ramp_filter.h:22-56, ramp_filter.cpp:5-20,
 *                        src/cpp/recon/proj_filt_kernel.cpp:5-45
 *   row convolution      src/cuda/recon/ramp_filtering_fft.cuh:79-219, ramp_filtering_fft.cu:14-96
 *                        (linear convolution with taps at offsets -N/2..N-1-N/2, output at N/2)
 *   backprojection       src/cuda/recon/back_proj.cuh:16-104, src/cuda/geom/coord_trans_proj.cuh:
 *                        142-345, src/cuda/geom/coord_trans_img.cuh:52-66, texture addressing of
 *                        src/cuda/data/nd_array_texture.cuh:33-56 (linear filter, border 0)
 *   final scale          src/cuda/recon/fdk_axial.cuh:196-199
 *   spiral scans         src/cuda/recon/fdk_spiral.cuh:33-94 (no Parker weights: or_filter_np;
 *                        the per-slice view windows are restated in oracle.py)
 * The texture unit's linear filter can be emulated (lerp_bits = 8: sample positions and the
 * bilinear corner weight on a 1/256 grid, as measured through the reference's texture objects)
 * to quantify that difference separately from the exact bilinear interpolation (lerp_bits = 0).
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define OR_PI 3.14159265358979323846
#define OR_TWO_PI (2.0 * OR_PI)

enum { K_PAR1 = 0, K_ARC = 1, K_LINE = 2, K_PAR2 = 3, K_REBIN = 4, K_CYL = 5, K_FLAT = 6 };

typedef struct {
    double rot_ang, det_row_center, det_col_center, src_det_dist, src_iso_dist;
    double src_pos[3], det_row_dir[3], det_col_dir[3], iso_ray_dir[3];
} or_view;

typedef struct {
    int kind;
    unsigned nc;   /* detector columns (DetRow samples) */
    double du;     /* DetRow sampling width */
    unsigned nr;   /* detector rows (DetCol samples; 1 for 1D kinds) */
    double dv;     /* DetCol sampling width */
    unsigned nv;
    const or_view *views;
} or_geom;

typedef struct {
    unsigned nx, ny, nz;
    double dx, dy, dz, mx, my, mz;
} or_vol;

static int is2d(int kind) { return kind >= K_PAR2; }
static int is_parallel(int kind) { return kind == K_PAR1 || kind == K_PAR2 || kind == K_REBIN; }
static int is_arc(int kind) { return kind == K_ARC || kind == K_CYL; }

/* ---- geometry ----------------------------------------------------------------------------- */

/* params: det_row_center, det_col_center, src_det_dist, src_iso_dist, dir, init_ang, ang_incr,
 * hel_pitch */
int or_make_view(int kind, const double *p, unsigned idx, or_view *v)
{
    memset(v, 0, sizeof(*v));
    const double theta = p[5] + p[6] * (double)idx;
    v->det_row_center = p[0];
    if (is_parallel(kind)) {
        v->rot_ang = theta;
        if (kind != K_PAR1) v->det_col_center = p[1];
        if (kind == K_REBIN) {
            v->src_det_dist = p[2];
            v->src_iso_dist = p[3];
        }
        return 0;
    }
    const int fan = !is2d(kind);
    const double phi = p[4] * theta; /* R_z(dir * theta) */
    const double c = cos(phi), s = sin(phi);
    v->src_det_dist = p[2];
    v->src_iso_dist = p[3];
    /* source R_z (SID, 0, -pitch theta); basis rows (0,1,0), (0,0,-1), (-1,0,0) rotated */
    v->src_pos[0] = p[3] * c;
    v->src_pos[1] = p[3] * s;
    v->src_pos[2] = fan ? 0.0 : -p[7] * theta;
    v->det_row_dir[0] = -s;
    v->det_row_dir[1] = c;
    if (!fan) {
        v->det_col_center = p[1];
        v->det_col_dir[2] = -1.0;
    }
    if (is_arc(kind)) {
        v->iso_ray_dir[0] = -c;
        v->iso_ray_dir[1] = -s;
    }
    return 0;
}

/* utils.h:338-348; angles within one FP32 step below 2 pi wrap to 0, as the reference's FP32 wrap
 * does for FP32 inputs (its 2 pi constant is float(2 pi)) */
static double wrap2pi(double a)
{
    while (a < 0.0) a += OR_TWO_PI;
    if (fabs(a - OR_TWO_PI) <= 4.8e-7) return 0.0;
    return (a >= OR_TWO_PI) ? remainder(a, OR_TWO_PI) : a;
}

static unsigned quadrant(double a)
{
    const double w = wrap2pi(a);
    if (w >= 0.0 && w < OR_PI / 2.0) return 1;
    if (w >= OR_PI / 2.0 && w < OR_PI) return 2;
    if (w >= OR_PI && w < 1.5 * OR_PI) return 3;
    return 4;
}

static double view_angle(int kind, const or_view *v)
{
    if (is_parallel(kind)) return wrap2pi(v->rot_ang);
    return wrap2pi(atan2(v->src_pos[1], v->src_pos[0]));
}

/* rot_dir from the first two angles (rotation_geom.cpp:7-43); 0 = undefined */
int or_rot_dir(const double *ang, unsigned n)
{
    if (n < 2) return 0;
    const double a0 = wrap2pi(ang[0]), a1 = wrap2pi(ang[1]);
    const unsigned q0 = quadrant(a0), q1 = quadrant(a1);
    if (q0 == 1 && q1 == 4) return -1;
    if (q0 == 4 && q1 == 1) return 1;
    if (a1 - a0 > 0.0) return 1;
    if (a1 - a0 < 0.0) return -1;
    return 0;
}

/* Fills dir, incr, range, num_proj_per_rot, angles and relative angles. Returns 0 on success,
 * -1 where the reference yields std::nullopt. */
int or_rotation(const or_geom *g, int *dir, double *incr, double *range, unsigned *nppr,
                double *rot, double *rel)
{
    const unsigned n = g->nv;
    for (unsigned i = 0; i < n; ++i) rot[i] = view_angle(g->kind, &g->views[i]);
    const int d = or_rot_dir(rot, n);
    if (d == 0) return -1;
    for (unsigned i = 0; i < n; ++i) rel[i] = wrap2pi(d < 0 ? rot[0] - rot[i] : rot[i] - rot[0]);
    double sum = 0.0, mx = rel[0];
    for (unsigned i = 0; i + 1 < n; ++i) sum += wrap2pi(rel[i + 1] - rel[i]);
    for (unsigned i = 0; i < n; ++i) mx = rel[i] > mx ? rel[i] : mx;
    *dir = d;
    *incr = sum / (double)(n - 1);
    *range = *incr + mx;
    *nppr = n;
    if (rel[0] != 0.0) return -1;
    for (unsigned i = 1; i < n; ++i) {
        if (fabs(rel[i]) < 1e-6) {
            *nppr = i;
            break;
        }
    }
    return 0;
}

/* ---- weights and taps --------------------------------------------------------------------- */

static double M(double t) { return t == 0.0 ? 0.5 : sin(t) / t + (cos(t) - 1.0) / (t * t); }

void or_ramp_taps(int kind, unsigned n, double width, double fc, int apod, double *taps)
{
    const double a = apod == 1 ? 0.5 : apod == 2 ? 0.54 : 1.0;
    for (unsigned j = 0; j < n; ++j) {
        const int off = (int)j - (int)(n / 2);
        const double nd = (double)off;
        double c = (fc * fc / (2.0 * width)) *
                   (a * M(fc * OR_PI * nd) + ((1.0 - a) / 2.0) * M(OR_PI * fc * nd + OR_PI) +
                    ((1.0 - a) / 2.0) * M(OR_PI * fc * nd - OR_PI));
        if (is_arc(kind) && off != 0) {
            const double b = nd * width;
            c *= pow(b / sin(b), 2.0);
        }
        taps[j] = c;
    }
}

double or_cos_weight(const or_geom *g, unsigned v, unsigned r, unsigned c)
{
    const or_view *pv = &g->views[v];
    const double u = ((double)c - pv->det_row_center) * g->du;
    const double t = is2d(g->kind) ? ((double)r - pv->det_col_center) * g->dv : 0.0;
    const double sdd = pv->src_det_dist;
    switch (g->kind) {
        case K_ARC: return cos(u);
        case K_LINE: return sdd / sqrt(u * u + sdd * sdd);
        case K_REBIN: return sdd / sqrt(t * t + sdd * sdd);
        case K_CYL: return cos(u) * sdd / sqrt(t * t + sdd * sdd);
        case K_FLAT: return sdd / sqrt(u * u + t * t + sdd * sdd);
        default: return 1.0;
    }
}

/* Parker weights [nv][nc]; fan/cone ranges <= pi give 1 (the reference leaves them unset). */
int or_parker(const or_geom *g, double *w)
{
    const unsigned nv = g->nv, nc = g->nc;
    double *rot = malloc(sizeof(double) * nv), *rel = malloc(sizeof(double) * nv);
    int dir = 0;
    double incr = 0, range = 0;
    unsigned nppr = 0;
    if (!rot || !rel || or_rotation(g, &dir, &incr, &range, &nppr, rot, rel) != 0) {
        free(rot);
        free(rel);
        return -1;
    }
    if (is_parallel(g->kind)) {
        const double val = (incr > 0.0 && range <= incr + OR_PI) ? 1.0 : 0.5;
        for (size_t i = 0; i < (size_t)nv * nc; ++i) w[i] = val;
    } else if (!(range > OR_PI)) {
        for (size_t i = 0; i < (size_t)nv * nc; ++i) w[i] = 1.0;
    } else {
        const or_view *v0 = &g->views[0];
        for (unsigned v = 0; v < nv; ++v) {
            const double b = (dir < 0) ? rel[nv - 1 - v] : rel[v];
            for (unsigned c = 0; c < nc; ++c) {
                const double t = ((double)c - v0->det_row_center) * g->du;
                const double gm = is_arc(g->kind) ? t : atan2(t, v0->src_det_dist);
                const double t2 = 2.0 * gm + range - OR_PI, t3 = 2.0 * gm + OR_PI;
                double x = 0.0;
                if (b >= 0.0 && b <= t2)
                    x = pow(sin(OR_PI * b / (2.0 * (range - OR_PI) + 4.0 * gm)), 2.0);
                else if (b >= t2 && b <= t3)
                    x = 1.0;
                else if (b >= t3 && b <= range)
                    x = pow(sin(OR_PI * (range - b) / (2.0 * (range - OR_PI) - 4.0 * gm)), 2.0);
                w[(size_t)v * nc + c] = x;
            }
        }
    }
    free(rot);
    free(rel);
    return 0;
}

/* ---- filtering ---------------------------------------------------------------------------- */

/* one weighted row -> filtered row (direct linear convolution) */
static void filter_row_direct(const or_geom *g, const float *in, const double *parker, const double *taps,
                              unsigned v, unsigned r, double *tmp, double *out)
{
    const unsigned n = g->nc;
    for (unsigned c = 0; c < n; ++c)
        tmp[c] = (double)in[c] * or_cos_weight(g, v, r, c) * parker[(size_t)v * n + c];
    for (unsigned c = 0; c < n; ++c) {
        double acc = 0.0;
        /* tap index j = c - k + n/2 in [0, n) */
        const long lo = (long)c + (long)(n / 2) - (long)(n - 1);
        const long kmin = lo > 0 ? lo : 0;
        const long khi = (long)c + (long)(n / 2);
        const long kmax = khi < (long)n - 1 ? khi : (long)n - 1;
        for (long k = kmin; k <= kmax; ++k) acc += tmp[k] * taps[(long)c - k + (long)(n / 2)];
        out[c] = acc;
    }
}

/* complex radix-2 FFT in double, in place, n a power of two; tw holds exp(-2 pi i m / n) for
 * m < n/2; sign -1 forward, +1 backward (unnormalised) */
static void fft_c(double *re, double *im, unsigned n, int sign, const double *twr, const double *twi)
{
    for (unsigned i = 1, j = 0; i < n; ++i) {
        unsigned bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            double t = re[i]; re[i] = re[j]; re[j] = t;
            t = im[i]; im[i] = im[j]; im[j] = t;
        }
    }
    for (unsigned len = 2; len <= n; len <<= 1) {
        const unsigned stride = n / len;
        for (unsigned i = 0; i < n; i += len) {
            for (unsigned k = 0; k < len / 2; ++k) {
                const double wr = twr[k * stride], wi = sign < 0 ? twi[k * stride] : -twi[k * stride];
                const unsigned a = i + k, b = i + k + len / 2;
                const double xr = re[b] * wr - im[b] * wi, xi = re[b] * wi + im[b] * wr;
                re[b] = re[a] - xr;
                im[b] = im[a] - xi;
                re[a] += xr;
                im[a] += xi;
            }
        }
    }
}

typedef struct {
    const or_geom *g;
    const float *proj;
    const double *parker, *taps;
    const long *rows; /* global row ids to filter, or NULL for all */
    long nrows;
    double *out;      /* row-major, one row of nc per entry of rows (or per global row) */
    int use_fft;
    double *Hre, *Him, *twr, *twi;
    unsigned L;
    long next;
    pthread_mutex_t mu;
} filt_job;

static void *filter_worker(void *arg)
{
    filt_job *J = arg;
    const unsigned n = J->g->nc;
    double *tmp = malloc(sizeof(double) * n);
    double *re = J->use_fft ? malloc(sizeof(double) * J->L) : NULL;
    double *im = J->use_fft ? malloc(sizeof(double) * J->L) : NULL;
    for (;;) {
        pthread_mutex_lock(&J->mu);
        const long t = J->next;
        J->next += 2;
        pthread_mutex_unlock(&J->mu);
        if (t >= J->nrows) break;
        for (int h = 0; h < 2 && t + h < J->nrows; ++h) {
            const long gr = J->rows ? J->rows[t + h] : t + h;
            const unsigned v = (unsigned)(gr / J->g->nr), r = (unsigned)(gr % J->g->nr);
            const float *in = J->proj + (size_t)gr * n;
            double *out = J->out + (size_t)(t + h) * n;
            if (!J->use_fft) {
                filter_row_direct(J->g, in, J->parker, J->taps, v, r, tmp, out);
                continue;
            }
            /* circular convolution of length L with circularly placed taps (no aliasing for
               L > 1.5 n), identical to the direct sum up to rounding */
            for (unsigned k = 0; k < J->L; ++k) re[k] = im[k] = 0.0;
            for (unsigned c = 0; c < n; ++c)
                re[c] = (double)in[c] * or_cos_weight(J->g, v, r, c) * J->parker[(size_t)v * n + c];
            fft_c(re, im, J->L, -1, J->twr, J->twi);
            for (unsigned k = 0; k < J->L; ++k) {
                const double a = re[k] * J->Hre[k] - im[k] * J->Him[k];
                const double b = re[k] * J->Him[k] + im[k] * J->Hre[k];
                re[k] = a;
                im[k] = b;
            }
            fft_c(re, im, J->L, +1, J->twr, J->twi);
            for (unsigned c = 0; c < n; ++c) out[c] = re[c] / J->L;
        }
    }
    free(tmp);
    free(re);
    free(im);
    return NULL;
}

static unsigned alias_free_len(unsigned n)
{
    long need = 2L * n - 2 - n / 2;
    if ((long)n - 1 + (long)(n / 2) > need) need = (long)n - 1 + n / 2;
    unsigned L = 64;
    while ((long)L <= need) L *= 2;
    return L;
}

static int run_filter(const or_geom *g, const float *proj, double fc, int apod, const long *rows,
                      long nrows, double *out, int use_fft, int nthreads, int use_parker)
{
    const unsigned n = g->nc;
    double *parker = malloc(sizeof(double) * (size_t)g->nv * n);
    double *taps = malloc(sizeof(double) * n);
    if (parker && !use_parker)
        for (size_t i = 0; i < (size_t)g->nv * n; ++i) parker[i] = 1.0;
    if (!parker || !taps || (use_parker && or_parker(g, parker) != 0)) {
        free(parker);
        free(taps);
        return -1;
    }
    or_ramp_taps(g->kind, n, g->du, fc, apod, taps);
    filt_job J;
    memset(&J, 0, sizeof(J));
    J.g = g;
    J.proj = proj;
    J.parker = parker;
    J.taps = taps;
    J.rows = rows;
    J.nrows = nrows;
    J.out = out;
    J.use_fft = use_fft;
    if (use_fft) {
        J.L = alias_free_len(n);
        J.Hre = calloc(J.L, sizeof(double));
        J.Him = calloc(J.L, sizeof(double));
        J.twr = malloc(sizeof(double) * (J.L / 2));
        J.twi = malloc(sizeof(double) * (J.L / 2));
        for (unsigned m = 0; m < J.L / 2; ++m) {
            J.twr[m] = cos(OR_TWO_PI * m / J.L);
            J.twi[m] = -sin(OR_TWO_PI * m / J.L);
        }
        for (unsigned j = 0; j < n; ++j) {
            const int off = (int)j - (int)(n / 2);
            J.Hre[(unsigned)((off % (int)J.L + (int)J.L) % (int)J.L)] += taps[j];
        }
        fft_c(J.Hre, J.Him, J.L, -1, J.twr, J.twi);
    }
    pthread_mutex_init(&J.mu, NULL);
    if (nthreads < 1) nthreads = 1;
    pthread_t *th = malloc(sizeof(pthread_t) * nthreads);
    for (int i = 0; i < nthreads; ++i) pthread_create(&th[i], NULL, filter_worker, &J);
    for (int i = 0; i < nthreads; ++i) pthread_join(th[i], NULL);
    pthread_mutex_destroy(&J.mu);
    free(th);
    free(J.Hre);
    free(J.Him);
    free(J.twr);
    free(J.twi);
    free(parker);
    free(taps);
    return 0;
}

/* Weighted + ramp-filtered projections [nv][nr][nc] (no backprojection scales). */
int or_filter(const or_geom *g, const float *proj, double fc, int apod, int use_fft, double *out,
              int nthreads)
{
    return run_filter(g, proj, fc, apod, NULL, (long)g->nv * g->nr, out, use_fft, nthreads, 1);
}

/* The same without Parker weights (the spiral FDK weights by cosine only). */
int or_filter_np(const or_geom *g, const float *proj, double fc, int apod, int use_fft, double *out,
                 int nthreads)
{
    return run_filter(g, proj, fc, apod, NULL, (long)g->nv * g->nr, out, use_fft, nthreads, 0);
}

/* ---- backprojection ----------------------------------------------------------------------- */

static double dot3(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

/* Detector pixel coordinates (col, row) and backprojection weight of world point X in view v.
 * Returns the weight; row is 0 for 1D detectors. */
static double project_point(const or_geom *g, unsigned vi, const double *X, double *col, double *row)
{
    const or_view *v = &g->views[vi];
    const int k = g->kind;
    double u = 0.0, t = 0.0, w = 1.0;
    if (is_parallel(k)) {
        const double th = v->rot_ang + OR_PI / 2.0;
        u = X[0] * cos(th) + X[1] * sin(th);
        if (k == K_PAR2) t = -X[2];
        if (k == K_REBIN) t = -X[2] * v->src_det_dist / v->src_iso_dist;
    } else {
        const int fan = !is2d(k);
        double S[3] = {v->src_pos[0], v->src_pos[1], fan ? 0.0 : v->src_pos[2]};
        double eu[3] = {v->det_row_dir[0], v->det_row_dir[1], fan ? 0.0 : v->det_row_dir[2]};
        double d[3] = {X[0] - S[0], X[1] - S[1], fan ? 0.0 : X[2] - S[2]};
        const double sid = sqrt(dot3(S, S));
        const double sdd = v->src_det_dist;
        if (k == K_LINE || k == K_FLAT) {
            double ew[3], ev[3] = {0, 0, 0};
            if (k == K_LINE) {
                ew[0] = -eu[1];
                ew[1] = eu[0];
                ew[2] = 0.0;
            } else {
                for (int i = 0; i < 3; ++i) ev[i] = v->det_col_dir[i];
                ew[0] = eu[1] * ev[2] - eu[2] * ev[1];
                ew[1] = eu[2] * ev[0] - eu[0] * ev[2];
                ew[2] = eu[0] * ev[1] - eu[1] * ev[0];
            }
            const double D = dot3(d, ew);
            u = sdd * dot3(d, eu) / D;
            if (k == K_FLAT) t = sdd * dot3(d, ev) / D;
            w = sdd * sid / (D * D);
        } else { /* arc kinds */
            double ew[3] = {v->iso_ray_dir[0], v->iso_ray_dir[1], fan ? 0.0 : v->iso_ray_dir[2]};
            const double dn = sqrt(dot3(d, d));
            double dh[3] = {d[0] / dn, d[1] / dn, d[2] / dn};
            u = atan2(dot3(dh, eu), dot3(dh, ew));
            if (k == K_CYL) {
                const double q = dot3(dh, v->det_col_dir);
                t = sdd * q / sqrt(1.0 - q * q);
            }
            w = sid / (dn * dn);
        }
    }
    *col = u / g->du + v->det_row_center;
    *row = is2d(k) ? t / g->dv + v->det_col_center : 0.0;
    return w;
}

static double quant(double a, int bits)
{
    if (bits <= 0) return a;
    const double s = (double)(1 << bits);
    return floor(a * s + 0.5) / s;
}

/* Bilinear value of texels t00 = T[r][c], t01 = T[r][c+1], t10 = T[r+1][c], t11 = T[r+1][c+1] at
 * fractions ac (along a row) and ar (across rows). lerp_bits = 0: exact weights. lerp_bits = 8:
 * the texture unit's linear filter as measured through the reference's own texture objects
 * (golden vectors tests/golden/tex_probe.npz): both fractions snap to the nearest 1/256 (the
 * callers snap them), the corner weight ac ar snaps to the nearest 1/256 too, and the other three
 * weights follow from it so that all four sum to one. A 1D fetch is the case ar = 0. */
static double bilerp(double t00, double t01, double t10, double t11, double ac, double ar, int lerp_bits)
{
    const double w11 = quant(ac * ar, lerp_bits);
    return (1.0 - ac - ar + w11) * t00 + (ac - w11) * t01 + (ar - w11) * t10 + w11 * t11;
}

/* bilinear sample of one filtered view at pixel coordinates with border 0 */
static double sample(const double *(*rowp)(void *, unsigned, long), void *ctx, unsigned v, const or_geom *g,
                     double col, double row, int lerp_bits)
{
    const double fc = floor(col);
    const long ic = (long)fc;
    const double ac = quant(col - fc, lerp_bits);
    if (!is2d(g->kind)) {
        const double *p = rowp(ctx, v, 0);
        const double a = (ic >= 0 && ic < (long)g->nc) ? p[ic] : 0.0;
        const double b = (ic + 1 >= 0 && ic + 1 < (long)g->nc) ? p[ic + 1] : 0.0;
        return bilerp(a, b, 0.0, 0.0, ac, 0.0, lerp_bits);
    }
    const double fr = floor(row);
    const long ir = (long)fr;
    const double ar = quant(row - fr, lerp_bits);
    double t[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
    for (int dr = 0; dr < 2; ++dr) {
        const long rr = ir + dr;
        if (rr < 0 || rr >= (long)g->nr) continue;
        const double *p = rowp(ctx, v, rr);
        t[dr][0] = (ic >= 0 && ic < (long)g->nc) ? p[ic] : 0.0;
        t[dr][1] = (ic + 1 >= 0 && ic + 1 < (long)g->nc) ? p[ic + 1] : 0.0;
    }
    return bilerp(t[0][0], t[0][1], t[1][0], t[1][1], ac, ar, lerp_bits);
}

/* The oracle's texture fetch on its own: texels [h][w], texture coordinates (x, y) as passed to
 * tex2D (texel centres at integer + 0.5; y = 0.5 for a one-row texture), border 0. Lets the
 * golden probe vectors pin the emulation used by or_fdk / or_backproject. */
double or_tex_fetch(const double *tex, unsigned w, unsigned h, double x, double y, int lerp_bits)
{
    const double px = x - 0.5, py = y - 0.5;
    const double fx = floor(px), fy = floor(py);
    const long i = (long)fx, j = (long)fy;
    const double ac = quant(px - fx, lerp_bits), ar = quant(py - fy, lerp_bits);
    double t[2][2];
    for (int dr = 0; dr < 2; ++dr)
        for (int dc = 0; dc < 2; ++dc) {
            const long r = j + dr, c = i + dc;
            t[dr][dc] = (r >= 0 && r < (long)h && c >= 0 && c < (long)w) ? tex[(size_t)r * w + (size_t)c] : 0.0;
        }
    return bilerp(t[0][0], t[0][1], t[1][0], t[1][1], ac, ar, lerp_bits);
}

typedef struct {
    const or_geom *g;
    const or_vol *vol;
    const unsigned *vox;  /* (i,j,k) triples or NULL for the whole grid */
    long nvox;
    double scale;
    int lerp_bits;
    const double *filt;   /* full stack [nv][nr][nc] or compact rows */
    const long *slot;     /* [nv*nr] -> compact row index, or NULL */
    double *out;
    long next;
    pthread_mutex_t mu;
} bp_job;

static const double *row_full(void *ctx, unsigned v, long r)
{
    bp_job *J = ctx;
    const size_t gr = (size_t)v * J->g->nr + (size_t)r;
    if (J->slot) return J->filt + (size_t)J->slot[gr] * J->g->nc;
    return J->filt + gr * J->g->nc;
}

static void voxel_pos(const or_vol *vol, int vol3d, unsigned i, unsigned j, unsigned k, double *X)
{
    X[0] = vol->mx - (vol->nx - 1.0) * vol->dx / 2.0 + i * vol->dx;
    X[1] = vol->my - (vol->ny - 1.0) * vol->dy / 2.0 + j * vol->dy;
    X[2] = vol3d ? vol->mz - (vol->nz - 1.0) * vol->dz / 2.0 + k * vol->dz : 0.0;
}

static void *bp_worker(void *arg)
{
    bp_job *J = arg;
    const int vol3d = is2d(J->g->kind);
    const long chunk = 256;
    for (;;) {
        pthread_mutex_lock(&J->mu);
        const long t0 = J->next;
        J->next += chunk;
        pthread_mutex_unlock(&J->mu);
        if (t0 >= J->nvox) break;
        const long t1 = t0 + chunk < J->nvox ? t0 + chunk : J->nvox;
        for (long t = t0; t < t1; ++t) {
            unsigned i, j, k;
            if (J->vox) {
                i = J->vox[3 * t];
                j = J->vox[3 * t + 1];
                k = J->vox[3 * t + 2];
            } else {
                i = (unsigned)(t % J->vol->nx);
                j = (unsigned)((t / J->vol->nx) % J->vol->ny);
                k = (unsigned)(t / ((long)J->vol->nx * J->vol->ny));
            }
            double X[3];
            voxel_pos(J->vol, vol3d, i, j, k, X);
            double acc = 0.0;
            for (unsigned v = 0; v < J->g->nv; ++v) {
                double col, row;
                const double w = project_point(J->g, v, X, &col, &row);
                acc += w * sample(row_full, J, v, J->g, col, row, J->lerp_bits);
            }
            J->out[t] = acc * J->scale;
        }
    }
    return NULL;
}

static double final_scale(const or_geom *g)
{
    double *rot = malloc(sizeof(double) * g->nv), *rel = malloc(sizeof(double) * g->nv);
    int dir = 0;
    double incr = 0, range = 0;
    unsigned nppr = 0;
    double s = 1.0;
    if (rot && rel && or_rotation(g, &dir, &incr, &range, &nppr, rot, rel) == 0 && incr > 0.0) s = incr;
    free(rot);
    free(rel);
    return s;
}

static void run_bp(bp_job *J, int nthreads)
{
    pthread_mutex_init(&J->mu, NULL);
    if (nthreads < 1) nthreads = 1;
    pthread_t *th = malloc(sizeof(pthread_t) * nthreads);
    for (int i = 0; i < nthreads; ++i) pthread_create(&th[i], NULL, bp_worker, J);
    for (int i = 0; i < nthreads; ++i) pthread_join(th[i], NULL);
    pthread_mutex_destroy(&J->mu);
    free(th);
}

/* Backprojects an already filtered stack [nv][nr][nc] into the whole grid (or the listed voxels),
 * including the final angular-increment scale. */
int or_backproject(const or_geom *g, const or_vol *vol, const double *filtered, const unsigned *vox,
                   long nvox, int lerp_bits, double *out, int nthreads)
{
    bp_job J;
    memset(&J, 0, sizeof(J));
    J.g = g;
    J.vol = vol;
    J.vox = vox;
    J.nvox = vox ? nvox : (long)vol->nx * vol->ny * vol->nz;
    J.scale = final_scale(g);
    J.lerp_bits = lerp_bits;
    J.filt = filtered;
    J.out = out;
    run_bp(&J, nthreads);
    return 0;
}

/* Full FDK of the listed voxels (or the whole grid when vox is NULL). Only the detector rows that
 * the voxels touch are filtered. */
int or_fdk(const or_geom *g, const or_vol *vol, const float *proj, double fc, int apod, int use_fft,
           const unsigned *vox, long nvox, int lerp_bits, double *out, int nthreads)
{
    const int vol3d = is2d(g->kind);
    const long total = vox ? nvox : (long)vol->nx * vol->ny * vol->nz;
    const size_t nrows_all = (size_t)g->nv * g->nr;
    long *slot = malloc(sizeof(long) * nrows_all);
    if (!slot) return -1;
    for (size_t i = 0; i < nrows_all; ++i) slot[i] = -1;
    /* pass 1: rows touched */
    for (long t = 0; t < total; ++t) {
        unsigned i, j, k;
        if (vox) {
            i = vox[3 * t];
            j = vox[3 * t + 1];
            k = vox[3 * t + 2];
        } else {
            i = (unsigned)(t % vol->nx);
            j = (unsigned)((t / vol->nx) % vol->ny);
            k = (unsigned)(t / ((long)vol->nx * vol->ny));
        }
        double X[3];
        voxel_pos(vol, vol3d, i, j, k, X);
        for (unsigned v = 0; v < g->nv; ++v) {
            double col, row;
            project_point(g, v, X, &col, &row);
            const long ir = (long)floor(row);
            for (long rr = ir; rr <= ir + 1; ++rr)
                if (rr >= 0 && rr < (long)g->nr) slot[(size_t)v * g->nr + rr] = 0;
        }
    }
    long nsel = 0;
    for (size_t i = 0; i < nrows_all; ++i)
        if (slot[i] == 0) ++nsel;
    long *rows = malloc(sizeof(long) * (nsel > 0 ? nsel : 1));
    double *filt = malloc(sizeof(double) * (size_t)(nsel > 0 ? nsel : 1) * g->nc);
    if (!rows || !filt) {
        free(slot);
        free(rows);
        free(filt);
        return -1;
    }
    long s = 0;
    for (size_t i = 0; i < nrows_all; ++i)
        if (slot[i] == 0) {
            rows[s] = (long)i;
            slot[i] = s++;
        }
    if (run_filter(g, proj, fc, apod, rows, nsel, filt, use_fft, nthreads, 1) != 0) {
        free(slot);
        free(rows);
        free(filt);
        return -1;
    }
    bp_job J;
    memset(&J, 0, sizeof(J));
    J.g = g;
    J.vol = vol;
    J.vox = vox;
    J.nvox = total;
    J.scale = final_scale(g);
    J.lerp_bits = lerp_bits;
    J.filt = filt;
    J.slot = slot;
    J.out = out;
    run_bp(&J, nthreads);
    free(slot);
    free(rows);
    free(filt);
    return 0;
}

/* Mapping of one world point (for the reference's projMapping known-answer tests): writes the
 * detector coordinates in mm / rad (DCS, before DCSToPCS) and returns the weight. */
double or_proj_mapping(const or_geom *g, unsigned v, const double *X, double *u, double *t)
{
    double col, row;
    const double w = project_point(g, v, X, &col, &row);
    *u = (col - g->views[v].det_row_center) * g->du;
    *t = is2d(g->kind) ? (row - g->views[v].det_col_center) * g->dv : 0.0;
    return w;
}

/* ---- analytic phantom --------------------------------------------------------------------- */

/* Ray of detector pixel (v, r, c): origin o and (unnormalised) direction d, in the geometry's
 * own convention (the inverse of projMapping + DCSToPCS, src/cuda/geom/coord_trans_proj.cuh:
 * 142-345): parallel kinds start on the detector line through the isocentre, the others at the
 * source and pass through the pixel. */
static void pixel_ray(const or_geom *g, unsigned v, unsigned r, unsigned c, double *o, double *d)
{
    const int k = g->kind;
    const or_view *pv = &g->views[v];
    const double u = ((double)c - pv->det_row_center) * g->du;
    const double t = is2d(k) ? ((double)r - pv->det_col_center) * g->dv : 0.0;
    for (int i = 0; i < 3; ++i) o[i] = d[i] = 0.0;
    if (is_parallel(k)) {
        const double th = pv->rot_ang;
        o[0] = -sin(th) * u;
        o[1] = cos(th) * u;
        o[2] = k == K_PAR2 ? -t : k == K_REBIN ? -t * pv->src_iso_dist / pv->src_det_dist : 0.0;
        d[0] = cos(th);
        d[1] = sin(th);
        return;
    }
    const int fan = !is2d(k);
    double S[3] = {pv->src_pos[0], pv->src_pos[1], fan ? 0.0 : pv->src_pos[2]};
    double eu[3] = {pv->det_row_dir[0], pv->det_row_dir[1], fan ? 0.0 : pv->det_row_dir[2]};
    double ev[3] = {0, 0, 0}, ew[3];
    if (k == K_FLAT || k == K_CYL)
        for (int i = 0; i < 3; ++i) ev[i] = pv->det_col_dir[i];
    if (k == K_LINE) {
        ew[0] = -eu[1];
        ew[1] = eu[0];
        ew[2] = 0.0;
    } else if (k == K_FLAT) {
        ew[0] = eu[1] * ev[2] - eu[2] * ev[1];
        ew[1] = eu[2] * ev[0] - eu[0] * ev[2];
        ew[2] = eu[0] * ev[1] - eu[1] * ev[0];
    } else {
        ew[0] = pv->iso_ray_dir[0];
        ew[1] = pv->iso_ray_dir[1];
        ew[2] = fan ? 0.0 : pv->iso_ray_dir[2];
    }
    for (int i = 0; i < 3; ++i) o[i] = S[i];
    if (k == K_LINE || k == K_FLAT) {
        for (int i = 0; i < 3; ++i) d[i] = pv->src_det_dist * ew[i] + u * eu[i] + t * ev[i];
    } else {
        for (int i = 0; i < 3; ++i) d[i] = cos(u) * ew[i] + sin(u) * eu[i] + (t / pv->src_det_dist) * ev[i];
    }
}

/* ellipsoids: 8 doubles each (cx, cy, cz, ax, ay, az, phi, mu). out [nv][nr][nc]. 1D-detector
 * kinds integrate the ellipses' cross-sections in the plane z = 0 (planar rays). */
void or_phantom(const or_geom *g, const double *ell, unsigned ne, double *out)
{
    const int planar = !is2d(g->kind);
    for (unsigned v = 0; v < g->nv; ++v) {
        for (unsigned r = 0; r < g->nr; ++r) {
            for (unsigned c = 0; c < g->nc; ++c) {
                double o[3], d[3];
                pixel_ray(g, v, r, c, o, d);
                const double dn = sqrt(dot3(d, d));
                double sum = 0.0;
                for (unsigned e = 0; e < ne; ++e) {
                    const double *E = ell + 8 * e;
                    const double cp = cos(E[6]), sp = sin(E[6]);
                    const double p0 = o[0] - E[0], p1 = o[1] - E[1], p2 = planar ? 0.0 : o[2] - E[2];
                    const double q2 = planar ? 0.0 : d[2];
                    const double px = (cp * p0 + sp * p1) / E[3], py = (-sp * p0 + cp * p1) / E[4], pz = p2 / E[5];
                    const double qx = (cp * d[0] + sp * d[1]) / E[3], qy = (-sp * d[0] + cp * d[1]) / E[4], qz = q2 / E[5];
                    const double A = qx * qx + qy * qy + qz * qz, B = px * qx + py * qy + pz * qz;
                    const double C = px * px + py * py + pz * pz - 1.0;
                    const double disc = B * B - A * C;
                    if (disc > 0.0) sum += E[7] * 2.0 * sqrt(disc) / A * dn;
                }
                out[((size_t)v * g->nr + r) * g->nc + c] = sum;
            }
        }
    }
}

/* Isotropic Gaussian blobs: 5 doubles each (cx, cy, cz, sigma, amplitude), density
 * a exp(-|x - c|^2 / (2 sigma^2)). The line integral of a blob along a line whose closest
 * approach to its centre is dist is a sigma sqrt(2 pi) exp(-dist^2 / (2 sigma^2)); 1D-detector
 * kinds integrate 2D blobs in the plane z = 0 (the same formula with the in-plane distance).
 * A smooth phantom with exact line integrals, for checking a projector that samples a voxel
 * grid. out [nv][nr][nc]. */
void or_gauss_project(const or_geom *g, const double *blobs, unsigned nb, double *out)
{
    const int planar = !is2d(g->kind);
    for (unsigned v = 0; v < g->nv; ++v) {
        for (unsigned r = 0; r < g->nr; ++r) {
            for (unsigned c = 0; c < g->nc; ++c) {
                double o[3], d[3];
                pixel_ray(g, v, r, c, o, d);
                if (planar) o[2] = d[2] = 0.0;
                const double dn = sqrt(dot3(d, d));
                const double e[3] = {d[0] / dn, d[1] / dn, d[2] / dn};
                double sum = 0.0;
                for (unsigned b = 0; b < nb; ++b) {
                    const double *B = blobs + 5 * b;
                    const double w[3] = {B[0] - o[0], B[1] - o[1], planar ? 0.0 : B[2] - o[2]};
                    const double along = dot3(w, e);
                    const double d2 = fmax(dot3(w, w) - along * along, 0.0);
                    sum += B[4] * B[3] * sqrt(2.0 * OR_PI) * exp(-d2 / (2.0 * B[3] * B[3]));
                }
                out[((size_t)v * g->nr + r) * g->nc + c] = sum;
            }
        }
    }
}
