/*
 * nufht_oracle.c -- CPU oracle (TEST INFRASTRUCTURE ONLY) for the batched NUFHT.
 *
 * A plain-C restatement of the reference library Ansal06/NUFHT, written for this
 * project from the reference's documented behaviour.  Every function cites the
 * reference file:line it follows.  It is the parity checker for the CUDA product
 * and the timed CPU baseline; the product never links it.  See nufht_oracle.h for
 * what stands in for GSL and FINUFFT.
 */
#define _GNU_SOURCE
#include "nufht_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ---------------------------------------------------------------------------
 * Tables (format of src/fast_hankel_nufht.c:183-312: magic|version|401|401|32|16,
 * then f64[401][64], f64[401][32][16], i32[401][32][16]).
 * ------------------------------------------------------------------------- */
#define O_NU_ROWS 401
#define O_COEF 64
#define O_I 401
#define O_J 32
#define O_K 16

static double g_coef[O_NU_ROWS][O_COEF];
static double g_z[O_I][O_J][O_K];
static int g_kw[O_I][O_J][O_K];
static int g_tables_ok = 0;
static int g_t3_mode = ORACLE_T3_EXACT;
static int g_threads = 1;

int oracle_load_tables(const char *path)
{
    FILE *f = fopen(path, "rb");
    if (!f) return -2;
    uint32_t hdr[6];
    if (fread(hdr, sizeof(uint32_t), 6, f) != 6) { fclose(f); return -3; }
    if (hdr[0] != 0x4E5546u || hdr[1] != 1u || hdr[2] != O_NU_ROWS || hdr[3] != O_I ||
        hdr[4] != O_J || hdr[5] != O_K) { fclose(f); return -4; }
    size_t n1 = (size_t)O_NU_ROWS * O_COEF, n2 = (size_t)O_I * O_J * O_K;
    if (fread(g_coef, sizeof(double), n1, f) != n1) { fclose(f); return -5; }
    if (fread(g_z, sizeof(double), n2, f) != n2) { fclose(f); return -6; }
    if (fread(g_kw, sizeof(int), n2, f) != n2) { fclose(f); return -7; }
    fclose(f);
    g_tables_ok = 1;
    return 0;
}

void oracle_set_type3_mode(int mode) { g_t3_mode = mode; }
int oracle_get_type3_mode(void) { return g_t3_mode; }
void oracle_set_threads(int nthreads) { g_threads = nthreads < 1 ? 1 : nthreads; }

/* is_integer_double: src/fast_hankel_nufht.c:316-319 */
static int o_is_int(double x) { return fabs(x - nearbyint(x)) < 1e-12; }
/* is_odd_integer_double: src/fast_hankel_nufht.c:848-852 */
static int o_is_odd_int(double x)
{
    long k = (long)llround(x);
    if (!o_is_int(x)) return 0;
    return (k & 1L) != 0;
}

/* fill_plan_parameters: src/fast_hankel_nufht.c:322-414 */
int oracle_plan_params(double nu, double tol, double z_opt, int K_asy_opt, int K_loc_opt,
                       double *z_split, int *K_asy, int *K_loc, double *asy_coef64)
{
    if (tol < 1e-15) return -1;
    int is2 = o_is_int(2.0 * nu), isi = o_is_int(nu);
    if (!is2 || (isi && fabs(nu) > 200.0) || (!isi && is2 && fabs(nu) > 9.5)) return -2;
    if (!g_tables_ok) return -100;
    int i_idx = (int)llround(fabs(nu));
    if (i_idx < 0 || i_idx >= O_I) return -3;
    int row = (int)llround(2.0 * fabs(nu) + 1.0) - 1;
    if (row < 0 || row >= O_NU_ROWS) return -4;
    for (int k = 0; k < O_COEF; ++k) asy_coef64[k] = g_coef[row][k];
    int j = (int)ceil(-log10(tol) - 3.0);
    if (j < 1) j = 1;
    int j_idx = j - 1;
    if (j_idx >= O_J) return -5;
    if (isi) {
        int kv;
        if (K_asy_opt <= 0) {
            int k0 = (int)floor(fabs(nu) / 5.0 + log10(1.0 / tol) / 4.0 + 1.0);
            kv = k0 < 10 ? k0 : 10;
        } else {
            kv = K_asy_opt;
        }
        if (kv < 0 || kv >= O_K) return -6;
        *K_asy = kv;
        *z_split = isnan(z_opt) ? g_z[i_idx][j_idx][kv] : z_opt;
        *K_loc = K_loc_opt <= 0 ? g_kw[i_idx][j_idx][kv] : K_loc_opt;
    } else {
        *K_asy = (int)llround(fabs(nu) - 0.5);
        *z_split = NAN;
        *K_loc = -1;
    }
    return 0;
}

/* ---------------------------------------------------------------------------
 * Planner: src/fast_hankel_nufht.c:416-744 (linear find_first as the reference).
 * ------------------------------------------------------------------------- */
typedef struct { int i0, i1, j0, j1; } OBox;
typedef struct { OBox *d; size_t len, cap; } OVec;

static void ov_push(OVec *v, int i0, int i1, int j0, int j1)
{
    if (v->len == v->cap) {
        size_t nc = v->cap ? 2 * v->cap : 8;
        OBox *t = (OBox *)realloc(v->d, nc * sizeof(OBox));
        if (!t) { fprintf(stderr, "oracle: box alloc failed\n"); abort(); }
        v->d = t; v->cap = nc;
    }
    OBox b = {i0, i1, j0, j1};
    v->d[v->len++] = b;
}

/* find_first_ws_greater / find_first_rs_greater: src/fast_hankel_nufht.c:454-466 */
static int o_first_greater(const double *a, int len, double thr)
{
    for (int i = 0; i < len; ++i)
        if (a[i] > thr) return i;
    return -1;
}

/* splitting_objective: src/fast_hankel_nufht.c:498-521 */
static long long o_split_obj(const double *rs, int m, const double *ws, const OBox *b,
                             double z, int i)
{
    int j = o_first_greater(rs, m, z / ws[i]);
    if (j < 0) return 0;
    return (long long)(i - b->i0 + 1) * (long long)(j - b->j0 + 1) +
           (long long)(b->i1 - i + 1) * (long long)(b->j1 - j + 1);
}

/* split_box: src/fast_hankel_nufht.c:523-574 (ten candidate rows) */
static void o_split_box(const double *rs, int m, const double *ws, const OBox *b, double z,
                        int *ispl, int *jspl)
{
    int cand[10], nc = 0;
    if (b->i1 <= b->i0) {
        cand[0] = b->i0; nc = 1;
    } else {
        for (int k = 0; k < 10; ++k) {
            double t = (double)k / 9.0;
            int idx = (int)llround(b->i0 + t * (double)(b->i1 - b->i0));
            if (idx < b->i0) idx = b->i0;
            if (idx > b->i1) idx = b->i1;
            if (nc == 0 || idx != cand[nc - 1]) cand[nc++] = idx;
        }
    }
    long long best = -1;
    int bi = b->i0;
    for (int c = 0; c < nc; ++c) {
        long long v = o_split_obj(rs, m, ws, b, z, cand[c]);
        if (v > best) { best = v; bi = cand[c]; }
    }
    int j = o_first_greater(rs, m, z / ws[bi]);
    if (j < 0) j = b->j0;
    *ispl = bi; *jspl = j;
}

/* generate_boxes: src/fast_hankel_nufht.c:578-744 */
static void o_boxes(const double *rs, int m, const double *ws, int n, double z, int max_levels,
                    int min_dim_prod, int Kthr, OVec *loc, OVec *asy, OVec *dir)
{
    memset(loc, 0, sizeof *loc); memset(asy, 0, sizeof *asy); memset(dir, 0, sizeof *dir);
    if (n <= 0 || m <= 0) return;
    if (max_levels <= 0) {
        int mn = n < m ? n : m;
        double ratio = (double)mn * (double)mn / (double)min_dim_prod;
        max_levels = ratio < 1.0 ? 0 : (int)floor(log2(ratio));
        if (max_levels < 0) max_levels = 0;
    }
    int i0 = o_first_greater(ws, n, z / rs[m - 1]), i1, j0, j1;
    if (m == 1) {
        i1 = i0 == -1 ? -1 : i0 - 1;
    } else {
        int idx = o_first_greater(ws, n, z / rs[0]);
        i1 = idx == -1 ? n - 1 : idx - 1;
    }
    j0 = o_first_greater(rs, m, z / ws[n - 1]);
    if (n == 1) {
        j1 = j0 == -1 ? -1 : j0 - 1;
    } else {
        int idx = o_first_greater(rs, m, z / ws[0]);
        j1 = idx == -1 ? m - 1 : idx - 1;
    }
    if (i0 == -1) { ov_push(loc, 0, n - 1, 0, m - 1); return; }
    if (i1 < 0) { ov_push(asy, 0, n - 1, 0, m - 1); return; }
    if (i0 > 0) ov_push(loc, 0, i0 - 1, 0, m - 1);
    if (j0 > 0) ov_push(loc, i0, n - 1, 0, j0 - 1);
    if (i1 < n - 1) ov_push(asy, i1 + 1, n - 1, 0, m - 1);
    if (j1 < m - 1) ov_push(asy, 0, i1, j1 + 1, m - 1);
    if (m == 1 || n == 1) return;
    ov_push(dir, i0, i1, j0, j1);
    for (int lev = 0; lev < max_levels; ++lev) {
        OVec nd; memset(&nd, 0, sizeof nd);
        for (size_t q = 0; q < dir->len; ++q) {
            OBox b = dir->d[q];
            long long d1 = b.i1 - b.i0 + 1, d2 = b.j1 - b.j0 + 1;
            if (d1 * d2 > 4LL * (long long)min_dim_prod) {
                int is, js;
                o_split_box(rs, m, ws, &b, z, &is, &js);
                if (is > b.i0) {
                    ov_push(loc, b.i0, is - 1, b.j0, js - 1);
                    ov_push(&nd, b.i0, is - 1, js, b.j1);
                }
                ov_push(asy, is, b.i1, js, b.j1);
                ov_push(&nd, is, b.i1, b.j0, js - 1);
            } else {
                ov_push(&nd, b.i0, b.i1, b.j0, b.j1);
            }
        }
        free(dir->d);
        *dir = nd;
    }
    OVec nl, na; memset(&nl, 0, sizeof nl); memset(&na, 0, sizeof na);
    for (size_t q = 0; q < loc->len; ++q) {
        OBox b = loc->d[q];
        int d1 = b.i1 - b.i0 + 1, d2 = b.j1 - b.j0 + 1;
        if ((d1 < d2 ? d1 : d2) < Kthr) ov_push(dir, b.i0, b.i1, b.j0, b.j1);
        else ov_push(&nl, b.i0, b.i1, b.j0, b.j1);
    }
    for (size_t q = 0; q < asy->len; ++q) {
        OBox b = asy->d[q];
        long long area = (long long)(b.i1 - b.i0 + 1) * (long long)(b.j1 - b.j0 + 1);
        if (area < (long long)min_dim_prod) ov_push(dir, b.i0, b.i1, b.j0, b.j1);
        else ov_push(&na, b.i0, b.i1, b.j0, b.j1);
    }
    free(loc->d); free(asy->d);
    *loc = nl; *asy = na;
}

long oracle_generate_boxes(const double *rs, int m, const double *ws, int n, double z_split,
                           int max_levels, int min_dim_prod, int K_loc_threshold, long *counts,
                           int *out, long cap)
{
    OVec L, A, D;
    o_boxes(rs, m, ws, n, z_split, max_levels, min_dim_prod, K_loc_threshold, &L, &A, &D);
    counts[0] = (long)L.len; counts[1] = (long)A.len; counts[2] = (long)D.len;
    long tot = counts[0] + counts[1] + counts[2];
    if (out && cap >= tot) {
        long p = 0;
        OVec *vs[3] = {&L, &A, &D};
        for (int v = 0; v < 3; ++v)
            for (size_t q = 0; q < vs[v]->len; ++q) {
                out[4 * p + 0] = vs[v]->d[q].i0; out[4 * p + 1] = vs[v]->d[q].i1;
                out[4 * p + 2] = vs[v]->d[q].j0; out[4 * p + 3] = vs[v]->d[q].j1;
                ++p;
            }
    }
    free(L.d); free(A.d); free(D.d);
    return tot;
}

/* ---------------------------------------------------------------------------
 * Bessel functions standing in for GSL (ORACLE ONLY).
 * Integer orders: the C library's jn().  Half-integer orders nu = n + 1/2:
 * J_nu(x) = sqrt(2x/pi) j_n(x) with j_0 = sin x / x, j_1 = sin x/x^2 - cos x/x and
 * the upward recurrence j_{k+1} = (2k+1)/x j_k - j_{k-1} for x >= n; the power
 * series of J_nu for x < n.
 * ------------------------------------------------------------------------- */
static double o_jhalf(int n, double x)
{
    double nu = n + 0.5;
    if (x == 0.0) return 0.0;
    if (x < (n > 1 ? (double)n : 1.0)) {
        double h = 0.5 * x;
        double t = exp(nu * log(h) - lgamma(nu + 1.0)), s = t, q = -h * h;
        for (int k = 1; k < 500; ++k) {
            t *= q / (k * (nu + k));
            s += t;
            if (fabs(t) <= 1e-17 * fabs(s)) break;
        }
        return s;
    }
    double sn = sin(x), cs = cos(x);
    double a = sn / x;
    if (n == 0) return sqrt(2.0 * x / M_PI) * a;
    double b = sn / (x * x) - cs / x;
    for (int k = 1; k < n; ++k) {
        double c = ((2.0 * k + 1.0) / x) * b - a;
        a = b; b = c;
    }
    return sqrt(2.0 * x / M_PI) * b;
}

double oracle_besselj(double nu, double x)
{
    double an = fabs(nu);
    if (o_is_int(an)) return jn((int)llround(an), x);
    return o_jhalf((int)llround(an - 0.5), x);
}

void oracle_besselj_all(int nmax, double z, double *out)
{
    for (int k = 0; k <= nmax; ++k) out[k] = jn(k, z);
}

/* ---------------------------------------------------------------------------
 * Type-3 transform stand-in for finufft1d3many (src/expansions.c:368-397):
 *   fk[t][k] = sum_j cj[t][j] exp(+i sk[k] xj[j]),  iflag = +1.
 * ------------------------------------------------------------------------- */
static void o_fft_pos(double *a, int n) /* in place, sum_l a_l e^{+2 pi i q l / n}, n = 2^p */
{
    for (int i = 1, j = 0; i < n; ++i) {
        int bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            double tr = a[2 * i], ti = a[2 * i + 1];
            a[2 * i] = a[2 * j]; a[2 * i + 1] = a[2 * j + 1];
            a[2 * j] = tr; a[2 * j + 1] = ti;
        }
    }
    /* twiddles exp(2 pi i k / n), k < n/2, computed once */
    double *tw = (double *)malloc(sizeof(double) * (size_t)(n > 1 ? n : 2));
    for (int k = 0; k < n / 2; ++k) {
        tw[2 * k] = cos(2.0 * M_PI * k / n);
        tw[2 * k + 1] = sin(2.0 * M_PI * k / n);
    }
    for (int len = 2; len <= n; len <<= 1) {
        int step = n / len;
        for (int i = 0; i < n; i += len) {
            for (int k = 0; k < len / 2; ++k) {
                double wr = tw[2 * k * step], wi = tw[2 * k * step + 1];
                double *u = a + 2 * (i + k), *v = a + 2 * (i + k + len / 2);
                double vr = v[0] * wr - v[1] * wi, vi = v[0] * wi + v[1] * wr;
                v[0] = u[0] - vr; v[1] = u[1] - vi;
                u[0] += vr; u[1] += vi;
            }
        }
    }
    free(tw);
}

static double o_es(double u, int w, double beta) /* ES kernel in grid units, support |u|<w/2 */
{
    double z = 2.0 * u / w;
    if (fabs(z) >= 1.0) return 0.0;
    return exp(beta * (sqrt(1.0 - z * z) - 1.0));
}

/* Gauss-Legendre nodes on [-1,1] by Newton iteration on P_n. */
static void o_gauss(int n, double *x, double *wt)
{
    for (int i = 0; i < n; ++i) {
        double z = cos(M_PI * (i + 0.75) / (n + 0.5)), pp = 0.0;
        for (int it = 0; it < 100; ++it) {
            double p1 = 1.0, p2 = 0.0;
            for (int j = 1; j <= n; ++j) {
                double p3 = p2; p2 = p1;
                p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
            }
            pp = n * (z * p1 - p2) / (z * z - 1.0);
            double dz = p1 / pp;
            z -= dz;
            if (fabs(dz) < 1e-16) break;
        }
        x[i] = z; wt[i] = 2.0 / ((1.0 - z * z) * pp * pp);
    }
}

typedef struct { int w; double beta; int nq; double qx[64], qw[64], qpsi[64]; } OKer;

static void o_ker_init(OKer *K, double eps)
{
    int w = (int)ceil(log10(1.0 / eps)) + 1;
    if (w < 2) w = 2;
    if (w > 16) w = 16;
    K->w = w; K->beta = 2.30 * w; K->nq = 2 * w + 16;
    double x[64], wt[64];
    o_gauss(K->nq, x, wt);
    for (int i = 0; i < K->nq; ++i) {
        K->qx[i] = (x[i] + 1.0) * 0.25 * w;  /* nodes on [0, w/2] */
        K->qw[i] = wt[i] * 0.25 * w;
        K->qpsi[i] = o_es(K->qx[i], w, K->beta);
    }
}

static double o_ker_hat(const OKer *K, double om) /* int psi(u) cos(om u) du */
{
    double s = 0.0;
    for (int i = 0; i < K->nq; ++i) s += K->qw[i] * K->qpsi[i] * cos(om * K->qx[i]);
    return 2.0 * s;
}

/* Per-box setup of the type-3 transform: grid geometry, kernel weights and phases of the
 * sources and targets, deconvolution factors.  The reference calls finufft1d3many 2(K+1)
 * times per box on the same points (src/expansions.c:499-557); the stand-in keeps the last
 * setup of each thread and reuses it when the next call has the same points, which makes
 * the CPU baseline faster than per-call setup, never slower. */
typedef struct {
    const double *xj, *sk;
    int nj, nk;
    double eps;
    int w;
    double C, D, h;
    long half, n2;
    double *wts, *ph, *corr, *kw, *post;
    long *l0s, *q0s;
} O3Setup;

static __thread O3Setup t3_cache;

static void o3_free(O3Setup *S)
{
    free(S->wts); free(S->ph); free(S->corr); free(S->kw); free(S->post); free(S->l0s); free(S->q0s);
    memset(S, 0, sizeof(*S));
}

static int o3_setup(O3Setup *S, int nj, const double *xj, double eps, int nk, const double *sk)
{
    if (S->wts && S->xj == xj && S->nj == nj && S->sk == sk && S->nk == nk && S->eps == eps) return 0;
    o3_free(S);
    OKer K; o_ker_init(&K, eps);
    int w = K.w;
    double xmin = xj[0], xmax = xj[0], smin = sk[0], smax = sk[0];
    for (int j = 1; j < nj; ++j) { if (xj[j] < xmin) xmin = xj[j]; if (xj[j] > xmax) xmax = xj[j]; }
    for (int k = 1; k < nk; ++k) { if (sk[k] < smin) smin = sk[k]; if (sk[k] > smax) smax = sk[k]; }
    double C = 0.5 * (xmin + xmax), X = 0.5 * (xmax - xmin);
    double D = 0.5 * (smin + smax), S_ = 0.5 * (smax - smin);
    if (S_ < 1e-12 * (fabs(D) + 1.0)) S_ = 1e-12 * (fabs(D) + 1.0);
    double h = M_PI / (2.0 * S_);
    long half = (long)ceil(X / h + 0.5 * w);
    long L1 = 2 * half + 1;
    long n2 = 2;
    while (n2 < 2 * L1) n2 *= 2;
    if (n2 > (1L << 28)) return -1;
    S->wts = (double *)malloc(sizeof(double) * (size_t)w * (size_t)nj);
    S->l0s = (long *)malloc(sizeof(long) * (size_t)nj);
    S->ph = (double *)malloc(sizeof(double) * 2 * (size_t)nj);
    S->corr = (double *)malloc(sizeof(double) * (size_t)L1);
    S->kw = (double *)malloc(sizeof(double) * (size_t)w * (size_t)nk);
    S->q0s = (long *)malloc(sizeof(long) * (size_t)nk);
    S->post = (double *)malloc(sizeof(double) * 2 * (size_t)nk);
    if (!S->wts || !S->l0s || !S->ph || !S->corr || !S->kw || !S->q0s || !S->post) { o3_free(S); return -2; }
    for (int j = 0; j < nj; ++j) {
        double x = xj[j] - C, u = x / h;
        long l0 = (long)ceil(u - 0.5 * w);
        S->l0s[j] = l0;
        for (int t = 0; t < w; ++t) S->wts[(size_t)j * w + t] = o_es((double)(l0 + t) - u, w, K.beta);
        S->ph[2 * j] = cos(D * x); S->ph[2 * j + 1] = sin(D * x);
    }
    for (long l = -half; l <= half; ++l) S->corr[l + half] = 1.0 / o_ker_hat(&K, 2.0 * M_PI * l / n2);
    for (int k = 0; k < nk; ++k) {
        double th = (sk[k] - D) * h, u = th * n2 / (2.0 * M_PI);
        long q0 = (long)ceil(u - 0.5 * w);
        S->q0s[k] = q0;
        for (int t = 0; t < w; ++t) S->kw[(size_t)k * w + t] = o_es(u - (double)(q0 + t), w, K.beta);
        double sc = 1.0 / o_ker_hat(&K, th);
        S->post[2 * k] = sc * cos(sk[k] * C); S->post[2 * k + 1] = sc * sin(sk[k] * C);
    }
    S->xj = xj; S->sk = sk; S->nj = nj; S->nk = nk; S->eps = eps;
    S->w = w; S->C = C; S->D = D; S->h = h; S->half = half; S->n2 = n2;
    return 0;
}

static int o_type3_nufft(int ntr, int nj, const double *xj, const double *cj, double eps,
                         int nk, const double *sk, double *fk)
{
    O3Setup *S = &t3_cache;
    int rc = o3_setup(S, nj, xj, eps, nk, sk);
    if (rc) return rc;
    const int w = S->w;
    const long half = S->half, n2 = S->n2;
    double *b = (double *)malloc(sizeof(double) * 2 * (size_t)n2);
    if (!b) return -2;
    for (int tr = 0; tr < ntr; ++tr) {
        const double *c = cj + 2 * (size_t)tr * nj;
        double *f = fk + 2 * (size_t)tr * nk;
        memset(b, 0, sizeof(double) * 2 * (size_t)n2);
        for (int j = 0; j < nj; ++j) {
            double ar = c[2 * j] * S->ph[2 * j] - c[2 * j + 1] * S->ph[2 * j + 1];
            double ai = c[2 * j] * S->ph[2 * j + 1] + c[2 * j + 1] * S->ph[2 * j];
            for (int t = 0; t < w; ++t) {
                long l = S->l0s[j] + t;
                long idx = ((l % n2) + n2) % n2;
                double wv = S->wts[(size_t)j * w + t];
                b[2 * idx] += wv * ar; b[2 * idx + 1] += wv * ai;
            }
        }
        for (long l = -half; l <= half; ++l) {
            long idx = ((l % n2) + n2) % n2;
            b[2 * idx] *= S->corr[l + half]; b[2 * idx + 1] *= S->corr[l + half];
        }
        o_fft_pos(b, (int)n2);
        for (int k = 0; k < nk; ++k) {
            double sr = 0.0, si = 0.0;
            for (int t = 0; t < w; ++t) {
                long q = S->q0s[k] + t;
                long idx = ((q % n2) + n2) % n2;
                double wv = S->kw[(size_t)k * w + t];
                sr += wv * b[2 * idx]; si += wv * b[2 * idx + 1];
            }
            f[2 * k] = sr * S->post[2 * k] - si * S->post[2 * k + 1];
            f[2 * k + 1] = sr * S->post[2 * k + 1] + si * S->post[2 * k];
        }
    }
    free(b);
    return 0;
}

static void o_type3_exact(int ntr, int nj, const double *xj, const double *cj, int nk,
                          const double *sk, double *fk)
{
#pragma omp parallel for schedule(dynamic, 16) num_threads(g_threads)
    for (int k = 0; k < nk; ++k) {
        for (int tr = 0; tr < ntr; ++tr) {
            const double *c = cj + 2 * (size_t)tr * nj;
            double sr = 0.0, si = 0.0;
            for (int j = 0; j < nj; ++j) {
                double s, co;
                sincos(sk[k] * xj[j], &s, &co);
                sr += c[2 * j] * co - c[2 * j + 1] * s;
                si += c[2 * j] * s + c[2 * j + 1] * co;
            }
            fk[2 * ((size_t)tr * nk + k)] = sr;
            fk[2 * ((size_t)tr * nk + k) + 1] = si;
        }
    }
}

int oracle_type3(int ntr, int nj, const double *xj, const double *cj, double eps, int nk,
                 const double *sk, double *fk)
{
    if (g_t3_mode == ORACLE_T3_EXACT) {
        o_type3_exact(ntr, nj, xj, cj, nk, sk, fk);
        return 0;
    }
    if (g_threads > 1 && ntr > 1) {
        int err = 0;
#pragma omp parallel for schedule(dynamic, 1) num_threads(g_threads) reduction(| : err)
        for (int tr = 0; tr < ntr; ++tr)
            err |= o_type3_nufft(1, nj, xj, cj + 2 * (size_t)tr * nj, eps, nk, sk,
                                 fk + 2 * (size_t)tr * nk);
        return err;
    }
    return o_type3_nufft(ntr, nj, xj, cj, eps, nk, sk, fk);
}

/* ---------------------------------------------------------------------------
 * Evaluators (src/expansions.c).
 * ------------------------------------------------------------------------- */

/* add_dir: src/expansions.c:61-76 */
void oracle_add_dir(double *gs, double nu, const double *rs, const double *cs,
                    const double *ws, int m, int n)
{
    for (int j = 0; j < n; ++j) {
        double s = gs[j];
        for (int k = 0; k < m; ++k) s += cs[k] * oracle_besselj(nu, ws[j] * rs[k]);
        gs[j] = s;
    }
}

/* add_dir_batch: src/expansions.c:78-97 (one Bessel value per (target, source), reused
 * across the batch columns). */
void oracle_add_dir_batch(double *gs, double nu, const double *rs, const double *cs,
                          const double *ws, int m, int n, int batch, int ld_cs, int ld_gs)
{
#pragma omp parallel for schedule(dynamic, 4) num_threads(g_threads)
    for (int j = 0; j < n; ++j) {
        double wj = ws[j];
        for (int k = 0; k < m; ++k) {
            double J = oracle_besselj(nu, wj * rs[k]);
            for (int t = 0; t < batch; ++t)
                gs[(size_t)t * ld_gs + j] += cs[(size_t)t * ld_cs + k] * J;
        }
    }
}

/* Chebyshev weight of source x = r/r_end for term l: src/expansions.c:242-273. */
static double o_cheb_val(int nu_int, int l, double x)
{
    if (x > 1.0) x = 1.0;
    if (x < -1.0) x = -1.0;
    double th = acos(x);
    if (nu_int == 0) {
        double cl = cos((double)l * th);
        return (l == 0 ? 1.0 : 2.0) * (2.0 * cl * cl - 1.0);
    } else if ((nu_int & 1) == 0) {
        return (l == 0 ? 1.0 : 2.0) * cos(2.0 * (double)l * th);
    }
    return 2.0 * cos((double)(2 * l + 1) * th);
}

/* Bessel products b[l] of the Wimp expansion at z: src/expansions.c:280-328. */
static void o_loc_products(int nu_int, int K, double z, double *b1, double *b2)
{
    int l0 = nu_int / 2, odd = nu_int & 1;
    if (nu_int == 0) {
        for (int l = 0; l <= K; ++l) {
            double J = jn(l, z);
            b1[l] = J * J * ((l & 1) ? -1.0 : 1.0);
        }
        return;
    }
    int maxo = l0 + K + odd;
    for (int k = 0; k <= maxo; ++k) b2[k] = jn(k, z);
    int st = l0 + odd;
    for (int l = 0; l <= K; ++l) b1[l] = b2[st + l];
    for (int t = 0; t <= l0; ++t) {
        int i = l0 - t;
        if (i >= 0 && i <= K) b1[i] *= b2[t];
    }
    for (int q = 0; q < K - l0; ++q) {
        int i = l0 + 1 + q, i2 = 1 + q;
        if (i <= K && i2 <= maxo) b1[i] *= b2[i2];
    }
    for (int l = l0 + 1; l <= K; l += 2) b1[l] = -b1[l];
}

/* add_loc: src/expansions.c:99-210 */
void oracle_add_loc(double *gs, double nu, const double *rs, const double *cs,
                    const double *ws, int m, int n, int K, double *cheb_buffer,
                    double *bessel_buffer_1, double *bessel_buffer_2)
{
    oracle_add_loc_batch(gs, nu, rs, cs, ws, m, n, K, 1, m, n, cheb_buffer, bessel_buffer_1,
                         bessel_buffer_2);
}

/* add_loc_batch: src/expansions.c:212-337 */
void oracle_add_loc_batch(double *gs, double nu, const double *rs, const double *cs,
                          const double *ws, int m, int n, int K, int batch, int ld_cs, int ld_gs,
                          double *cheb, double *bb1, double *bb2)
{
    (void)bb1; (void)bb2;
    int nu_int = (int)llround(nu);
    if (fabs(nu - (double)nu_int) > 1e-12) { fprintf(stderr, "add_loc_batch: nu must be integer\n"); return; }
    double r_end = rs[m - 1];
    int stride = K + 1;
    for (int t = 0; t < batch; ++t)
        for (int l = 0; l <= K; ++l) cheb[(size_t)t * stride + l] = 0.0;
#pragma omp parallel for schedule(static) num_threads(g_threads)
    for (int l = 0; l <= K; ++l) {
        for (int k = 0; k < m; ++k) {
            /* r_end = 0 (all sources at the origin): the reference divides by zero and
             * returns NaN; only the l = 0 term survives there, so any x serves. */
            double v = o_cheb_val(nu_int, l, r_end > 0.0 ? rs[k] / r_end : 0.0);
            for (int t = 0; t < batch; ++t) cheb[(size_t)t * stride + l] += v * cs[(size_t)t * ld_cs + k];
        }
    }
    int l0 = nu_int / 2;
    int nb2 = l0 + K + 2;
#pragma omp parallel num_threads(g_threads)
    {
        double *b1 = (double *)malloc(sizeof(double) * (size_t)(K + 1));
        double *b2 = (double *)malloc(sizeof(double) * (size_t)nb2);
#pragma omp for schedule(static)
        for (int j = 0; j < n; ++j) {
            o_loc_products(nu_int, K, ws[j] * r_end / 2.0, b1, b2);
            for (int t = 0; t < batch; ++t) {
                double acc = 0.0;
                for (int l = 0; l <= K; ++l) acc += b1[l] * cheb[(size_t)t * stride + l];
                gs[(size_t)t * ld_gs + j] += acc;
            }
        }
        free(b1); free(b2);
    }
}

/* add_asy_batch: src/expansions.c:483-559.  For each l = 0..K, two type-3 transforms
 * with inputs c r^{-2l-1/2} and c r^{-2l-3/2}; outputs rotated by exp(i pi(-nu/2-1/4))
 * and scaled by sqrt(2/pi)(-1)^l a_{2l} k^{-2l-1/2} (real part added) and
 * sqrt(2/pi)(-1)^l a_{2l+1} k^{-2l-3/2} (imaginary part subtracted). */
void oracle_add_asy_batch(double *gs, double nu, const double *rs, const double *cs,
                          const double *ws, int m, int n, int K, double tol,
                          const double *asy_coef, int batch, int ld_cs, int ld_gs,
                          double *in_buffer, double *out_buffer)
{
    double *cin = in_buffer, *cout = out_buffer;
    int own = 0;
    if (!cin || !cout) {
        cin = (double *)malloc(sizeof(double) * 2 * (size_t)m * batch);
        cout = (double *)malloc(sizeof(double) * 2 * (size_t)n * batch);
        own = 1;
    }
    double s2p = sqrt(2.0 / M_PI);
    double pa = M_PI * (-nu / 2.0 - 0.25);
    double pr = cos(pa), pi_ = sin(pa);
    if (g_t3_mode == ORACLE_T3_NUFFT && g_threads > 1 && K >= 0) {
        /* Parallel over the 2(K+1) independent transforms (the reference runs them one after
         * another); the terms are added to gs in the reference's order. */
        int nq = 2 * (K + 1), err = 0;
        double *terms = (double *)malloc(sizeof(double) * (size_t)nq * n * batch);
#pragma omp parallel for schedule(dynamic, 1) num_threads(g_threads) reduction(| : err)
        for (int q = 0; q < nq; ++q) {
            int l = q / 2, half = q & 1;
            int e = half == 0 ? -2 * l - 1 : -2 * l - 2;
            double *ci = (double *)malloc(sizeof(double) * 2 * (size_t)m * batch);
            double *co = (double *)malloc(sizeof(double) * 2 * (size_t)n * batch);
            for (int t = 0; t < batch; ++t)
                for (int k = 0; k < m; ++k) {
                    double rk = rs[k];
                    ci[2 * ((size_t)t * m + k)] = cs[(size_t)t * ld_cs + k] * pow(rk, (double)e) * sqrt(rk);
                    ci[2 * ((size_t)t * m + k) + 1] = 0.0;
                }
            err |= o_type3_nufft(batch, m, rs, ci, tol, n, ws, co);
            double sl = (l & 1) ? -1.0 : 1.0;
            double coeff = s2p * sl * asy_coef[2 * l + half];
            double *tq = terms + (size_t)q * n * batch;
            for (int t = 0; t < batch; ++t)
                for (int j = 0; j < n; ++j) {
                    double wj = ws[j];
                    double sc = coeff * pow(wj, (double)e) * sqrt(wj);
                    double fr = co[2 * ((size_t)t * n + j)], fi = co[2 * ((size_t)t * n + j) + 1];
                    double vr = fr * pr - fi * pi_, vi = fr * pi_ + fi * pr;
                    tq[(size_t)t * n + j] = half == 0 ? vr * sc : -vi * sc;
                }
            free(ci);
            free(co);
        }
        if (err) fprintf(stderr, "oracle add_asy_batch: type-3 failed\n");
        for (int q = 0; q < nq; ++q)
            for (int t = 0; t < batch; ++t)
                for (int j = 0; j < n; ++j) gs[(size_t)t * ld_gs + j] += terms[((size_t)q * batch + t) * n + j];
        free(terms);
        if (own) { free(cin); free(cout); }
        return;
    }
    for (int l = 0; l <= K; ++l) {
        for (int half = 0; half < 2; ++half) {
            int e = half == 0 ? -2 * l - 1 : -2 * l - 2;
            for (int t = 0; t < batch; ++t)
                for (int k = 0; k < m; ++k) {
                    double rk = rs[k];
                    cin[2 * ((size_t)t * m + k)] = cs[(size_t)t * ld_cs + k] * pow(rk, (double)e) * sqrt(rk);
                    cin[2 * ((size_t)t * m + k) + 1] = 0.0;
                }
            if (oracle_type3(batch, m, rs, cin, tol, n, ws, cout) != 0) {
                fprintf(stderr, "oracle add_asy_batch: type-3 failed\n");
                goto done;
            }
            double sl = (l & 1) ? -1.0 : 1.0;
            double coeff = s2p * sl * asy_coef[2 * l + half];
            for (int t = 0; t < batch; ++t)
                for (int j = 0; j < n; ++j) {
                    double wj = ws[j];
                    double sc = coeff * pow(wj, (double)e) * sqrt(wj);
                    double fr = cout[2 * ((size_t)t * n + j)], fi = cout[2 * ((size_t)t * n + j) + 1];
                    double vr = fr * pr - fi * pi_, vi = fr * pi_ + fi * pr;
                    if (half == 0) gs[(size_t)t * ld_gs + j] += vr * sc;
                    else gs[(size_t)t * ld_gs + j] -= vi * sc;
                }
        }
    }
done:
    if (own) { free(cin); free(cout); }
}

/* add_asy: src/expansions.c:399-481 */
void oracle_add_asy(double *gs, double nu, const double *rs, const double *cs,
                    const double *ws, int m, int n, int K, double tol, const double *asy_coef,
                    double *real_buffer_1, double *real_buffer_2, double *in_buffer,
                    double *out_buffer)
{
    (void)real_buffer_1; (void)real_buffer_2;
    oracle_add_asy_batch(gs, nu, rs, cs, ws, m, n, K, tol, asy_coef, 1, m, n, in_buffer,
                         out_buffer);
}

/* ---------------------------------------------------------------------------
 * Driver: nufht_plan_init (src/fast_hankel_nufht.c:759-786) + nufht_batch (:989-1107).
 * ------------------------------------------------------------------------- */
int oracle_nufht_batch(double nu, const double *rs, int m, const double *ws, int n,
                       const double *cs, int ld_cs, double *gs, int ld_gs, int batch, double tol,
                       int max_levels, int min_dim_prod, double z_opt, int K_asy_opt,
                       int K_loc_opt, int faithful)
{
    if (!rs || !ws || m <= 0 || n <= 0) return -200;
    double z, coef[64];
    int Ka, Kl;
    int rc = oracle_plan_params(nu, tol, z_opt, K_asy_opt, K_loc_opt, &z, &Ka, &Kl, coef);
    if (rc) return rc;
    if (!cs || !gs || batch <= 0) return -400;
    if (ld_cs < m || ld_gs < n) return -401;
    OVec L, A, D;
    o_boxes(rs, m, ws, n, z, max_levels, min_dim_prod, Kl < 0 ? 0 : Kl, &L, &A, &D);
    for (int t = 0; t < batch; ++t) memset(gs + (size_t)t * ld_gs, 0, sizeof(double) * (size_t)n);
    long long dp = (long long)m * (long long)n;
    int use_direct = dp < (long long)min_dim_prod;
    int nu_int = o_is_int(nu);
    double anu = fabs(nu);
    size_t cheb_len = (size_t)(Kl < 0 ? 1 : Kl + 1) * (size_t)batch;
    double *cheb = (double *)calloc(cheb_len, sizeof(double));
    int nb = (int)(anu / 2) + (Kl < 0 ? 0 : Kl) + 3;
    double *b1 = (double *)calloc((size_t)nb, sizeof(double));
    double *b2 = (double *)calloc((size_t)nb, sizeof(double));
    if (use_direct) {
        /* The reference passes the signed nu here (:1049); the oracle uses |nu|, as
         * every other path does, with the sign of J_{-n} applied below. */
        oracle_add_dir_batch(gs, anu, rs, cs, ws, m, n, batch, ld_cs, ld_gs);
    } else if (!nu_int) {
        oracle_add_asy_batch(gs, anu, rs, cs, ws, m, n, Ka, tol, coef, batch, ld_cs, ld_gs,
                             NULL, NULL);
    } else {
        for (size_t q = 0; q < L.len && Kl >= 0; ++q) {
            OBox b = L.d[q];
            oracle_add_loc_batch(gs + b.i0, anu, rs + b.j0, cs + b.j0, ws + b.i0, b.j1 - b.j0 + 1,
                                 b.i1 - b.i0 + 1, Kl, batch, ld_cs, ld_gs, cheb, b1, b2);
        }
        for (size_t q = 0; q < A.len; ++q) {
            OBox b = A.d[q];
            oracle_add_asy_batch(gs + b.i0, anu, rs + b.j0, cs + b.j0, ws + b.i0, b.j1 - b.j0 + 1,
                                 b.i1 - b.i0 + 1, Ka, tol, coef, batch, ld_cs, ld_gs, NULL, NULL);
        }
        for (size_t q = 0; q < D.len; ++q) {
            OBox b = D.d[q];
            oracle_add_dir_batch(gs + b.i0, anu, rs + b.j0, cs + b.j0, ws + b.i0, b.j1 - b.j0 + 1,
                                 b.i1 - b.i0 + 1, batch, ld_cs, ld_gs);
        }
        /* execute_boxes_single negates once more for batch == 1 (:916-920). */
        if (faithful && batch == 1 && nu < 0.0 && o_is_odd_int(nu))
            for (int i = 0; i < n; ++i) gs[i] = -gs[i];
    }
    if (nu < 0.0 && o_is_odd_int(nu))
        for (int t = 0; t < batch; ++t)
            for (int i = 0; i < n; ++i) gs[(size_t)t * ld_gs + i] = -gs[(size_t)t * ld_gs + i];
    free(cheb); free(b1); free(b2);
    free(L.d); free(A.d); free(D.d);
    return 0;
}

void oracle_direct_sum(double nu, const double *rs, int m, const double *ws, const double *cs,
                       int ld_cs, int batch, const long *idx, int nidx, double *out)
{
    double sgn = (nu < 0.0 && o_is_odd_int(nu)) ? -1.0 : 1.0;
    double anu = fabs(nu);
#pragma omp parallel for schedule(dynamic, 1) num_threads(g_threads)
    for (int q = 0; q < nidx; ++q) {
        double k = ws[idx[q]];
        double *acc = (double *)calloc((size_t)batch, sizeof(double));
        double *cmp = (double *)calloc((size_t)batch, sizeof(double));
        for (int j = 0; j < m; ++j) {
            double J = oracle_besselj(anu, k * rs[j]);
            for (int t = 0; t < batch; ++t) { /* Kahan-compensated sum */
                double y = cs[(size_t)t * ld_cs + j] * J - cmp[t];
                double s = acc[t] + y;
                cmp[t] = (s - acc[t]) - y;
                acc[t] = s;
            }
        }
        for (int t = 0; t < batch; ++t) out[(size_t)t * nidx + q] = sgn * acc[t];
        free(acc); free(cmp);
    }
}
