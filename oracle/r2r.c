/*
 * r2r.c -- FP64 r2r transforms for the oracle (test infrastructure only; never shipped
 * in the product path).  Definitions and reductions are documented in r2r.h.
 */
#include "r2r.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_MAX_N 8192
#define ORC_MAX_STAGES 32

typedef struct {
    int n;
    int nstages;
    int radix[ORC_MAX_STAGES];
    double *wre, *wim;   /* W_n^m = exp(-2 pi i m / n), m < n */
    double *tre, *tim;   /* Makhoul twiddle exp(-i pi k / (2n)), k < n */
} orc_plan;

static orc_plan *g_plans[ORC_MAX_N + 1];
static int g_threads = 0;

void orc_set_threads(int nthreads) { g_threads = nthreads; }

int orc_get_threads(void)
{
#ifdef _OPENMP
    return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
    return 1;
#endif
}

static orc_plan *plan_build(int n)
{
    orc_plan *p = (orc_plan *)calloc(1, sizeof(orc_plan));
    p->n = n;
    int m = n, s = 0;
    /* radix-4 first, then 2, 3, 5, then any remaining prime factor (generic DFT) */
    while (m % 4 == 0) { p->radix[s++] = 4; m /= 4; }
    while (m % 2 == 0) { p->radix[s++] = 2; m /= 2; }
    while (m % 3 == 0) { p->radix[s++] = 3; m /= 3; }
    while (m % 5 == 0) { p->radix[s++] = 5; m /= 5; }
    for (int f = 7; m > 1; f += 2) {
        while (m % f == 0) { p->radix[s++] = f; m /= f; }
    }
    p->nstages = s;
    p->wre = (double *)malloc(sizeof(double) * n);
    p->wim = (double *)malloc(sizeof(double) * n);
    p->tre = (double *)malloc(sizeof(double) * n);
    p->tim = (double *)malloc(sizeof(double) * n);
    for (int k = 0; k < n; k++) {
        double a = -2.0 * M_PI * (double)k / (double)n;
        p->wre[k] = cos(a);
        p->wim[k] = sin(a);
        double b = -M_PI * (double)k / (2.0 * (double)n);
        p->tre[k] = cos(b);
        p->tim[k] = sin(b);
    }
    return p;
}

static orc_plan *plan_get(int n)
{
    orc_plan *p = g_plans[n];
    if (p) return p;
#pragma omp critical(orc_plan_cache)
    {
        if (!g_plans[n]) g_plans[n] = plan_build(n);
        p = g_plans[n];
    }
    return p;
}

/* Stockham auto-sort complex FFT, sign = -1 forward, +1 backward (unnormalised).
 * Data in (are, aim); (bre, bim) is scratch.  Result returned through the pointers. */
static void fft_stockham(const orc_plan *p, double **are, double **aim, double **bre, double **bim,
                         int sign)
{
    const int n = p->n;
    int ns = 1;
    double vr[64], vi[64], ur[64], ui[64];
    for (int s = 0; s < p->nstages; s++) {
        const int r = p->radix[s];
        const int m = n / r;
        const int tstep = n / (ns * r);
        double *ar = *are, *ai = *aim, *br = *bre, *bi = *bim;
        for (int j = 0; j < m; j++) {
            const int k = j % ns;
            for (int q = 0; q < r; q++) {
                double xr = ar[j + q * m], xi = ai[j + q * m];
                int t = (k * q * tstep) % n;
                double wr = p->wre[t], wi = -sign * p->wim[t];
                vr[q] = xr * wr - xi * wi;
                vi[q] = xr * wi + xi * wr;
            }
            /* size-r DFT */
            if (r == 2) {
                ur[0] = vr[0] + vr[1]; ui[0] = vi[0] + vi[1];
                ur[1] = vr[0] - vr[1]; ui[1] = vi[0] - vi[1];
            } else if (r == 4) {
                double s0r = vr[0] + vr[2], s0i = vi[0] + vi[2];
                double d0r = vr[0] - vr[2], d0i = vi[0] - vi[2];
                double s1r = vr[1] + vr[3], s1i = vi[1] + vi[3];
                double d1r = vr[1] - vr[3], d1i = vi[1] - vi[3];
                /* multiply d1 by -i*sign... forward (sign=-1): X1 = d0 - i d1 */
                double jr = -sign * d1i, ji = sign * d1r; /* sign*i*d1 */
                ur[0] = s0r + s1r; ui[0] = s0i + s1i;
                ur[2] = s0r - s1r; ui[2] = s0i - s1i;
                ur[1] = d0r + jr;  ui[1] = d0i + ji;
                ur[3] = d0r - jr;  ui[3] = d0i - ji;
            } else {
                for (int a = 0; a < r; a++) {
                    double sr = 0.0, si = 0.0;
                    for (int b = 0; b < r; b++) {
                        int t = ((a * b) % r) * m;
                        double wr = p->wre[t], wi = -sign * p->wim[t];
                        sr += vr[b] * wr - vi[b] * wi;
                        si += vr[b] * wi + vi[b] * wr;
                    }
                    ur[a] = sr; ui[a] = si;
                }
            }
            const int dst = (j / ns) * ns * r + k;
            for (int q = 0; q < r; q++) {
                br[dst + q * ns] = ur[q];
                bi[dst + q * ns] = ui[q];
            }
        }
        double *t0 = *are, *t1 = *aim;
        *are = *bre; *aim = *bim;
        *bre = t0; *bim = t1;
        ns *= r;
    }
}

/* DCT-II (REDFT10) of x into y, via Makhoul. */
static void dct2(const orc_plan *p, const double *x, double *y, double *w0, double *w1, double *w2,
                 double *w3)
{
    const int n = p->n;
    double *ar = w0, *ai = w1, *br = w2, *bi = w3;
    for (int m = 0; 2 * m < n; m++) { ar[m] = x[2 * m]; ai[m] = 0.0; }
    for (int m = 0; 2 * m + 1 < n; m++) { ar[n - 1 - m] = x[2 * m + 1]; ai[n - 1 - m] = 0.0; }
    fft_stockham(p, &ar, &ai, &br, &bi, -1);
    for (int k = 0; k < n; k++) y[k] = 2.0 * (p->tre[k] * ar[k] - p->tim[k] * ai[k]);
}

/* DCT-III (REDFT01) of x into y: y = 2n * inverse(DCT-II). */
static void dct3(const orc_plan *p, const double *x, double *y, double *w0, double *w1, double *w2,
                 double *w3)
{
    const int n = p->n;
    double *ar = w0, *ai = w1, *br = w2, *bi = w3;
    for (int k = 0; k < n; k++) {
        double xr = x[k];
        double xi = (k == 0) ? 0.0 : -x[n - k];
        /* multiply by conj(tw) = exp(+i pi k / 2n) */
        double cr = p->tre[k], ci = -p->tim[k];
        ar[k] = xr * cr - xi * ci;
        ai[k] = xr * ci + xi * cr;
    }
    fft_stockham(p, &ar, &ai, &br, &bi, +1);
    for (int m = 0; 2 * m < n; m++) y[2 * m] = ar[m];
    for (int m = 0; 2 * m + 1 < n; m++) y[2 * m + 1] = ar[n - 1 - m];
}

static void r2r_line(const orc_plan *p, const double *in, double *out, int kind, double *scratch)
{
    const int n = p->n;
    double *w0 = scratch, *w1 = scratch + n, *w2 = scratch + 2 * n, *w3 = scratch + 3 * n;
    double *t = scratch + 4 * n, *u = scratch + 5 * n;
    switch (kind) {
    case ORC_REDFT10:
        dct2(p, in, u, w0, w1, w2, w3);
        memcpy(out, u, sizeof(double) * n);
        break;
    case ORC_REDFT01:
        dct3(p, in, u, w0, w1, w2, w3);
        memcpy(out, u, sizeof(double) * n);
        break;
    case ORC_RODFT10:
        for (int j = 0; j < n; j++) t[j] = (j & 1) ? -in[j] : in[j];
        dct2(p, t, u, w0, w1, w2, w3);
        for (int k = 0; k < n; k++) out[k] = u[n - 1 - k];
        break;
    case ORC_RODFT01:
        for (int j = 0; j < n; j++) t[j] = in[n - 1 - j];
        dct3(p, t, u, w0, w1, w2, w3);
        for (int k = 0; k < n; k++) out[k] = (k & 1) ? -u[k] : u[k];
        break;
    default:
        break;
    }
}

void orc_r2r_1d(const double *in, double *out, int n, int kind)
{
    if (n <= 0 || n > ORC_MAX_N) return;
    const orc_plan *p = plan_get(n);
    double *scratch = (double *)malloc(sizeof(double) * 6 * n);
    r2r_line(p, in, out, kind, scratch);
    free(scratch);
}

/* Transform every line along one axis.  Lines are gathered into a contiguous buffer. */
static void axis_pass(const double *in, double *out, int nx, int ny, int nz, int axis, int kind)
{
    int n, nl1, nl2;
    long s_n, s_1, s_2;
    if (axis == 2) { n = nz; nl1 = nx; nl2 = ny; s_n = 1; s_1 = (long)ny * nz; s_2 = nz; }
    else if (axis == 1) { n = ny; nl1 = nx; nl2 = nz; s_n = nz; s_1 = (long)ny * nz; s_2 = 1; }
    else { n = nx; nl1 = ny; nl2 = nz; s_n = (long)ny * nz; s_1 = nz; s_2 = 1; }
    const orc_plan *p = plan_get(n);
    const long nlines = (long)nl1 * nl2;
    int nth = orc_get_threads();
#pragma omp parallel num_threads(nth)
    {
        double *scratch = (double *)malloc(sizeof(double) * 8 * n);
        double *line = scratch + 6 * n, *res = scratch + 7 * n;
#pragma omp for schedule(static)
        for (long l = 0; l < nlines; l++) {
            long a = l / nl2, b = l % nl2;
            long base = a * s_1 + b * s_2;
            for (int q = 0; q < n; q++) line[q] = in[base + q * s_n];
            r2r_line(p, line, res, kind, scratch);
            for (int q = 0; q < n; q++) out[base + q * s_n] = res[q];
        }
        free(scratch);
    }
}

void orc_r2r_3d(const double *in, double *out, int nx, int ny, int nz, int kx, int ky, int kz)
{
    if (nx <= 0 || ny <= 0 || nz <= 0 || nx > ORC_MAX_N || ny > ORC_MAX_N || nz > ORC_MAX_N) return;
    plan_get(nx);
    plan_get(ny);
    plan_get(nz);
    axis_pass(in, out, nx, ny, nz, 2, kz);
    axis_pass(out, out, nx, ny, nz, 1, ky);
    axis_pass(out, out, nx, ny, nz, 0, kx);
}
