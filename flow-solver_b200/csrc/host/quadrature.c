/*
 * quadrature.c - adaptive Gauss-Legendre quadrature (see quadrature.h).
 *
 * Stands in for gsl_integration_qags as called by the reference at
 * curved_boundaries.C:240,256,557,572,1123 (NACA arc length, abs/rel
 * tolerance 1e-8, 1000 subintervals).  The algorithm is the textbook
 * globally-adaptive bisection scheme; it is written here from that
 * description, not from GSL.
 */
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include "quadrature.h"

#define GL_LO 10
#define GL_HI 20

/* Gauss-Legendre nodes/weights on [-1,1] by Newton iteration on P_n. */
static void gauss_legendre(int n, double *x, double *w)
{
    const double pi = 3.14159265358979323846;
    int m = (n + 1) / 2;
    for (int i = 0; i < m; i++) {
        double z = cos(pi * (i + 0.75) / (n + 0.5));
        double pp = 0.0;
        for (int it = 0; it < 100; it++) {
            double p1 = 1.0, p2 = 0.0;
            for (int j = 1; j <= n; j++) {
                double p3 = p2;
                p2 = p1;
                p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
            }
            pp = n * (z * p1 - p2) / (z * z - 1.0);
            double z1 = z;
            z = z1 - p1 / pp;
            if (fabs(z - z1) <= 1e-15) break;
        }
        x[i] = -z;
        x[n - 1 - i] = z;
        w[i] = 2.0 / ((1.0 - z * z) * pp * pp);
        w[n - 1 - i] = w[i];
    }
}

/* The two rules are the same on every call: computed once per process
 * (pthread_once: preprocessing may run on several threads at a time). */
static double g_xl[GL_LO], g_wl[GL_LO], g_xh[GL_HI], g_wh[GL_HI];
static pthread_once_t g_rules_once = PTHREAD_ONCE_INIT;

static void init_rules(void)
{
    gauss_legendre(GL_LO, g_xl, g_wl);
    gauss_legendre(GL_HI, g_xh, g_wh);
}

typedef struct {
    flow_quad_fn f;
    void *params;
    int substitute; /* integrate g(t) = f(t^2) 2t */
} integrand_t;

static double eval(const integrand_t *g, double t)
{
    if (g->substitute) return g->f(t * t, g->params) * 2.0 * t;
    return g->f(t, g->params);
}

static void panel(const integrand_t *g, double a, double b,
                  const double *xl, const double *wl,
                  const double *xh, const double *wh,
                  double *val, double *err)
{
    double c = 0.5 * (a + b), h = 0.5 * (b - a);
    double lo = 0.0, hi = 0.0;
    for (int i = 0; i < GL_LO; i++) lo += wl[i] * eval(g, c + h * xl[i]);
    for (int i = 0; i < GL_HI; i++) hi += wh[i] * eval(g, c + h * xh[i]);
    *val = hi * h;
    *err = fabs(hi - lo) * h;
}

int flow_quad_adaptive(flow_quad_fn f, void *params, double a, double b,
                       double epsabs, double epsrel, int limit,
                       double *result, double *abserr)
{
    pthread_once(&g_rules_once, init_rules);
    const double *xl = g_xl, *wl = g_wl, *xh = g_xh, *wh = g_wh;

    integrand_t g;
    g.f = f;
    g.params = params;
    g.substitute = 0;
    double sign = 1.0;
    if (b < a) { double t = a; a = b; b = t; sign = -1.0; }
    if (a >= 0.0) { g.substitute = 1; a = sqrt(a); b = sqrt(b); }

    if (limit < 1) limit = 1;
    double *pa = (double *)malloc(sizeof(double) * 4 * (size_t)limit);
    if (!pa) { *result = 0.0; *abserr = INFINITY; return 2; }
    double *pb = pa + limit, *pv = pb + limit, *pe = pv + limit;
    int np = 1;
    pa[0] = a; pb[0] = b;
    panel(&g, a, b, xl, wl, xh, wh, &pv[0], &pe[0]);

    int status = 1;
    for (;;) {
        double tot = 0.0, etot = 0.0;
        int worst = 0;
        for (int i = 0; i < np; i++) {
            tot += pv[i];
            etot += pe[i];
            if (pe[i] > pe[worst]) worst = i;
        }
        double tol = epsabs > epsrel * fabs(tot) ? epsabs : epsrel * fabs(tot);
        *result = sign * tot;
        *abserr = etot;
        if (etot <= tol) { status = 0; break; }
        if (np >= limit) break;
        double m = 0.5 * (pa[worst] + pb[worst]);
        pa[np] = m; pb[np] = pb[worst];
        pb[worst] = m;
        panel(&g, pa[worst], pb[worst], xl, wl, xh, wh, &pv[worst], &pe[worst]);
        panel(&g, pa[np], pb[np], xl, wl, xh, wh, &pv[np], &pe[np]);
        np++;
    }
    free(pa);
    return status;
}
