/*
 * quadrature.h - adaptive 1-D quadrature used for curved-boundary arc lengths.
 *
 * The reference integrates the NACA 0012 arc-length integrand with GSL's
 * gsl_integration_qags (curved_boundaries.C:238-256, 555-572, 1101-1127).
 * GSL is not part of the reference tree, so this file provides the
 * quadrature used both by the solver's host preprocessing and by the
 * oracle's stand-in for that GSL call: the geometry fed to the residual is
 * then identical on both sides.
 *
 * Method: for 0 <= a < b the substitution x = t^2 removes the 1/sqrt(x)
 * endpoint singularity of the arc-length integrand; the smooth integrand is
 * integrated by globally adaptive bisection, each panel estimated with the
 * 10- and 20-point Gauss-Legendre rules (nodes computed at first use by
 * Newton iteration on the Legendre polynomials), error = |G20 - G10|.
 */
#ifndef FLOW_QUADRATURE_H
#define FLOW_QUADRATURE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef double (*flow_quad_fn)(double x, void *params);

/* Returns 0 on convergence to max(epsabs, epsrel*|I|), 1 when `limit`
 * panels were used up (the best estimate is still returned). */
int flow_quad_adaptive(flow_quad_fn f, void *params, double a, double b,
                       double epsabs, double epsrel, int limit,
                       double *result, double *abserr);

#ifdef __cplusplus
}
#endif

#endif
