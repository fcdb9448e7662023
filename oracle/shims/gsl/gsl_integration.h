/*
 * Stand-in declarations for the two GSL integration entry points the
 * reference calls (curved_boundaries.C:16,101-113,238-292,555-626,1101-1127).
 * Only the names and argument lists match GSL; the implementation
 * (gsl_shim.c) forwards to the solver's own adaptive quadrature.
 * Oracle build only: nothing in the solver includes this header.
 */
#ifndef ORACLE_SHIM_GSL_INTEGRATION_H
#define ORACLE_SHIM_GSL_INTEGRATION_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  double (*function)(double x, void *params);
  void *params;
} gsl_function;

typedef struct {
  size_t limit;
} gsl_integration_workspace;

gsl_integration_workspace *gsl_integration_workspace_alloc(size_t n);
void gsl_integration_workspace_free(gsl_integration_workspace *w);
int gsl_integration_qags(const gsl_function *f, double a, double b,
                         double epsabs, double epsrel, size_t limit,
                         gsl_integration_workspace *workspace,
                         double *result, double *abserr);

#ifdef __cplusplus
}
#endif
#endif
