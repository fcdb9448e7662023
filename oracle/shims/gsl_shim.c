/*
 * gsl_shim.c - oracle-only stand-in for the GSL calls of the reference's
 * curved_boundaries.C.  Forwards gsl_integration_qags to the solver's
 * flow_quad_adaptive, so the oracle and the solver compute identical
 * curved-boundary geometry.  Test infrastructure: never linked into the
 * solver.
 */
#include <stdlib.h>
#include "gsl/gsl_integration.h"
#include "gsl/gsl_errno.h"
#include "quadrature.h"

gsl_integration_workspace *gsl_integration_workspace_alloc(size_t n)
{
  gsl_integration_workspace *w =
      (gsl_integration_workspace *)malloc(sizeof(gsl_integration_workspace));
  if (w) w->limit = n;
  return w;
}

void gsl_integration_workspace_free(gsl_integration_workspace *w) { free(w); }

int gsl_integration_qags(const gsl_function *f, double a, double b,
                         double epsabs, double epsrel, size_t limit,
                         gsl_integration_workspace *workspace, double *result,
                         double *abserr)
{
  (void)workspace;
  return flow_quad_adaptive(f->function, f->params, a, b, epsabs, epsrel,
                            (int)limit, result, abserr);
}

gsl_error_handler_t *gsl_set_error_handler_off(void) { return NULL; }
