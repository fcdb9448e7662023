/*
 * lapack_shim.c - oracle-only stand-in for LAPACK dgesvd_ as declared by the
 * reference (include/liblapack_interface.h:14-21) and called with
 * JOBU='A', JOBVT='A' (compute_derivatives.C:845,928).  Forwards to the
 * solver's one-sided Jacobi SVD with full U, so the oracle and the solver
 * use identical pseudo-inverse factors.  Test infrastructure only.
 */
#include "svd.h"

void dgesvd_(char *jobu, char *jobvt, int *m, int *n, double *A, int *lda,
             double *S, double *U, int *ldu, double *VT, int *ldvt,
             double *work, int *lwork, int *info)
{
  (void)jobu; (void)jobvt; (void)work; (void)lwork;
  int mm = *m, nn = *n;
  if (*lda != mm || *ldu != mm || *ldvt != nn) { *info = -6; return; }
  *info = flow_svd_jacobi(mm, nn, A, S, U, VT, 1);
}
