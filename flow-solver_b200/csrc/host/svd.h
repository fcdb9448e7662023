/*
 * svd.h - small dense SVD for the k=2 least-squares stencils.
 *
 * The reference factors each node's weighted m x 5 reconstruction matrix with
 * LAPACK dgesvd_ (JOBU='A', JOBVT='A'; compute_derivatives.C:845,928) and
 * keeps U (m x m), S (5) and VT (5 x 5) for the per-iteration apply
 * (compute_derivatives.C:1478-1521).  LAPACK is not part of the reference
 * tree; this one-sided (Hestenes) Jacobi SVD produces factors with the same
 * LAPACK storage conventions.  It is used by the host preprocessing and by
 * the oracle's stand-in for dgesvd_, so both sides see identical factors.
 */
#ifndef FLOW_SVD_H
#define FLOW_SVD_H

#ifdef __cplusplus
extern "C" {
#endif

/* A: m x n column-major (lda = m), m >= n >= 1, m <= 64, n <= 16.
 * s: min(m,n) singular values, descending.
 * U: column-major with leading dimension m; the first n columns are the left
 *    singular vectors; with full_u != 0 the remaining m-n columns are an
 *    orthonormal completion (U is then m x m, as dgesvd JOBU='A' returns).
 * VT: n x n column-major, rows = right singular vectors.
 * Returns 0 on success. */
int flow_svd_jacobi(int m, int n, const double *A, double *s, double *U,
                    double *VT, int full_u);

#ifdef __cplusplus
}
#endif

#endif
