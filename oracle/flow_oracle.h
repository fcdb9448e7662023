/*
 * flow_oracle.h - CPU restatement of the reference's nonlinear iteration.
 *
 * TEST INFRASTRUCTURE (the oracle).  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg use it, as the checker.  It is plain C over the
 * reference's own array layout (1-based, array-of-structs, see
 * include/grid.h / include/sys_mem.h of the reference) and restates, in the
 * reference's arithmetic order, the functions of the hot path:
 *   solve.C:44-933, init_memory.C:159-310, cv_calc.C:790-965,
 *   gradient.C:382-403, compute_derivatives.C:1438-1534, limiter.C:511-983,
 *   reconstruct.C:38-446,467-,1109-1399,1420-,1708-1890, flux.C:37-68,299-541,
 *   residual.C:40-342,359-1230, jacobian.C:45-185,681-962, cvbc.C:37-481,
 *   curved_boundaries.C:701-877, linear_algebra.C:122-401,571-638,
 *   grid_io.C:1390-1697.
 * It is checked bit-for-bit against the compiled reference (oracle/_ref).
 */
#ifndef FLOW_ORACLE_H
#define FLOW_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  /* PARAMS fields used on the path (include/params.h:19-76) */
  int iter, jufreq, ramp, subits, unsteady, tacc, method, order;
  int foits, soits, toits, limit;
  double CFL, gamma, alpha, mach, mintime;
  /* precision form only (no reference counterpart): 1 = interior face
   * Jacobians by the approximate Roe form instead of forward differences */
  int jac_approx;
} orc_params;

typedef struct {
  int nn, nn_ghost, nedges, nsubedges, nbedges, nb;
  /* topology (1-based, reference layout) */
  const int *edges;      /* (nedges+1)*2 */
  const int *subedges;   /* (nsubedges+1)*2: edge, element */
  const int *bedges;     /* (nbedges+1)*5: node, ghost, element, boundary, segment */
  const int *bedge_seg;  /* (nbedges+1)*2: bs[b][s][0..1] of the bedge's segment */
  const int *bbc;        /* nb+1 */
  const int *node_order; /* nn+nn_ghost+1 */
  const int *ia, *iau, *ja;
  /* geometry */
  const double *x;           /* (nn+nn_ghost+1)*2 */
  const double *cv_area;     /* nn+1 */
  const double *el_cent;
  const double *xn_subedges, *xm_subedges, *xg_subedges;
  double *xn_bedges;         /* (nbedges+1)*3, mutated by the k=2 boundary pass */
  const double *xg_bedges, *xgn_bedges;
  const double *edge_weight; /* (nedges+1)*4 */
  const double *moments;     /* (nn+1)*9 */
  /* k=2 stencils and SVD factors (compute_derivatives.C:845-940) */
  const int *gnsn, *gnnsn, *gnnsn1;
  const long *svd_off;       /* nn+1: offset of node i's U (m*m doubles) in svd_U */
  const int *svd_m;          /* nn+1 */
  const double *svd_U;       /* concatenated column-major m x m */
  const double *svd_VT;      /* (nn+1)*25 */
  const double *svd_S;       /* (nn+1)*5 */
  /* state */
  double *Q, *nQ, *pQ, *dQ, *R, *grad, *hess, *phi, *point_value, *dt, *ev_con;
  double *LHS, *RHS;
  double cfl;
  int citer;
} orc_grid;

/* Stages (return 0, or a nonzero code where the reference would exit()). */
int orc_build_matrix(orc_grid *g, const orc_params *p);
void orc_gradient_lsq(orc_grid *g);
void orc_derivatives_k2(orc_grid *g);
int orc_limiter_venkat(orc_grid *g, const orc_params *p);
void orc_interior_residuals(orc_grid *g, const orc_params *p, int jupdate, int ts);
int orc_set_boundary_values(orc_grid *g, const orc_params *p);
int orc_boundary_residuals(orc_grid *g, const orc_params *p, int jupdate);
double orc_linear_solve(orc_grid *g, const orc_params *p);
void orc_body_forces(orc_grid *g, const orc_params *p, double *forces);
/* One pseudo-time step (solve.C:44-933 for steady implicit runs,
 * order 1 or 3, limiter 2); the k=2 stencils must already be grown.
 * Returns ||dQ||_2 in *dq, 0 on success. */
int orc_solve(orc_grid *g, const orc_params *p, int ts, double *dq);

/* ---- precision form: FP32 Jacobian blocks, multicolour block GS ----
 * Not in the reference: the defect-correction preconditioner of the
 * precision form.  The residual, geometry and update stay FP64; the linear
 * solve rounds the off-diagonal blocks and the LU factors of each diagonal
 * block (factored in FP64 with the reference's lu, linear_algebra.C:571-590)
 * to FP32, keeps reciprocal pivots, and runs p->subits sweeps of block
 * Gauss-Seidel in colour order (forward: colours ascending, backward:
 * descending) with FP32 arithmetic in a fixed fused-multiply-add order.
 * Rows of one colour share no block, so their order inside a colour does not
 * matter and the result is unique. */
/* Greedy distance-1 colouring of the block pattern in row order 1..nn:
 * each row takes the smallest colour no earlier neighbour holds.
 * color[1..nn] receives the colours; returns the number of colours. */
int orc_greedy_colors(const orc_grid *g, int *color);
void orc_linear_solve_mixed(orc_grid *g, const orc_params *p, const int *color, int ncolors);
/* color == NULL: FP32 blocks with the sweeps in the reference's row order.
 * orc_solve_mixed: orc_solve with orc_linear_solve_mixed in place of
 * orc_linear_solve (color == NULL again selects the reference order). */
int orc_solve_mixed(orc_grid *g, const orc_params *p, int ts, double *dq, const int *color,
                    int ncolors);

/* FP32 sweeps visiting rows in `order` (a permutation of 1..nn) forward and
 * in reverse backward (the chunked order of the precision form is one such
 * permutation); orc_solve_mixed_order is the step around it. */
void orc_linear_solve_mixed_order(orc_grid *g, const orc_params *p, const int *order);
int orc_solve_mixed_order(orc_grid *g, const orc_params *p, int ts, double *dq,
                          const int *order);

/* Building blocks, exposed for unit checks. */
int orc_roe_flux(double nx, double ny, double len, double gamma, const double *ql,
                 const double *qr, double *flux);
void orc_curved_normal(int bc, const double *x, double *nx, double *ny);

#ifdef __cplusplus
}
#endif

#endif
