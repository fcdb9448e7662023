/*
 * stages_gpu.C - the stage functions of the reference's solve() on the GPU.
 *
 * For a caller that keeps the reference's own solve() (its Newton loop, the
 * gradient, the limiter and the k=2 derivatives stay on the host) and moves
 * its face loops and its linear solve onto the device.  Linked with the
 * reference's sources, whose definitions of these four functions are made
 * weak, and with libflowgpu.so; the reference's signatures are kept:
 *   build_matrix              (include/init_memory.h:24)
 *                              -> flow_build_matrix
 *   build_interior_residuals  (include/residual.h:21)
 *                              -> flow_residual_stage(FLOW_STAGE_INTERIOR)
 *   build_boundary_residuals  (include/residual.h:23)
 *                              -> flow_residual_stage(FLOW_STAGE_BOUNDARY)
 *   linear_solve              (include/linear_algebra.h:23)
 *                              -> flow_linear_solve
 * Each call hands the device what the host side of solve() has written
 * since the last call (the current nQ; the gradient, limiter and k=2
 * derivatives; the right-hand side) and copies back what the reference's
 * function writes (LHS, dt and GRID::cfl; R; the ghost states and the
 * curved-wall normals; dQ), so every array the host reads next holds the
 * reference's values.  One device context per GRID, made on the first call;
 * for k=2 it takes no stencils, since the derivatives are the host's.
 * Where the library reports an error, the shim prints it and exits, as the
 * reference does at the same points (init_memory.C:257-268, cvbc.C:330-382).
 */
#include <stdio.h>
#include <stdlib.h>
#include "grid.h"
#include "sys_mem.h"
#include "params.h"
#include "gradient.h"
#include "init_memory.h"
#include "residual.h"
#include "linear_algebra.h"
#include "flow_gpu.h"
#include "grid_view.h"

static flow_ctx *s_ctx = NULL;
static const GRID *s_grid = NULL;
static ShimView s_view;

static flow_params stage_params(const PARAMS &p) {
  flow_params f = {p.nsteps, p.iter, p.jufreq, p.CFL, p.ramp, p.gamma, p.alpha, p.mach,
                   p.subits, p.unsteady, p.tacc, p.mintime, p.method, p.order, p.foits,
                   p.soits, p.toits, p.isrestart, p.limit, p.reorder, p.ic, p.p_or_cv,
                   p.start_post_pro, p.post_pro_freq};
  return f;
}

static void stage_fail(const char *what, int rc) {
  printf("FATAL ERROR: %s status %d (%s)\n", what, rc, flow_last_error());
  fflush(stdout);
  exit(1);
}

static long nq_of(const GRID *grid) { return (long)(grid->nn + grid->nn_ghost + 1) * 4; }
static long nnz_of(const GRID *grid, const SYS_MEM *smem) { return smem->ia[grid->nn + 1]; }

static void put(const char *name, const double *host, long n) {
  int rc = flow_set(s_ctx, name, host, n);
  if (rc) stage_fail(name, rc);
}

static void get(const char *name, double *host, long n) {
  int rc = flow_get(s_ctx, name, host, n);
  if (rc) stage_fail(name, rc);
}

static void ensure_context(GRID *grid, SYS_MEM *smem, const PARAMS &p) {
  if (s_ctx && s_grid == grid) return;
  // the LSQ edge weights the reference builds at its first gradient
  // (gradient.C:363-366); they depend on the mesh alone
  if (grid->edge_weight == NULL) Compute_Edge_Weights(grid);
  shim_view_fill(grid, smem, 0, &s_view);
  const flow_params fp = stage_params(p);
  int st = 0;
  if (s_ctx) flow_destroy(s_ctx);
  s_ctx = flow_create(&s_view.v, &fp, 0, &st);
  if (!s_ctx) stage_fail("flow_create", st);
  s_grid = grid;
}

void build_matrix(GRID *grid, PARAMS p, SYS_MEM *smem) {
  ensure_context(grid, smem, p);
  const flow_params fp = stage_params(p);
  const int nn = grid->nn;
  // the matrix and right-hand side the reference allocates on first use
  // (init_memory.C:176-186)
  if (smem->LHS == NULL) smem->LHS = (double *)malloc(sizeof(double) * 16 * nnz_of(grid, smem));
  if (smem->RHS == NULL) smem->RHS = (double *)malloc(sizeof(double) * 4 * (nn + 1));
  put("nQ", grid->nQ, nq_of(grid));
  put("xn_bedges", grid->xn_bedges, (long)(grid->nbedges + 1) * 3);
  int rc = flow_build_matrix(s_ctx, &fp, grid->citer);
  if (rc) stage_fail("flow_build_matrix", rc);
  get("LHS", smem->LHS, 16 * nnz_of(grid, smem));
  get("dt", grid->dt, nn + 1);
  get("cfl", &grid->cfl, 1);
}

void build_interior_residuals(GRID *grid, SYS_MEM *smem, PARAMS p, int jupdate, int ts) {
  ensure_context(grid, smem, p);
  const flow_params fp = stage_params(p);
  const int nn = grid->nn;
  // the residual the reference allocates on first use (residual.C:75-89)
  if (grid->R == NULL) grid->R = (double *)calloc((nn + 1) * 4, sizeof(double));
  // the reconstruction the host side of solve() formed for this step
  put("nQ", grid->nQ, nq_of(grid));
  if (grid->grad) put("grad", grid->grad, (long)(nn + 1) * 8);
  if (grid->phi) put("phi", grid->phi, (long)(nn + 1) * 8);
  if (p.order == 3 && grid->hess) put("hess", grid->hess, (long)(nn + 1) * 36);
  if (p.order == 3 && grid->point_value) put("point_value", grid->point_value, (long)(nn + 1) * 4);
  int rc = flow_residual_stage(s_ctx, &fp, jupdate, ts, FLOW_STAGE_INTERIOR);
  if (rc) stage_fail("build_interior_residuals", rc);
  get("R", grid->R, (long)(nn + 1) * 4);
  if (jupdate) get("LHS", smem->LHS, 16 * nnz_of(grid, smem));
}

void build_boundary_residuals(GRID *grid, SYS_MEM *smem, PARAMS p, int jupdate) {
  ensure_context(grid, smem, p);
  const flow_params fp = stage_params(p);
  const int nn = grid->nn;
  int rc = flow_residual_stage(s_ctx, &fp, jupdate, grid->citer, FLOW_STAGE_BOUNDARY);
  if (rc) stage_fail("build_boundary_residuals", rc);
  get("R", grid->R, (long)(nn + 1) * 4);
  get("nQ", grid->nQ, nq_of(grid));  // the ghost states Set_Boundary_Values wrote
  get("xn_bedges", grid->xn_bedges, (long)(grid->nbedges + 1) * 3);
  if (jupdate) get("LHS", smem->LHS, 16 * nnz_of(grid, smem));
}

double linear_solve(GRID *grid, SYS_MEM *smem, PARAMS p) {
  ensure_context(grid, smem, p);
  const flow_params fp = stage_params(p);
  // solve() formed RHS = -R (and cleared dQ) on the host
  put("RHS", smem->RHS, (long)(grid->nn + 1) * 4);
  double rms = 0.;
  int rc = flow_linear_solve(s_ctx, &fp, &rms);
  if (rc) stage_fail("linear_solve", rc);
  get("dQ", grid->dQ, (long)(grid->nn + 1) * 4);
  return rms;
}
