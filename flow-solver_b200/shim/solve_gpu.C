/*
 * solve_gpu.C - the shim that drops libflowgpu.so into the reference solver.
 *
 * Compiled with the reference's own sources in place of solve.C's solve()
 * (the rest of solve.C is debug / manufactured-solution code), with the
 * reference's include/ and this repository's include/ on the include path,
 * and linked against libflowgpu.so.  It keeps the reference's signatures
 * (include/solve.h:21, include/grid_io.h:22-36), so main.C relinks
 * unchanged:
 *   solve                    -> flow_create (first call), flow_solve, flow_get
 *   Compute_Body_Forces      -> flow_body_forces
 *   write_surface_cp         -> flow_write_surface_cp
 * The Tecplot and mesh writers stay the reference's own: main.C calls
 * write_tecplot_solutionC before the first solve() (main.C:704), when no
 * device context exists yet, and solve() copies the state back into the
 * GRID after every step, so the host writers see the current solution.
 * k=1 and k=2 are wired: the device context takes the LSQ edge weights
 * (k=1, or k=2 with second-order start-up steps) and, for k=2, the grown
 * two-ring stencils and their SVD factors, made on the host by the
 * reference's own functions before the context is created.  Where the
 * library returns an error bit, the shim prints the message and exits as
 * the reference does at the same points (cvbc.C:330-382,
 * init_memory.C:257-268, limiter.C:965-977).
 */
#include <stdio.h>
#include <stdlib.h>
#include "grid.h"
#include "sys_mem.h"
#include "params.h"
#include "gradient.h"
#include "maps.h"
#include "compute_derivatives.h"
#include "flow_gpu.h"
#include "grid_view.h"

static flow_ctx *g_ctx = NULL;
static const GRID *g_grid = NULL;
static ShimView g_view;

static flow_params to_flow(const PARAMS &p) {
  flow_params f = {p.nsteps, p.iter, p.jufreq, p.CFL, p.ramp, p.gamma, p.alpha, p.mach,
                   p.subits, p.unsteady, p.tacc, p.mintime, p.method, p.order, p.foits,
                   p.soits, p.toits, p.isrestart, p.limit, p.reorder, p.ic, p.p_or_cv,
                   p.start_post_pro, p.post_pro_freq};
  return f;
}

static int stencil_rows(const GRID *grid, int i) {
  return grid->gnnsn[grid->gnnsn1[i + 1]] - grid->gnnsn[grid->gnnsn1[i] + 1];
}

static void add_layer(GRID *grid, int i) {
  Add_Layer_to_GNSN(grid->nn, grid->num_elem, grid->c2n, grid->esn, grid->nnsn, grid->edges,
                    &(grid->gnsn), &(grid->gnnsn), grid->gnnsn1, grid->node_fill_level, i);
}

/* The k=2 stencils the reference's solve() builds on its first high-order
 * step (solve.C:57-114): one layer of neighbours for every node, a second
 * for the nodes of order 3, then up to three more for any k=2 node whose
 * stencil still has fewer than 6 rows (a node that needs more ends the run,
 * as there).  All through the reference's own Add_Layer_to_GNSN.  The
 * stencils depend on the mesh alone, so building them at the run's first
 * step gives the arrays the reference builds later. */
static void grow_stencils(GRID *grid) {
  for (int i = 1; i <= grid->nn; i++) add_layer(grid, i);
  for (int i = 1; i <= grid->nn; i++)
    if (grid->node_order[i] > 2) add_layer(grid, i);
  for (int i = 1; i <= grid->nn; i++) {
    if (grid->node_order[i] < 3) continue;
    int extra = 0;
    while (stencil_rows(grid, i) < 6) {
      if (extra == 3) {
        printf("FATAL ERROR: Node %d has attempted to add too many layers of neighbors. "
               "Halting...\n", i);
        fflush(stdout);
        exit(0);
      }
      add_layer(grid, i);
      extra++;
    }
  }
}

/* A device context for `grid`: the view, plus for k=2 the stencils and the
 * pseudo-inverse factors.  The factors come from the reference's own
 * Compute_Derivatives (compute_derivatives.C:274-1072 factors every node on
 * its first call), run once here on the host from the current state. */
static void make_context(GRID *grid, SYS_MEM *smem, const PARAMS &p) {
  const flow_params fp = to_flow(p);
  const long nq = (long)(grid->nn + grid->nn_ghost + 1) * 4;
  // the LSQ edge weights the reference builds on its first gradient
  // (gradient.C:363-366): k=1, and the second-order start-up steps of k=2
  if ((p.order == 1 || (p.order == 3 && p.soits > 0)) && grid->edge_weight == NULL)
    Compute_Edge_Weights(grid);
  if (p.order == 3) {
    if (grid->SVD_U == NULL) {
      for (long k = 0; k < nq; k++) grid->nQ[k] = grid->Q[k];
      grow_stencils(grid);
      Compute_Derivatives(grid, p, 3);
    }
  }
  shim_view_fill(grid, smem, p.order == 3, &g_view);
  int st = 0;
  if (g_ctx) flow_destroy(g_ctx);  // a new GRID: the old device mirror goes
  g_ctx = flow_create(&g_view.v, &fp, 0, &st);
  if (!g_ctx) { printf("flow_create failed: %s\n", flow_last_error()); exit(1); }
  g_grid = grid;
  if (flow_set_state(g_ctx, grid->Q)) {
    printf("FATAL ERROR: flow_set_state failed (%s)\n", flow_last_error());
    exit(1);
  }
}

double solve(GRID *grid, SYS_MEM *smem, PARAMS p, int ts) {
  flow_params fp = to_flow(p);
  long nq = (long)(grid->nn + grid->nn_ghost + 1) * 4;
  if (g_ctx == NULL || g_grid != grid) {
    // the arrays the reference's solve() allocates on first use
    // (solve.C:239-286); the GRID destructor frees them
    if (grid->nQ == NULL) grid->nQ = (double *)calloc(nq, sizeof(double));
    if (grid->pQ == NULL) grid->pQ = (double *)calloc(nq, sizeof(double));
    if (grid->R == NULL) grid->R = (double *)calloc((grid->nn + 1) * 4, sizeof(double));
    if (grid->dQ == NULL) grid->dQ = (double *)calloc((grid->nn + 1) * 4, sizeof(double));
    if (grid->hess == NULL) grid->hess = (double *)calloc((grid->nn + 1) * 36, sizeof(double));
    make_context(grid, smem, p);
  }
  double dq = 0.;
  int rc = flow_solve(g_ctx, &fp, ts, &dq, NULL);
  if (rc) { printf("FATAL ERROR: flow_solve status %d (%s)\n", rc, flow_last_error()); exit(1); }
  // the state back into the GRID for the reference's writers, with GRID::cfl
  // (the ramp's CFL of this step, which write_mesh prints); a failed read
  // would hand them the previous step's arrays, so it ends the run
  rc = flow_get(g_ctx, "Q", grid->Q, nq);
  rc |= flow_get(g_ctx, "nQ", grid->nQ, nq);
  rc |= flow_get(g_ctx, "pQ", grid->pQ, nq);
  rc |= flow_get(g_ctx, "R", grid->R, (long)(grid->nn + 1) * 4);
  rc |= flow_get(g_ctx, "dQ", grid->dQ, (long)(grid->nn + 1) * 4);
  rc |= flow_get(g_ctx, "xn_bedges", grid->xn_bedges, (long)(grid->nbedges + 1) * 3);
  rc |= flow_get(g_ctx, "cfl", &grid->cfl, 1);
  if (grid->phi) rc |= flow_get(g_ctx, "phi", grid->phi, (long)(grid->nn + 1) * 8);
  if (rc) {
    printf("FATAL ERROR: reading the state back failed (status %d: %s)\n", rc, flow_last_error());
    exit(1);
  }
  return dq;
}

static int *flat_segments(const GRID *grid) {
  int n = 0, k = 0;
  for (int b = 1; b <= grid->nb; b++) n += grid->nbs[b];
  int *seg = (int *)malloc(sizeof(int) * 2 * (n > 0 ? n : 1));
  for (int b = 1; b <= grid->nb; b++)
    for (int s = 1; s <= grid->nbs[b]; s++) {
      seg[k++] = grid->bs[b][s][0];
      seg[k++] = grid->bs[b][s][1];
    }
  return seg;
}

void write_surface_cp(GRID *grid, PARAMS p) {
  flow_params fp = to_flow(p);
  int *seg = flat_segments(grid);
  if (flow_write_surface_cp(g_ctx, &fp, ".", grid->nb, grid->bbc, grid->nbs, seg, grid->x)) {
    printf("%s\n", flow_last_error()); exit(0);
  }
  free(seg);
}

void Compute_Body_Forces(GRID *grid, PARAMS p, double *Forces) {
  flow_params fp = to_flow(p);
  (void)grid;
  if (flow_body_forces(g_ctx, &fp, Forces)) {
    printf("%s\n", flow_last_error()); exit(1);
  }
}
