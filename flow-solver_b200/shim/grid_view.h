/*
 * grid_view.h - flow_grid_view from the reference's GRID and SYS_MEM, for the
 * shims that link libflowgpu.so into the reference solver (solve_gpu.C,
 * stages_gpu.C).  Header-only: each shim is one translation unit.
 *
 * The view points into the GRID's own arrays (include/grid.h:223-307,
 * include/sys_mem.h:43-49); only what the GRID does not hold in the view's
 * layout is packed into arrays the ShimView owns:
 *   seg      GRID::bs[b][s][0..1] of every boundary edge, in bedge order;
 *   svd_*    the k=2 pseudo-inverse factors, which the reference keeps as
 *            one malloc per node (GRID::SVD_U[i] m x m, SVD_V[i] 5 x 5,
 *            SVD_S[i] 5, SVD_size[i*3] = m; compute_derivatives.C:497-1072),
 *            packed node after node with offsets.
 */
#ifndef FLOW_SHIM_GRID_VIEW_H
#define FLOW_SHIM_GRID_VIEW_H

#include <stdlib.h>
#include <string.h>

#include "grid.h"
#include "sys_mem.h"
#include "flow_gpu.h"

struct ShimView {
  flow_grid_view v;
  int *seg;
  int *svd_m;
  long *svd_off;
  double *svd_U, *svd_VT, *svd_S;
};

static void shim_view_free(ShimView *sv) {
  free(sv->seg);
  free(sv->svd_m);
  free(sv->svd_off);
  free(sv->svd_U);
  free(sv->svd_VT);
  free(sv->svd_S);
  memset(sv, 0, sizeof(*sv));
}

/* The view of `grid`; with_k2 != 0 also packs the grown stencils and the SVD
 * factors (the GRID must hold them: GRID::gnsn after the k=2 growth and
 * GRID::SVD_U etc. after Compute_Derivatives(grid, p, 3)). */
static void shim_view_fill(GRID *grid, SYS_MEM *smem, int with_k2, ShimView *sv) {
  shim_view_free(sv);
  flow_grid_view &v = sv->v;
  const int nn = grid->nn;
  sv->seg = (int *)malloc(sizeof(int) * 2 * (grid->nbedges + 1));
  sv->seg[0] = sv->seg[1] = 0;
  for (int i = 1; i <= grid->nbedges; i++) {
    const int b = grid->bedges[i * 5 + 3], s = grid->bedges[i * 5 + 4];
    sv->seg[2 * i] = grid->bs[b][s][0];
    sv->seg[2 * i + 1] = grid->bs[b][s][1];
  }
  v.nn = nn;
  v.nn_ghost = grid->nn_ghost;
  v.nedges = grid->nedges;
  v.nsubedges = grid->nsubedges;
  v.nbedges = grid->nbedges;
  v.nb = grid->nb;
  v.nelem = grid->num_elem[Tri] + grid->num_elem[Quad];
  v.edges = grid->edges;
  v.subedges = grid->subedges;
  v.bedges = grid->bedges;
  v.bedge_seg = sv->seg;
  v.bbc = grid->bbc;
  v.node_order = grid->node_order;
  v.ia = smem->ia;
  v.iau = smem->iau;
  v.ja = smem->ja;
  v.x = grid->x;
  v.cv_area = grid->cv_area;
  v.el_cent = grid->el_cent;
  v.xn_subedges = grid->xn_subedges;
  v.xm_subedges = grid->xm_subedges;
  v.xg_subedges = grid->xg_subedges;
  v.xn_bedges = grid->xn_bedges;
  v.xg_bedges = grid->xg_bedges;
  v.xgn_bedges = grid->xgn_bedges;
  v.edge_weight = grid->edge_weight;
  v.moments = grid->Moments;
  if (!with_k2) return;
  v.gnsn = grid->gnsn;
  v.gnnsn = grid->gnnsn;
  v.gnnsn1 = grid->gnnsn1;
  sv->svd_m = (int *)calloc(nn + 1, sizeof(int));
  sv->svd_off = (long *)calloc(nn + 1, sizeof(long));
  sv->svd_VT = (double *)calloc((size_t)(nn + 1) * 25, sizeof(double));
  sv->svd_S = (double *)calloc((size_t)(nn + 1) * 5, sizeof(double));
  long total = 0;
  for (int i = 1; i <= nn; i++) {
    if (!grid->SVD_U[i]) continue;
    const int m = (int)grid->SVD_size[i * 3 + 0];
    sv->svd_m[i] = m;
    sv->svd_off[i] = total;
    total += (long)m * m;
  }
  sv->svd_U = (double *)malloc(sizeof(double) * (total > 0 ? total : 1));
  for (int i = 1; i <= nn; i++) {
    if (!grid->SVD_U[i]) continue;
    const int m = sv->svd_m[i];
    memcpy(sv->svd_U + sv->svd_off[i], grid->SVD_U[i], sizeof(double) * m * m);
    memcpy(sv->svd_VT + (size_t)i * 25, grid->SVD_V[i], sizeof(double) * 25);
    memcpy(sv->svd_S + (size_t)i * 5, grid->SVD_S[i], sizeof(double) * 5);
  }
  v.svd_m = sv->svd_m;
  v.svd_off = sv->svd_off;
  v.svd_U = sv->svd_U;
  v.svd_VT = sv->svd_VT;
  v.svd_S = sv->svd_S;
}

#endif
