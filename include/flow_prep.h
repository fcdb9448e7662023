/*
 * flow_prep.h - host preprocessing: mesh -> the grid arrays the nonlinear
 * iteration consumes (libflowgpu.so).
 *
 * Replaces the set-up half of the reference driver (main.C:107-666):
 * read_mesh (mesh_io.C:31-297), Cuthill_McKee (reorder.C:58-303), the maps
 * of maps.C (Cells/Nodes/Edges_Surrounding_Node, generic 2-ring stencils),
 * Find_Element_Centroids, Build_Edge_Data, Build_Boundary_Edge_Data,
 * Fix_Subedge_Data, Generate_Gaussian_Data_For_Edge (geometry.C),
 * cv_calc_area_Green and cv_calc_Moments (cv_calc.C), Build_CRS
 * (init_memory.C:36-138), Compute_Edge_Weights (gradient.C:923-1121), the
 * k=2 stencil growth of solve.C:57-114 and the SVD factorisation of
 * compute_derivatives.C:845-940, and the free-stream initial condition
 * ic_0 (ic.C:808-836).  Same algorithms and operation order as the
 * reference, linear-time where the reference is quadratic, so the arrays
 * match the reference's own set-up.
 */
#ifndef FLOW_PREP_H
#define FLOW_PREP_H

#include "flow_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct flow_mesh flow_mesh;

/* Read a mesh in the reference's format (mesh_io.C:31-277) with one boundary
 * condition per boundary (the contents of bc.dat), and preprocess it for a
 * run of reconstruction order `order` (1 or 3).  reorder != 0 applies the
 * Cuthill-McKee renumbering.  Returns NULL and sets *status on failure. */
flow_mesh *flow_prep_read(const char *mesh_path, const int *bbc, int nb, int reorder, int order,
                          int *status);

/* Same from in-memory arrays: x (nn x 2), tri (ntri x 3, 1-based),
 * quad (nquad x 4, 1-based), boundaries given as nb segment lists with
 * nbs[b] segments each, seg = all segments' (n0, n1) pairs in boundary order. */
flow_mesh *flow_prep_build(int nn, const double *x, int ntri, const int *tri, int nquad,
                           const int *quad, int nb, const int *nbs, const int *seg,
                           const int *bbc, int reorder, int order, int *status);

/* Fill a view of the preprocessed arrays (valid while the mesh lives). */
int flow_prep_view(const flow_mesh *m, flow_grid_view *view);

/* Free-stream initial state ic_0 (ic.C:808-836), ghosts copied from their
 * real node (ic.C:84-96): Q has (nn+nn_ghost+1)*4 entries. */
int flow_prep_initial_state(const flow_mesh *m, const flow_params *p, double *Q);

/* The restart block of the mesh file, if it had one (as the reference's
 * write_mesh appends it, mesh_io.C:380-390, and read_mesh reads it back with
 * isrestart = 1, mesh_io.C:217-262): Q receives the conserved variables of
 * every node ((nn+nn_ghost+1)*4 doubles; each ghost a copy of its real node,
 * main.C:602-622), *citer the last step run and *cfl its CFL (either may be
 * NULL); the solve resumes at step *citer + 1.  Read a restart file without
 * reordering, as the reference does.  FLOW_ERR_NOT_FOUND if the file had no
 * restart block. */
int flow_prep_restart_state(const flow_mesh *m, double *Q, long nQ, int *citer, double *cfl);

/* nn_map of the renumbering (old 1-based id -> new id), nn+1 ints. */
const int *flow_prep_node_map(const flow_mesh *m);

/* Element connectivity after the renumbering (GRID::c2n[Tri] and
 * GRID::c2n[Quad], reorder.C:58-303): 1-based rows with row 0 unused,
 * (ntri+1)*3 and (nquad+1)*4 ints, valid while the mesh lives. */
int flow_prep_elements(const flow_mesh *m, int *ntri, const int **tri, int *nquad,
                       const int **quad);

/* Boundaries after the renumbering: nb, bbc and nbs (nb+1 ints each, index
 * 0 unused; GRID::nb, GRID::bbc, GRID::nbs) and the segments' (n0, n1) node
 * pairs GRID::bs[b][s][0..1] of every boundary in order, boundary 1 first,
 * 2 ints per segment. */
int flow_prep_segments(const flow_mesh *m, int *nb, const int **bbc, const int **nbs,
                       const int **seg);

void flow_prep_free(flow_mesh *m);

/* Message of the last failed flow_prep_* call of this thread. */
const char *flow_prep_last_error(void);

#ifdef __cplusplus
}
#endif

#endif
