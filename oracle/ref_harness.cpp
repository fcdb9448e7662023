/*
 * ref_harness.cpp - C entry points around the UNMODIFIED reference solver.
 *
 * Test infrastructure (the oracle): compiled together with the reference's
 * own *.C files (everything except main.C) by oracle/build_ref.sh into
 * oracle/_ref/libflowref.so.  It replays the set-up sequence of the
 * reference driver (main.C:107-666: read_parameters, read_mesh,
 * Cuthill_McKee, metrics2D, the maps of maps.C, Find_Element_Centroids,
 * Build_Edge_Data, Build_Boundary_Edge_Data, Fix_Subedge_Data,
 * Generate_Gaussian_Data_For_Edge, cv_calc_*, Build_CRS, node_order, init_pv)
 * and then exposes solve(), the individual hot-path stages and the GRID /
 * SYS_MEM arrays to the tests.  It never runs inside the solver.
 *
 * The reference prints to stdout on every call; the harness sends fd 1 to
 * /dev/null for the duration of each call.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>
#include <fcntl.h>
#include "grid.h"
#include "sys_mem.h"
#include "params.h"
#include "Defined_Variables.h"
#include "mesh_io.h"
#include "reorder.h"
#include "metrics.h"
#include "maps.h"
#include "geometry.h"
#include "cv_calc.h"
#include "init_memory.h"
#include "ic.h"
#include "solve.h"
#include "grid_io.h"
#include "residual.h"
#include "linear_algebra.h"
#include "gradient.h"
#include "compute_derivatives.h"
#include "limiter.h"
#include "cvbc.h"

struct RefCase {
  GRID grid;
  SYS_MEM smem;
  PARAMS p;
};

static int g_quiet = 1;

struct Mute {
  int saved;
  Mute() : saved(-1) {
    if (!g_quiet) return;
    fflush(stdout);
    saved = dup(1);
    int dn = open("/dev/null", O_WRONLY);
    if (dn >= 0) { dup2(dn, 1); close(dn); }
  }
  ~Mute() {
    if (saved < 0) return;
    fflush(stdout);
    dup2(saved, 1);
    close(saved);
  }
};

struct Cwd {
  char old[4096];
  int ok;
  Cwd(const char *dir) : ok(0) {
    if (getcwd(old, sizeof(old)) && chdir(dir) == 0) ok = 1;
  }
  ~Cwd() { if (ok && chdir(old) != 0) { /* nothing to restore into */ } }
};

extern "C" {

void ref_set_quiet(int q) { g_quiet = q; }

/* Set-up exactly as main.C does it for a fresh (non-restart) run. */
void *ref_open(const char *casedir, const char *meshname)
{
  RefCase *c = new RefCase();
  Cwd cwd(casedir);
  if (!cwd.ok) { delete c; return NULL; }
  Mute mute;
  GRID &grid = c->grid;
  read_parameters(&c->p);
  char name[1024];
  strncpy(name, meshname, sizeof(name) - 1);
  name[sizeof(name) - 1] = 0;
  read_mesh(name, &grid, c->p);
  strcpy(grid.gridname, "mesh");
  if (c->p.isrestart == 0 && c->p.reorder == 1) Cuthill_McKee(&grid);
  metrics2D(&grid);
  Cells_Surrounding_Node(grid.nn, grid.num_elem, grid.c2n, &(grid.csn), &(grid.ncsn));
  Nodes_Surrounding_Node(grid.nn, grid.num_elem, grid.c2n, grid.csn, grid.ncsn,
                         &(grid.nsn), &(grid.nnsn));
  Edges_Surrounding_Node(grid.nn, grid.nsn, grid.nnsn, &(grid.nedges), &(grid.edges),
                         &(grid.esn));
  Build_Cell_to_Edge_Map(grid.c2n, grid.num_elem, grid.nsn, grid.nnsn, grid.esn, &(grid.c2e));
  Elements_Surrounding_Element(grid.num_elem, grid.c2n, grid.csn, grid.ncsn, &(grid.ese),
                               &(grid.nese));
  Nodes_Surrounding_Node2(grid.nn, grid.num_elem, grid.c2n, grid.esn, grid.nnsn, grid.edges,
                          &(grid.nsn2), &(grid.nnsn2));
  Initialize_Generic_Nodes_Surrounding_Node(grid.nn, grid.num_elem, grid.c2n, grid.esn,
                                            grid.nnsn, grid.edges, &(grid.gnsn),
                                            &(grid.gnnsn), &(grid.gnnsn1),
                                            &(grid.node_fill_level));
  Find_Element_Centroids(&grid);
  Build_Edge_Data(&grid);
  Build_Boundary_Edge_Data(&grid);
  Fix_Subedge_Data(&grid);
  Generate_Gaussian_Data_For_Edge(&grid);
  cv_calc_area_Green(&grid);
  cv_calc_check_closure(&grid);
  cv_calc_length_scale(&grid);
  cv_calc_Moments(&grid);
  Build_CRS(&grid, c->p, &c->smem);
  for (int i = 1; i <= grid.nn; i++) grid.node_order[i] = c->p.order;
  for (int i = 1; i <= grid.nbedges; i++) {
    int n = grid.bedges[i * 5 + 0];
    int gn = grid.bedges[i * 5 + 1] + grid.nn;
    grid.node_order[gn] = grid.node_order[n];
  }
  init_pv(&grid, c->p);
  return c;
}

void ref_close(void *h) { delete (RefCase *)h; }

/* One pseudo-time step as main.C:789-815 runs it; returns ||dQ||_2. */
double ref_solve(void *h, int ts)
{
  RefCase *c = (RefCase *)h;
  Mute mute;
  c->grid.eltime = ts * c->p.mintime;
  c->grid.citer = ts;
  c->grid.iter = ts;
  return solve(&c->grid, &c->smem, c->p, ts);
}

void ref_body_forces(void *h, double *forces)
{
  RefCase *c = (RefCase *)h;
  Mute mute;
  forces[0] = 0.;
  forces[1] = 0.;
  Compute_Body_Forces(&c->grid, c->p, forces);
}

/* ---- individual stages (same calls solve() makes, solve.C:344-881) ---- */
void ref_set_citer(void *h, int citer) { ((RefCase *)h)->grid.citer = citer; }

void ref_build_matrix(void *h)
{
  RefCase *c = (RefCase *)h;
  Mute mute;
  build_matrix(&c->grid, c->p, &c->smem);
}

void ref_gradient(void *h)
{
  RefCase *c = (RefCase *)h;
  Mute mute;
  Compute_Gradient_LeastSquares(&c->grid);
}

void ref_derivatives(void *h, int order)
{
  RefCase *c = (RefCase *)h;
  Mute mute;
  Compute_Derivatives(&c->grid, c->p, order);
}

void ref_limiter(void *h)
{
  RefCase *c = (RefCase *)h;
  Mute mute;
  compute_limiter_venkatakrishnan(&c->grid, c->p);
}

void ref_interior(void *h, int jupdate, int ts)
{
  RefCase *c = (RefCase *)h;
  Mute mute;
  build_interior_residuals(&c->grid, &c->smem, c->p, jupdate, ts);
}

void ref_boundary(void *h, int jupdate)
{
  RefCase *c = (RefCase *)h;
  Mute mute;
  build_boundary_residuals(&c->grid, &c->smem, c->p, jupdate);
}

void ref_set_boundary_values(void *h)
{
  RefCase *c = (RefCase *)h;
  Mute mute;
  Set_Boundary_Values(&c->grid, c->p);
}

double ref_linear_solve(void *h)
{
  RefCase *c = (RefCase *)h;
  Mute mute;
  return linear_solve(&c->grid, &c->smem, c->p);
}

/* Add the two k=2 stencil layers exactly as solve.C:57-114 does on the first
 * high-order step (normally done inside solve()). */
void ref_grow_stencils(void *h)
{
  RefCase *c = (RefCase *)h;
  GRID *grid = &c->grid;
  Mute mute;
  for (int i = 1; i <= grid->nn; i++)
    Add_Layer_to_GNSN(grid->nn, grid->num_elem, grid->c2n, grid->esn, grid->nnsn, grid->edges,
                      &(grid->gnsn), &(grid->gnnsn), grid->gnnsn1, grid->node_fill_level, i);
  for (int i = 1; i <= grid->nn; i++)
    if (grid->node_order[i] > 2)
      Add_Layer_to_GNSN(grid->nn, grid->num_elem, grid->c2n, grid->esn, grid->nnsn, grid->edges,
                        &(grid->gnsn), &(grid->gnnsn), grid->gnnsn1, grid->node_fill_level, i);
}

/* Allocate the per-iteration arrays that solve() allocates lazily
 * (solve.C:239-257, residual.C:75-89, init_memory.C:176-186), so that single
 * stages can be driven without a full solve(). */
void ref_alloc_work(void *h)
{
  RefCase *c = (RefCase *)h;
  GRID *g = &c->grid;
  int nn = g->nn;
  if (!g->phi) g->phi = (double *)calloc((nn + 1) * 8, sizeof(double));
  if (!g->grad) g->grad = (double *)calloc((nn + 1) * NDIM * NUM_VAR, sizeof(double));
  if (!g->hess) g->hess = (double *)calloc((nn + 1) * NUM_MOM * NUM_VAR, sizeof(double));
  if (!c->smem.RHS) c->smem.RHS = (double *)calloc((nn + 1) * NUM_VAR, sizeof(double));
  if (!c->smem.LHS)
    c->smem.LHS = (double *)calloc((size_t)c->smem.ia[nn + 1] * NUM_VAR * NUM_VAR, sizeof(double));
}

/* ---- data access ---- */
void ref_scalars(void *h, int *out)
{
  RefCase *c = (RefCase *)h;
  GRID &g = c->grid;
  out[0] = g.nn;
  out[1] = g.nn_ghost;
  out[2] = g.nedges;
  out[3] = g.nsubedges;
  out[4] = g.nbedges;
  out[5] = g.nb;
  out[6] = g.num_elem[Tri];
  out[7] = g.num_elem[Quad];
  out[8] = g.citer;
  out[9] = c->smem.ia ? c->smem.ia[g.nn + 1] : 0;
  out[10] = g.gnnsn1 ? g.gnnsn1[g.nn + 1] : 0;
  out[11] = (g.gnnsn && g.gnnsn1) ? g.gnnsn[g.gnnsn1[g.nn + 1]] : 0;
  out[12] = g.num_elem[Edge];
  out[13] = g.nnsn ? g.nnsn[g.nn + 1] : 0;
}

void ref_params(void *h, double *out)
{
  PARAMS &p = ((RefCase *)h)->p;
  double v[] = {(double)p.nsteps, (double)p.iter, (double)p.jufreq, p.CFL, (double)p.ramp,
                p.gamma, p.alpha, p.mach, (double)p.subits, (double)p.unsteady, (double)p.tacc,
                p.mintime, (double)p.method, (double)p.order, (double)p.foits, (double)p.soits,
                (double)p.toits, (double)p.isrestart, (double)p.limit, (double)p.reorder,
                (double)p.ic, (double)p.p_or_cv, (double)p.start_post_pro,
                (double)p.post_pro_freq, ((RefCase *)h)->grid.cfl};
  memcpy(out, v, sizeof(v));
}

/* Pointer + element count of a named array; kind: 0 = double, 1 = int. */
long ref_array(void *h, const char *name, void **ptr, int *kind)
{
  RefCase *c = (RefCase *)h;
  GRID &g = c->grid;
  SYS_MEM &s = c->smem;
  long nn = g.nn, ng = g.nn_ghost, ne = g.nedges, ns = g.nsubedges, nb = g.nbedges;
  long nel = g.num_elem[Tri] + g.num_elem[Quad];
  long nnz = s.ia ? s.ia[g.nn + 1] : 0;
#define D(nm, p, n) if (!strcmp(name, nm)) { *ptr = (void *)(p); *kind = 0; return (p) ? (n) : 0; }
#define I(nm, p, n) if (!strcmp(name, nm)) { *ptr = (void *)(p); *kind = 1; return (p) ? (n) : 0; }
  D("x", g.x, (nn + ng + 1) * 2);
  D("Q", g.Q, (nn + ng + 1) * 4);
  D("nQ", g.nQ, (nn + ng + 1) * 4);
  D("pQ", g.pQ, (nn + ng + 1) * 4);
  D("dQ", g.dQ, (nn + 1) * 4);
  D("R", g.R, (nn + 1) * 4);
  D("dt", g.dt, (nn + 1));
  D("grad", g.grad, (nn + 1) * 8);
  D("hess", g.hess, (nn + 1) * 36);
  D("phi", g.phi, (nn + 1) * 8);
  D("point_value", g.point_value, (nn + 1) * 4);
  D("cv_area", g.cv_area, nn + 1);
  D("ev_con", g.ev_con, nn + 1);
  D("Moments", g.Moments, (nn + 1) * 9);
  D("el_cent", g.el_cent, (nel + 1) * 2);
  D("xn_edges", g.xn_edges, (ne + 1) * 3);
  D("xn_subedges", g.xn_subedges, (ns + 1) * 3);
  D("xm_subedges", g.xm_subedges, (ns + 1) * 2);
  D("xg_subedges", g.xg_subedges, (ns + 1) * 6);
  D("xn_bedges", g.xn_bedges, (nb + 1) * 3);
  D("xg_bedges", g.xg_bedges, (nb + 1) * 6);
  D("xgn_bedges", g.xgn_bedges, (nb + 1) * 9);
  D("edge_weight", g.edge_weight, (ne + 1) * 4);
  D("length_scale", g.length_scale, nn + 1);
  D("SVD_size", g.SVD_size, (nn + 1) * 3);
  D("LHS", s.LHS, nnz * 16);
  D("RHS", s.RHS, (nn + 1) * 4);
  I("edges", g.edges, (ne + 1) * 2);
  I("subedges", g.subedges, (ns + 1) * 2);
  I("bedges", g.bedges, (nb + 1) * 5);
  I("bbc", g.bbc, g.nb + 1);
  I("node_order", g.node_order, nn + ng + 1);
  I("node_state", g.node_state, nn + ng + 1);
  I("nn_map", g.nn_map, nn + 1);
  I("ia", s.ia, nn + 2);
  I("iau", s.iau, nn + 1);
  I("ja", s.ja, nnz);
  I("nsn", g.nsn, g.nnsn ? g.nnsn[g.nn + 1] : 0);
  I("nnsn", g.nnsn, nn + 2);
  I("esn", g.esn, g.nnsn ? g.nnsn[g.nn + 1] : 0);
  I("c2n_tri", g.c2n ? g.c2n[Tri] : 0, (g.num_elem[Tri] + 1) * 3);
  I("c2n_quad", g.c2n ? g.c2n[Quad] : 0, (g.num_elem[Quad] + 1) * 4);
  I("c2n_edge", g.c2n ? g.c2n[Edge] : 0, (g.num_elem[Edge] + 1) * 2);
  I("gnnsn1", g.gnnsn1, nn + 2);
  I("gnnsn", g.gnnsn, g.gnnsn1 ? g.gnnsn1[g.nn + 1] + 1 : 0);
  I("gnsn", g.gnsn, (g.gnnsn && g.gnnsn1) ? g.gnnsn[g.gnnsn1[g.nn + 1]] : 0);
  I("node_fill_level", g.node_fill_level, nn + 1);
#undef D
#undef I
  *ptr = NULL;
  *kind = -1;
  return -1;
}

/* Boundary segment b, s -> its two nodes (bs[b][s][0..1]). */
void ref_segment(void *h, int b, int s, int *n0n1)
{
  GRID &g = ((RefCase *)h)->grid;
  n0n1[0] = g.bs[b][s][0];
  n0n1[1] = g.bs[b][s][1];
}

int ref_nbs(void *h, int b) { return ((RefCase *)h)->grid.nbs[b]; }

/* SVD factors of node i (after Compute_Derivatives): m x m U, 5 x 5 VT, S. */
int ref_svd(void *h, int i, double **U, double **VT, double **S)
{
  GRID &g = ((RefCase *)h)->grid;
  if (!g.SVD_U || !g.SVD_U[i]) return 0;
  *U = g.SVD_U[i];
  *VT = g.SVD_V[i];
  *S = g.SVD_S[i];
  return (int)g.SVD_size[i * 3 + 0];
}

double ref_cfl(void *h) { return ((RefCase *)h)->grid.cfl; }

/* write_surface_cp (grid_io.C:841-1375) from the current GRID::Q: it writes
 * surface_<b>_pressure.dat into the working directory and orders each file
 * with the shell's `sort -g`, so the call runs in `dir` with LC_ALL=C for
 * its duration (ties then order bytewise).  Returns 0, or -1 if dir cannot
 * be entered. */
int ref_write_surface_cp(void *h, const char *dir)
{
  RefCase *c = (RefCase *)h;
  Cwd cwd(dir);
  if (!cwd.ok) return -1;
  const char *old = getenv("LC_ALL");
  char saved[256] = {0};
  if (old) strncpy(saved, old, sizeof(saved) - 1);
  setenv("LC_ALL", "C", 1);
  {
    Mute mute;
    write_surface_cp(&c->grid, c->p);
  }
  if (old) setenv("LC_ALL", saved, 1); else unsetenv("LC_ALL");
  return 0;
}

/* write_mesh (mesh_io.C:300-393): the mesh and the restart block of the
 * current GRID::Q, GRID::citer and GRID::cfl. */
void ref_write_mesh(void *h, const char *path)
{
  RefCase *c = (RefCase *)h;
  char name[4096];
  strncpy(name, path, sizeof(name) - 1);
  name[sizeof(name) - 1] = 0;
  Mute mute;
  write_mesh(name, &c->grid);
}

/* write_tecplot_solutionC (primitive 0, grid_io.C:102-199) or
 * write_tecplot_solutionP (grid_io.C:216-331) of the current GRID::Q. */
void ref_write_tecplot(void *h, const char *path, int primitive)
{
  RefCase *c = (RefCase *)h;
  char name[4096];
  strncpy(name, path, sizeof(name) - 1);
  name[sizeof(name) - 1] = 0;
  Mute mute;
  if (primitive) write_tecplot_solutionP(name, &c->grid, c->p.gamma);
  else write_tecplot_solutionC(name, &c->grid);
}

}  // extern "C"
