/*
 * flow_gpu.h - C ABI of the B200 implementation of the flow solver's
 * nonlinear iteration (libflowgpu.so).
 *
 * The reference solver (shedsaw/flow-solver) exposes this path as C++
 * functions over its GRID / SYS_MEM / PARAMS objects.  Every entry point
 * below replaces one of them and takes the same data as plain pointers in the
 * reference's own array layout (1-based, array-of-structs), so a C++ shim
 * with the reference's signatures can forward GRID fields directly.  No
 * torch or CUDA types appear in the signatures.
 *
 * Error behaviour: where the reference prints and calls exit() (cvbc.C:330,
 * init_memory.C:257-268, limiter.C:965-977, cv_calc.C:868-875), these entry
 * points return a nonzero FLOW_ERR_* bit set instead and leave the context
 * usable.  All functions are synchronous with respect to the host buffers
 * they take; the device work of one context runs on its own CUDA stream.
 */
#ifndef FLOW_GPU_H
#define FLOW_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

/* Error bits (sticky per context until flow_clear_status). */
#define FLOW_OK 0
#define FLOW_ERR_ARG 1          /* bad argument or unsupported option */
#define FLOW_ERR_CUDA 2         /* CUDA runtime error */
#define FLOW_ERR_EIGEN 4        /* non-finite wave speed (cv_calc.C:868-875) */
#define FLOW_ERR_DT 8           /* dt <= 0 or non-finite (init_memory.C:257-268) */
#define FLOW_ERR_LIMITER 16     /* phi outside [0,1] (limiter.C:965-977) */
#define FLOW_ERR_BC 32          /* invalid far-field state (cvbc.C:330-382) */
#define FLOW_ERR_SWEEP_TIMEOUT 64 /* an ordered sweep waited past its bound */
#define FLOW_ERR_NOT_FOUND 128  /* unknown array name */
#define FLOW_ERR_NOT_CONVERGED 256 /* flow_converge reached max_steps */
#define FLOW_ERR_BUDGET 512     /* the arena (or the server's slot table) has no room now */
#define FLOW_ERR_STALLED 1024   /* a served solve's residual stopped falling (flow_server_set_stall) */

/* Mirrors PARAMS (include/params.h:19-76 of the reference), same field
 * order and meaning as euler.params (params.C:44-217). */
typedef struct flow_params {
  int nsteps;
  int iter;
  int jufreq;
  double CFL;
  int ramp;
  double gamma;
  double alpha;
  double mach;
  int subits;
  int unsteady;
  int tacc;
  double mintime;
  int method;
  int order;
  int foits;
  int soits;
  int toits;
  int isrestart;
  int limit;
  int reorder;
  int ic;
  int p_or_cv;
  int start_post_pro;
  int post_pro_freq;
} flow_params;

/* Read-only view of a pre-processed grid in the reference's layout
 * (include/grid.h:223-307 and include/sys_mem.h:43-49).  Array lengths are
 * those the reference allocates (index 0 unused unless noted).  For order 3
 * the stencil and SVD fields may all be NULL when the caller forms the k=2
 * derivatives itself (flow_set "hess" / "point_value"); steps of the k=2
 * scheme on the device (flow_solve, flow_run, flow_reconstruct ...) then
 * return FLOW_ERR_ARG. */
typedef struct flow_grid_view {
  int nn;          /* GRID::nn */
  int nn_ghost;    /* GRID::nn_ghost */
  int nedges;      /* GRID::nedges */
  int nsubedges;   /* GRID::nsubedges */
  int nbedges;     /* GRID::nbedges */
  int nb;          /* GRID::nb */
  int nelem;       /* triangles + quads */
  const int *edges;       /* (nedges+1)*2 */
  const int *subedges;    /* (nsubedges+1)*2 */
  const int *bedges;      /* (nbedges+1)*5 */
  const int *bedge_seg;   /* (nbedges+1)*2: GRID::bs[b][s][0..1] of each bedge */
  const int *bbc;         /* nb+1 */
  const int *node_order;  /* nn+nn_ghost+1 */
  const int *ia;          /* nn+2   (SYS_MEM::ia) */
  const int *iau;         /* nn+1   (SYS_MEM::iau) */
  const int *ja;          /* ia[nn+1] (SYS_MEM::ja) */
  const double *x;            /* (nn+nn_ghost+1)*2 */
  const double *cv_area;      /* nn+1 */
  const double *el_cent;      /* (nelem+1)*2 */
  const double *xn_subedges;  /* (nsubedges+1)*3 */
  const double *xm_subedges;  /* (nsubedges+1)*2 */
  const double *xg_subedges;  /* (nsubedges+1)*6 */
  const double *xn_bedges;    /* (nbedges+1)*3, initial values */
  const double *xg_bedges;    /* (nbedges+1)*6 */
  const double *xgn_bedges;   /* (nbedges+1)*9 */
  const double *edge_weight;  /* (nedges+1)*4 (gradient.C:923-1121); needed for order 1,
                                 and for order 3 with soits > 0; may be NULL otherwise */
  const double *moments;      /* (nn+1)*9 (GRID::Moments); NULL if order != 3 */
  /* k=2 two-ring stencils after the growth of solve.C:57-114 (GRID::gnsn,
   * gnnsn, gnnsn1) and the SVD factors of compute_derivatives.C:845-940
   * (GRID::SVD_U / SVD_V / SVD_S); NULL if order != 3. */
  const int *gnsn;
  const int *gnnsn;
  const int *gnnsn1;
  const int *svd_m;           /* nn+1: rows m of node i's system */
  const long *svd_off;        /* nn+1: offset of node i's U block in svd_U */
  const double *svd_U;        /* per node, column-major with leading dimension m;
                                 only the first 5 columns are read */
  const double *svd_VT;       /* (nn+1)*25 */
  const double *svd_S;        /* (nn+1)*5 */
} flow_grid_view;

typedef struct flow_ctx flow_ctx;

/* Upload a grid (and the CSR pattern of Build_CRS, init_memory.C:36-138) to
 * device `device`.  Replaces the lazily built device mirror the reference's
 * solve() would need; returns NULL and sets *status on failure. */
flow_ctx *flow_create(const flow_grid_view *grid, const flow_params *p, int device,
                      int *status);
void flow_destroy(flow_ctx *ctx);

/* Start a solve from GRID::Q = Q (and nQ = Q), (nn+nn_ghost+1)*4 doubles
 * (ic.C:36-99 output).  The boundary normals that the k=2 boundary pass
 * rewrites (residual.C:1103-1143) go back to their initial values. */
int flow_set_state(flow_ctx *ctx, const double *Q);

/* double solve(GRID*, SYS_MEM*, PARAMS, int ts)  (include/solve.h:21,
 * solve.C:44-933): one pseudo-time step at time step ts (GRID::citer = ts).
 * *dq_norm receives the return value ||dQ||_2 and *r_rho the density
 * residual norm ||R[:,0]||_2 of the last Newton iteration (either may be
 * NULL). */
int flow_solve(flow_ctx *ctx, const flow_params *p, int ts, double *dq_norm, double *r_rho);

/* Run `nsteps` steps ts = ts0 .. ts0+nsteps-1 without host round trips
 * (the driver loop of main.C:789-815); stops early on error.  r_rho_hist and
 * dq_hist (optional, nsteps entries) receive the per-step norms. */
int flow_run(flow_ctx *ctx, const flow_params *p, int ts0, int nsteps, double *r_rho_hist,
             double *dq_hist);

/* The driver loop of main.C:789-815 run to convergence: steps
 * ts = ts0, ts0+1, ... until ||R[:,0]||_2 < drop * (its value at step ts0)
 * or max_steps steps.  The test runs on the device; the host looks at it
 * every `chunk` steps, and steps enqueued after convergence do no work.
 * *steps receives the steps taken (the step that met the target included),
 * *r_first / *r_last the density residual norms of the first / last step.
 * Returns FLOW_ERR_NOT_CONVERGED when max_steps ran out.  The reference's
 * driver has no convergence test (it runs nsteps steps); this is the
 * 1e-10-drop criterion the solves/s metric is quoted on. */
int flow_converge(flow_ctx *ctx, const flow_params *p, int ts0, int max_steps, double drop,
                  int chunk, int *steps, double *r_first, double *r_last);

/* flow_converge for n independent contexts at once (a batch of solves):
 * each context's steps run on its own stream so the solves overlap on the
 * device; the host issues `chunk` steps per context per round and reads each
 * context's stop flag one round later.  steps[i] / status[i] (optional)
 * receive each solve's step count and status; the return value ORs the
 * statuses.  Use flow_last_device_ms per context for its device span. */
int flow_converge_batch(flow_ctx **ctxs, int n, const flow_params *p, int ts0, int max_steps,
                        double drop, int chunk, int *steps, int *status);

/* void build_matrix(GRID*, PARAMS, SYS_MEM*)  (include/init_memory.h:24,
 * init_memory.C:159-310) with GRID::citer = citer; writes dt and the V/dt
 * diagonal (LHS otherwise zero). */
int flow_build_matrix(flow_ctx *ctx, const flow_params *p, int citer);

/* Compute_Gradient_LeastSquares (gradient.C:245-403) or, for order 3,
 * Compute_Derivatives(grid, p, 3) (compute_derivatives.C:1438-1534),
 * followed by compute_limiter_venkatakrishnan (limiter.C:511-983) when
 * p->limit == 2.  Uses the current nQ. */
int flow_reconstruct(flow_ctx *ctx, const flow_params *p, int ts);

/* void build_interior_residuals(GRID*, SYS_MEM*, PARAMS, int jupdate, int ts)
 * (include/residual.h:21, residual.C:40-342) together with
 * void build_boundary_residuals(GRID*, SYS_MEM*, PARAMS, int jupdate)
 * (include/residual.h:23, residual.C:359-1230) and the Jacobian callbacks of
 * include/jacobian.h:21-33; assembles R, RHS = -R and the LHS blocks on top
 * of the diagonal written by flow_build_matrix. */
int flow_residuals(flow_ctx *ctx, const flow_params *p, int jupdate, int ts);

/* The same two functions one at a time, as the reference's solve() calls
 * them (solve.C:689, 729) with host code between them:
 * stage FLOW_STAGE_INTERIOR is build_interior_residuals (residual.C:40-342):
 * the interior faces' fluxes and, with jupdate, their Jacobians summed into
 * R and onto the LHS blocks that flow_build_matrix left; FLOW_STAGE_BOUNDARY
 * is build_boundary_residuals (residual.C:359-1230): the ghost states, the
 * boundary fluxes and approximate Jacobians added to R and the diagonal
 * blocks.  Interior then boundary gives the bits flow_residuals gives.  The
 * reconstruction inputs (grad, phi, hess, point_value) are those on the
 * device: flow_reconstruct's, or the caller's own through flow_set.  FP64
 * drop-in only (precision mode 0). */
#define FLOW_STAGE_INTERIOR 1
#define FLOW_STAGE_BOUNDARY 2
int flow_residual_stage(flow_ctx *ctx, const flow_params *p, int jupdate, int ts, int stage);

/* double linear_solve(GRID*, SYS_MEM*, PARAMS)  (include/linear_algebra.h:23,
 * linear_algebra.C:122-401): p->subits alternating ordered block Gauss-Seidel
 * sweeps from dQ = 0; *rms receives the returned b-Ax RMS. */
int flow_linear_solve(flow_ctx *ctx, const flow_params *p, double *rms);

/* The b - Ax RMS that stops linear_solve's sweep loop below 1e-15
 * (linear_algebra.C:348-387) is reduced as a tree on the device; when it
 * lies within the tree sum's rounding bound of 1e-15, it is summed again in
 * the reference's row order, so the loop stops where the reference's does.
 * on != 0 sums every RMS in that order (slow; for checking the returned RMS
 * bit for bit). */
int flow_set_exact_rms(flow_ctx *ctx, int on);

/* void Compute_Body_Forces(GRID*, PARAMS, double*)  (include/grid_io.h:36,
 * grid_io.C:1390-1697): raw pressure lift and drag on the wall boundaries. */
int flow_body_forces(flow_ctx *ctx, const flow_params *p, double *forces);

/* ---- Outputs of a solve (grid_io.C), from the resident state GRID::Q ----
 * The GRID arrays these writers read besides the state are passed as plain
 * host pointers: x is GRID::x ((nn+1)*2 or more doubles), tri / quad are
 * GRID::c2n[Tri] / c2n[Quad] (1-based rows, row 0 unused), bbc and nbs are
 * GRID::bbc and GRID::nbs (nb+1 ints, index 0 unused) and seg is every
 * boundary's GRID::bs[b][s][0..1] pairs in order, boundary 1 first.  Where
 * the reference prints a message and exits (a file it cannot open) these
 * return FLOW_ERR_ARG with the message in flow_last_error().  They work on
 * the context's stream and take a small stream-ordered device temporary
 * (cudaMallocAsync: 12 bytes a wall node, 32 bytes a node for Tecplot). */

/* Pressure coefficient of write_surface_cp (grid_io.C:841-1375, its active
 * branch grid_io.C:1292-1354) on boundary b: the boundary's segment nodes in
 * first-appearance order (n0 before n1 of each segment) into nodes_out and
 * Cp = (P/p_inf - 1) * 2/(gamma M^2), p_inf = 1/gamma, into cp_out, computed
 * on the device.  *count receives the number of nodes; FLOW_ERR_ARG if it
 * exceeds cap. */
int flow_surface_cp(flow_ctx *ctx, const flow_params *p, int nb, const int *nbs, const int *seg,
                    int b, int *nodes_out, double *cp_out, int cap, int *count);

/* void write_surface_cp(GRID*, PARAMS)  (include/grid_io.h:34, grid_io.C:841-1375):
 * one file dir/surface_<b>_pressure.dat per inviscid boundary (bbc[b] odd),
 * lines "%f  %f" of (float) x and (float) Cp, ordered as the reference's
 * `sort -g` orders them under the C locale (by the leading number, ties by
 * the line's bytes).  dir NULL or "" writes into the working directory. */
int flow_write_surface_cp(flow_ctx *ctx, const flow_params *p, const char *dir, int nb,
                          const int *bbc, const int *nbs, const int *seg, const double *x);

/* void write_tecplot_solutionC(char*, GRID*) (primitive = 0, include/grid_io.h:22,
 * grid_io.C:102-199) and void write_tecplot_solutionP(char*, GRID*, double)
 * (primitive != 0, include/grid_io.h:24, grid_io.C:216-331): the Tecplot point-data file of the nn real nodes
 * (x, y and Q, or rho, u, v, P) with the element connectivity, the same
 * bytes as the reference writes. */
int flow_write_tecplot(flow_ctx *ctx, const flow_params *p, const char *path, int primitive,
                       const double *x, int ntri, const int *tri, int nquad, const int *quad);

/* void write_mesh(char*, GRID*)  (include/mesh_io.h:21, mesh_io.C:300-393):
 * the mesh followed by the restart block (the last step run, its CFL and the
 * conserved variables of the nn real nodes), the same bytes as the
 * reference writes; flow_prep_read and flow_prep_restart_state read it back
 * to resume the solve. */
int flow_write_restart(flow_ctx *ctx, const flow_params *p, const char *path, const double *x,
                       int ntri, const int *tri, int nquad, const int *quad, int nb,
                       const int *nbs, const int *seg);

/* Copy a named array back in the reference layout: "Q", "nQ", "pQ", "dQ",
 * "R", "RHS", "LHS", "grad", "phi", "hess" ((nn+1)*36), "point_value",
 * "dt", "xn_bedges".  n is the number of doubles the caller provides. */
int flow_get(flow_ctx *ctx, const char *name, double *out, long n);
/* Number of doubles flow_get(name) writes, or -1.  "cfl" (1 double, get
 * only) is GRID::cfl of the last step run: the CFL the ramp of build_matrix
 * set (init_memory.C:200-224). */
long flow_size(flow_ctx *ctx, const char *name);
/* Copy a named array from the host into the context, in the reference
 * layout, the inverse of flow_get: every name flow_get takes but "cfl".  A
 * caller that runs some stages of solve() itself (its own gradient, limiter
 * or k=2 derivatives) hands their results over this way.  "hess" keeps the
 * five derivatives of each variable the k=2 scheme uses; "LHS" also forms the
 * LU factors of the diagonal blocks that the sweeps read.  n is the number
 * of doubles provided (at least flow_size(name)). */
int flow_set(flow_ctx *ctx, const char *name, const double *in, long n);

/* Sweep kernel; both reproduce the reference's sequential block
 * Gauss-Seidel sweeps exactly: 0 = rows dispensed in order to warps across
 * the whole GPU (default); 1 = one CTA per mesh, matrix streamed through a
 * shared-memory ring (uses one SM; for many concurrent meshes; refused when
 * the matrix bandwidth exceeds its dQ window). */
int flow_set_sweep_mode(flow_ctx *ctx, int mode);

/* Precision form (no counterpart in the reference; its defect-correction
 * preconditioner): mode 0 (default) is the FP64 drop-in, bit-identical to
 * the reference.  Mode 1 keeps the residual, geometry, limiter, fluxes,
 * face Jacobians and the update in FP64, but rounds the assembled
 * off-diagonal blocks and the LU factors of the diagonal blocks to FP32
 * and runs p->subits multicolour block Gauss-Seidel sweeps in FP32 (greedy
 * colouring of the block pattern in row order; forward sweeps take the
 * colours ascending, backward sweeps descending).  The converged state is
 * that of mode 0 (same residual); the iterates differ.  Mode 2 is mode 1
 * with the sweeps in the reference's row order (forward rows 1..nn, backward
 * nn..1, the FP64 drop-in's dependency-ordered sweep on FP32 blocks): steps
 * to converge as in mode 0, sweeps latency-bound as in mode 0.  In modes 1
 * and 2 the FP64 LHS is not formed (flow_get "LHS" is stale) and
 * flow_linear_solve reports rms = -1.  Switching builds the FP32 tables.
 * Mode 3 cuts the reference row order into chunks of consecutive rows (at
 * most `rows` rows and `levels` dependency levels each, flow_set_chunk),
 * colours the chunks so that chunks of one colour share no block, and sweeps
 * the colours in order (forward ascending, backward descending), each chunk
 * by one CTA in the reference's order inside the chunk: close to the
 * reference order's convergence with a few launches per sweep.  It needs at
 * most 8 off-diagonal blocks per row and a matrix bandwidth whose chunk
 * windows fit in shared memory; otherwise switching to it fails. */
int flow_set_precision(flow_ctx *ctx, int mode);
/* The context's precision mode (0..3; -1 for a null context). */
int flow_precision_of(flow_ctx *ctx);
/* Face Jacobians of the precision form (no reference counterpart): mode 0
 * (default) the reference's forward differences (jacobian.C:45-185, eight
 * extra Roe fluxes per face); mode 1 the approximate Roe Jacobian
 * dF/dqL = (A(qL) + |A~|) len / 2, dF/dqR = (A(qR) - |A~|) len / 2 with the
 * dissipation matrix |A~| frozen (the form the reference gives its boundary
 * faces, jacobian.C:681-962), which costs no extra flux.  The residual is
 * unchanged, so the converged state is too; only the preconditioner
 * differs.  With mode 1 the interior faces are formed by the nodes that sum
 * them, in one kernel with the assembly (no per-face arrays through device
 * memory; rows of at most 8 off-diagonal blocks, else as mode 2); mode 2 is
 * the same arithmetic in two kernels (faces written, then gathered): the
 * same bits.  Used in precision modes 1-3 only: the FP64 drop-in (mode 0)
 * always differences, as the reference does. */
int flow_set_jacobian(flow_ctx *ctx, int mode);
/* Sweep schedule (no reference counterpart): steps up to `until_step` (0:
 * the end of the CFL ramp, p->ramp) run `sweeps` Gauss-Seidel sweeps instead
 * of p->subits; sweeps = 0 turns the schedule off (default).  Fewer sweeps
 * while the CFL ramps keep the early, poorly conditioned Newton steps from
 * overshooting when the precision form solves them too accurately. */
int flow_set_sweep_schedule(flow_ctx *ctx, int sweeps, int until_step);
/* Paired passes of the mode 3 sweeps (no counterpart in the reference): a
 * symmetric Gauss-Seidel step ends each forward sweep with the colour the
 * backward sweep begins with (and each backward sweep with the colour the
 * next forward begins with).  on != 0 (the default) runs those two passes
 * of a colour as one launch in which every chunk sweeps itself twice with
 * its window kept in shared memory: S sweeps over C colours take S*C - S + 1
 * launches instead of S*C, with the same bits (chunks of one colour read
 * only rows of other colours, which do not change between the two passes). */
int flow_set_sweep_pairs(flow_ctx *ctx, int on);
/* Chunk limits of precision mode 3 (0: defaults, rows = twice the matrix
 * bandwidth up to 2048, levels = 32). */
int flow_set_chunk(flow_ctx *ctx, int rows, int levels);
/* Ring shape of the mode 3 sweep (no counterpart in the reference): the
 * records of sub-levels of `rows` rows (64, 32 or 16; 0 = 64) are prefetched
 * into a shared-memory ring of 3, 6 or 12 slots.  Rows of one dependency
 * level are independent, so every shape gives the same results; smaller
 * sub-levels prefetch further ahead.  FLOW_ERR_ARG (shape unchanged) if a
 * chunk would hold more sub-levels than the sweep kernel does. */
int flow_set_sweep_ring(flow_ctx *ctx, int rows);
/* One-launch mode 3 sweeps (no counterpart in the reference): on != 0 runs
 * each sweep as one launch in which a chunk starts as soon as the chunks of
 * earlier colours that its window overlaps have finished, instead of one
 * launch per colour; the same results (each chunk reads its neighbours at
 * the same point of the sweep).  Waits are bounded: one that runs out sets
 * FLOW_ERR_SWEEP_TIMEOUT.  Used with the 64-row ring shape. */
int flow_set_sweep_dataflow(flow_ctx *ctx, int on);
/* Mode 3 chunks in use: starts[0..nchunks] (first row of each chunk, then
 * nn+1; up to cap entries written), their number and the colour count. */
int flow_chunk_starts(flow_ctx *ctx, int *starts, int cap, int *nchunks, int *ncolours);

/* flow_converge / flow_converge_batch issue steps in chunks; with graphs on
 * (the default) every full chunk after the first is replayed from a CUDA
 * graph captured once per chunk length, with the step index and the CFL
 * ramp advancing on the device.  Results are identical either way; off
 * launches every kernel from the host.  A capture that fails (another
 * thread of the host application synchronised the whole device while it was
 * open) is dropped and its chunk launched kernel by kernel instead, with the
 * same results; only a failure of those launches fails the call.  The
 * library's own device-wide calls (allocation, pinned memory, kernel
 * loading, context teardown) wait for open captures, so several threads may
 * create, run and destroy contexts at once. */
int flow_set_graphs(flow_ctx *ctx, int on);
/* Test hook (no counterpart in the reference): the next `count` chunk
 * captures of this context are discarded as if they had failed, so their
 * chunks take the eager path.  flow_capture_fallbacks returns how many
 * chunks of this context were launched eagerly after a failed capture. */
int flow_set_capture_fault(flow_ctx *ctx, int count);
long flow_capture_fallbacks(flow_ctx *ctx);

/* Recreate the context's stream with a CUDA stream priority (clamped to the
 * device's range; numerically lower is served first).  Kernels of
 * higher-priority streams get free SMs first when solves share the GPU. */
int flow_set_stream_priority(flow_ctx *ctx, int priority);

/* Device snapshot of the solution state (Q, nQ, pQ and the boundary normals
 * the k=2 pass rewrites): flow_save_state keeps a copy on the device,
 * flow_restore_state puts it back (pre-emption / restart without host
 * round trips; the reference's restart goes through the mesh file,
 * mesh_io.C:218-277). */
int flow_save_state(flow_ctx *ctx);
int flow_restore_state(flow_ctx *ctx);

/* Per-kernel device timing with CUDA events on the context's stream
 * (off by default).  flow_kernel_times fills, per kernel class
 * (0 node_prepare, 1 subedge_flux, 2 boundary, 3 assemble, 4 sweep,
 * 5 lin_residual, 6 other), the number of launches and total milliseconds
 * since timing was switched on. */
int flow_set_timing(flow_ctx *ctx, int on);
int flow_kernel_times(flow_ctx *ctx, long *launches, double *ms, int nclasses);

/* The context's CUDA stream (a cudaStream_t), for callers that order their
 * own work or events against it. */
void *flow_stream(flow_ctx *ctx);

int flow_status(flow_ctx *ctx);
void flow_clear_status(flow_ctx *ctx);
const char *flow_last_error(void);
/* Self-test of the sweeps' bounded waits (no counterpart in the reference):
 * one forward ordered sweep whose dispenser skips row 1, so the rows that
 * depend on row 1 poll for a value nothing writes until their spin limit
 * (max_spin polls, at most 2^21), report FLOW_ERR_SWEEP_TIMEOUT, publish a
 * value so that nothing waits on them, and the kernel ends.  *status
 * receives the status bits the sweep left (FLOW_ERR_SWEEP_TIMEOUT expected);
 * the call then clears them.  The solution state is untouched and the
 * context stays usable.  Call it between steps. */
int flow_selftest_sweep_timeout(flow_ctx *ctx, long max_spin, int *status);
/* Number of kernel launches issued by this context so far. */
long flow_launch_count(flow_ctx *ctx);
/* Device time (ms) of the last flow_run / flow_solve call, CUDA events. */
double flow_last_device_ms(flow_ctx *ctx);

/* ---- Autotuner (no counterpart in the reference) -------------------------
 * k_node_prepare4 comes in five variants, k_subedge_flux in three; the
 * results are bit-identical, the speed depends on the mesh.  Variants 0..2
 * of both set the minimum resident blocks per SM the compiler must allow
 * (how many registers a thread may hold); node variant 3 is the staged
 * kernel (a CTA of 32 nodes copies its incidence and stencil slices, then
 * gathers every face record and neighbour state into shared memory with
 * asynchronous copies before the arithmetic), offered where its shared
 * memory fits the mesh; node variant 4 gives each node 16 lanes instead of
 * 4 (its stencil columns, gradient components and face points spread over
 * them, every sum still in the reference's order); node variants 5, 6 and
 * 7 are variants 0, 1 and 4 with a limiter that divides no zero and by no
 * zero (a face point whose reconstruction equals the node's value, or whose
 * bound is the node's own value, folds in the value the reference's
 * quotients give there without dividing), variant 5 also forming the
 * wave-speed face terms in the limiter's walk over the faces; every variant
 * gives the same bits.
 * flow_autotune times each variant over `steps`
 * pseudo-time steps from step index `ts` (CUDA events, after one warm-up
 * step), keeps the fastest, and puts the solution state back as it was
 * with a clear status (the returned status still reports what the timing
 * steps ran into).  variants[2] receives the choice, ms[11] (may be NULL)
 * the average kernel times per variant (ms[0..7] node, ms[8..10] flux;
 * 1e30 for a variant that does not fit).  flow_set_variants sets a choice
 * directly (node 0..7, flux 0..2). */
int flow_autotune(flow_ctx *ctx, const flow_params *p, int ts, int steps, int *variants,
                  double *ms);
int flow_set_variants(flow_ctx *ctx, int node_prepare, int flux);
/* The sweep of precision mode 3 in the shape that runs fastest on this mesh:
 * the record ring of 64, 32 or 16-row sub-levels with one launch per colour
 * (colours per launch = 1), and, with allow_df, the 64-row ring with the
 * whole sweep in one launch (flow_set_sweep_dataflow; its chunks wait for
 * their neighbours on the device, so among many solves it holds SMs that
 * others could use).  Every shape gives the same bits.  Timed like
 * flow_autotune, the state put back; *choice = the rows of the chosen ring,
 * plus 1000 for one launch per sweep; ms[4] (may be NULL) the sweep times
 * (1e30 where a shape does not fit or is not allowed).  The sweep count is
 * not chosen here: it changes the iterates, not only their speed. */
int flow_autotune_sweep(flow_ctx *ctx, const flow_params *p, int ts, int steps, int allow_df,
                        int *choice, double *ms);

/* ---- Device arena (no counterpart in the reference) ----------------------
 * One cudaMalloc of `bytes` on `device`, carved into the buffers of the
 * contexts created in it (256-byte aligned, first fit, freed blocks merge).
 * It is the HBM budget of the serving engine.  Destroy its contexts first. */
typedef struct flow_arena flow_arena;
flow_arena *flow_arena_create(int device, long long bytes, int *status);
void flow_arena_destroy(flow_arena *arena);
long long flow_arena_free_bytes(flow_arena *arena);
long long flow_arena_largest_free(flow_arena *arena);
/* flow_create with every device buffer carved from `arena` (on its device);
 * NULL with *status = FLOW_ERR_BUDGET when the arena has no room for it, and
 * with FLOW_ERR_CUDA for a CUDA error (a failed copy, a device fault). */
flow_ctx *flow_create_in(flow_arena *arena, const flow_grid_view *g, const flow_params *p,
                         int *status);
/* Device bytes a context holds. */
long long flow_ctx_device_bytes(flow_ctx *ctx);

/* ---- Serving engine (no counterpart in the reference) ---------------------
 * Continuous batching of steady solves on one GPU: each submitted solve gets
 * a context in the arena (admission fails with FLOW_ERR_BUDGET while the
 * arena or the slot table is full, and only then: a CUDA error during
 * admission is returned as FLOW_ERR_CUDA) and its own stream; flow_server_progress
 * keeps two chunks of `chunk` pseudo-time steps in flight per running solve
 * and retires solves whose ||R_rho|| dropped by `drop` (status 0), that hit
 * max_steps (FLOW_ERR_NOT_CONVERGED) or failed.  Solves of any mesh, order,
 * flow condition and precision (flow_set_precision modes) share the GPU; each
 * one's iterates are those it has when run alone.  Threads: flow_server_submit
 * and flow_server_stage may be called from several host threads at once
 * (each builds its context concurrently, then takes the server's lock to
 * record it) beside one thread that drives progress / start / result /
 * release; every call but flow_server_destroy is safe against the others,
 * and flow_server_destroy comes after all of them have returned. */
typedef struct flow_server flow_server;
typedef struct {
  long long tag;     /* the submitter's tag */
  int slot;          /* slot to read with flow_server_result, then release */
  int status;        /* 0 converged, FLOW_ERR_NOT_CONVERGED, or error bits */
  int steps;         /* pseudo-time steps taken */
  double r_first;    /* ||R_rho|| of the first step */
  double r_last;     /* ||R_rho|| of the last step */
  double device_ms;  /* device time from the start of the run to retirement */
  long long launches; /* kernel launches the solve issued (graph replays included) */
  int recovered_at;  /* 0, or the step a solve on the approximate face Jacobians went back
                        to after a non-physical state (flow_server_set_recovery) */
} flow_completion;
flow_server *flow_server_create(flow_arena *arena, int chunk, int max_slots, int *status);
void flow_server_destroy(flow_server *srv);
int flow_server_submit(flow_server *srv, const flow_grid_view *g, const flow_params *p,
                       const double *Q0, int precision, double drop, int max_steps,
                       long long tag, int *slot);
/* flow_server_submit split in two: flow_server_stage creates the context and
 * uploads the state (hold = 1: nothing is launched yet) and
 * flow_server_start launches a staged solve. */
/* precision 3 falls back to precision 1 for a mesh that mode 3 cannot take
 * (a row with more than 8 off-diagonal blocks, or a bandwidth whose chunk
 * windows do not fit in shared memory). */
int flow_server_stage(flow_server *srv, const flow_grid_view *g, const flow_params *p,
                      const double *Q0, int precision, double drop, int max_steps,
                      long long tag, int hold, int *slot);
/* A start that fails returns its error (the slot is then finished with that
 * status and must be released); progress never reports it. */
int flow_server_start(flow_server *srv, int slot);
/* Launch further chunks and collect retired solves (at most max_out); waits
 * up to wait_us microseconds for at least one when none is ready. */
int flow_server_progress(flow_server *srv, int wait_us, flow_completion *out, int max_out,
                         int *nout);
/* Converged state Q ((nn+nn_ghost+1)*4 doubles, may be NULL) and the raw
 * lift/drag forces (may be NULL) of a retired solve. */
int flow_server_result(flow_server *srv, int slot, double *Q, long nQ, double *forces);
/* Free a retired solve's context (its arena memory returns to the pool). */
int flow_server_release(flow_server *srv, int slot);
int flow_server_running(flow_server *srv);
/* Autotune the kernel variants of each admitted solve over `steps` steps
 * (flow_autotune), once per (device, order, precision, mesh-size bucket of
 * a factor sqrt(2) in nodes); later admissions in the bucket, by this server
 * or any later one in the process, reuse the choice (the variants' results
 * are bit-identical).  0 (default) turns it off. */
int flow_server_set_autotune(flow_server *srv, int steps);
/* Retire a running solve with FLOW_ERR_STALLED once its best ||R_rho||
 * (relative to its first step, tracked in factors of 10 at chunk
 * boundaries) has not dropped tenfold for `steps` pseudo-time steps -- a
 * limit cycle or a stalled solve that will not reach its drop.  0 (default)
 * turns it off: solves then run to their drop or max_steps. */
int flow_server_set_stall(flow_server *srv, int steps);
/* The stall test of later admissions (no reference counterpart): retire a
 * solve whose best ||R_rho|| has not dropped by the factor `drop` (> 1;
 * default 10) within its window; with steps_per_sqrt_node > 0 the window of
 * a mesh of n nodes is max(steps, steps_per_sqrt_node * sqrt(n)) rounded up
 * to whole chunks (the gaps between a converging solve's improvements grow
 * with the mesh), with 0 (the default) the fixed `steps` of
 * flow_server_set_stall. */
int flow_server_set_stall_rule(flow_server *srv, double drop, double steps_per_sqrt_node);
/* Priority policy for later admissions: 0 (default) one priority for all;
 * 1 the larger the mesh, the greater its stream priority (the longest solves
 * of a batch keep the GPU first, the small ones fill the gaps). */
int flow_server_set_priority_policy(flow_server *srv, int policy);
/* flow_set_jacobian(mode) for every precision-form solve admitted later
 * (0, the default: forward differences). */
int flow_server_set_jacobian(flow_server *srv, int mode);
/* Recovery of precision-form solves on the approximate face Jacobians
 * (flow_set_jacobian 1 or 2; no reference counterpart).  on != 0 (the
 * default): the server keeps the state at the start of each solve's last two
 * chunks (two copies of GRID::Q carved from the arena at admission); when a
 * chunk ends with a non-physical state (FLOW_ERR_EIGEN, _DT, _LIMITER or
 * _BC) it puts the state of that chunk's first step back, switches the solve
 * to the forward-difference Jacobians (mode 0) and runs on from there, once
 * per solve.  flow_completion::recovered_at reports the step.  on == 0: such
 * a solve retires with its error bits, as a context run alone does. */
int flow_server_set_recovery(flow_server *srv, int on);
/* flow_set_sweep_schedule for every precision-form solve admitted later on
 * a mesh of at least min_nodes nodes (measured: the 1.05M-node O-grid needs
 * 2 sweeps during the CFL ramp, meshes up to 124k nodes converge faster
 * without the schedule). */
int flow_server_set_sweep_schedule(flow_server *srv, int sweeps, int until_step,
                                   long long min_nodes);
const char *flow_server_last_error(void);

/* ---- b - A x RMS with no device allocation ------------------------------
 * No counterpart in the reference.  It computes the b - A x RMS that
 * flow_linear_solve returns (linear_algebra.C:348-387) for a 4x4-block BCSR
 * system that sits in the caller's own device memory, and allocates
 * nothing: no cudaMalloc or cudaFree, no allocating library routine.  It is
 * for callers that cannot allocate device memory: host applications that
 * hand all of a GPU's memory to their own arena or caching allocator at
 * start-up (a cudaMalloc behind the arena's back fails once the arena holds
 * the GPU, or fragments it), and time-step loops that must not take the
 * implicit device-wide synchronisation cudaMalloc and cudaFree can cause.
 *
 * Layout (the reference's SYS_MEM): row j = 1..nn owns blocks
 * ia[j] .. ia[j+1]-1, ja[k] is the 1-based column of block k, lhs holds 16
 * doubles per block (row-major 4x4), rhs and x hold (nn+1)*4 doubles with
 * row 0 unused.  ia holds nn+2 entries (ia[nn+1] is read); nnz = ia[nn+1],
 * and ja and lhs hold nnz blocks (ja nnz ints, lhs 16*nnz doubles).  All
 * five are device pointers on the current device.  The
 * work runs on `stream` (NULL: the legacy default stream); the call waits
 * for it and stores the RMS in the host double *rms.  A row pointer or
 * column outside the system is reported as FLOW_ERR_ARG.
 *
 * Scratch: one file-scope __device__ array per device (about 2 MB), sized
 * for FLOW_NOALLOC_MAX_ROWS rows; a larger nn is rejected with FLOW_ERR_ARG
 * and a message in flow_last_error().  The first call on each device does a
 * one-time set-up (its look-up of the array's device address also loads
 * this library's device code on that device): make that first call before
 * any stream capture starts.  Later calls look the address up again, which
 * allocates nothing and follows a module reloaded after cudaDeviceReset.
 * Every call on a device shares the array, which
 * keeps the last call's contents; each call clears the one word that must
 * start at zero.  Calls whose GPU work overlaps (several host threads on
 * different streams) race on the array and return wrong results: serialise
 * them. */
#define FLOW_NOALLOC_MAX_ROWS 262144
int flow_linear_residual_noalloc(const int *ia, const int *ja, const double *lhs,
                                 const double *rhs, const double *x, int nn, long nnz,
                                 void *stream, double *rms);

#ifdef __cplusplus
}
#endif

#endif
