// flow_state.h - device-resident mesh and solver state of one flow context.
//
// Node arrays keep the reference's 1-based array-of-structs layout (a node's
// 4 conserved variables are one aligned 32-byte sector, its gradient one
// 64-byte line), because every face kernel gathers whole node records by
// index.  Face data is re-laid out per face as small aligned structs so each
// face is read with one or two vector loads.  All incidence lists are sorted
// by face index, which is what makes the per-node gathers reproduce the
// reference's sequential scatter order bit for bit.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace flow {

struct DevMesh {
  int nn;        // real nodes (1..nn)
  int ng;        // ghost nodes (nn+1..nn+ng)
  int ne;        // edges (1..ne)
  int ns;        // subedges (1..ns)
  int nbe;       // boundary edges (1..nbe)
  int nnz;       // CSR blocks
  int order;     // reconstruction order of the run (1 or 3)
  int stencil_max;
  // node -> incident subedges, (s << 1) | side, side 0 = node is the edge's L
  const int* nsub_ptr;
  const int* nsub;
  const int* nsub_slot;  // per incidence: the row position (k - ia[node]) of the block
                         // (node, the face's other node); used by k_faces_assemble
  // node -> incident boundary edges (ascending)
  const int* nbed_ptr;
  const int* nbed;
  // node -> incident edges, (e << 1) | side, and the node at the edge's other end
  const int* nedg_ptr;
  const int* nedg;
  const int* nedg_nbr;
  // block CSR (reference Build_CRS layout: diagonal block last in each row)
  const int* ia;
  const int* iau;
  const int* ja;
  const int4* csr_sub;   // per block: {first subedge, second subedge or -1, role, 0}
  // faces
  const int2* sub_lr;
  const double4* sub_geo;  // nx, ny, len, 0
  const double4* sub_dx;   // face point - x[L], face point - x[R]
  const double* sub_xg;    // 3 Gauss points, 6 doubles
  const int2* edge_lr;
  const double4* edge_w;   // LSQ weights wL (2), wR (2)
  const int4* bed_info;    // real node, ghost node (absolute), bc, is_wall
  const double2* bed_cnrm; // curved-boundary normal at the real node
  const double* xg_bedges; // 6 per bedge
  const double* xgn_bedges;// 9 per bedge
  // nodes
  const double* x;
  const double* cv_area;
  const int* node_order;
  const double* moments;   // 9 per node
  // k=2 stencil and factors
  const int* st_ptr;
  const int* st_idx;
  const double* st_w;
  const double* svd_U1;    // per node: first 5 columns of U, row by row, offset 5*st_ptr[i]
  const double* svd_VT;    // 25 per node
  const double* svd_S;     // 5 per node
};

// Precision form: FP32 off-diagonal blocks and LU factors laid out in
// colour order (rows of one colour contiguous), for the multicolour sweeps.
struct MixedTables {
  int ncolors;
  const int* color_ptr;   // ncolors+1: first position of each colour
  const int* rows;        // nn: row at each position (colour-sorted, ascending)
  const int* pos;         // nn+1: position of each row
  const int* offd_ptr;    // nn+1: first off-diagonal block of each position
  const int4* rowinfo;    // nn: {row, first block, end block, 0} of each position
  const int* offd_col;    // column (row index) of each off-diagonal block
  float* lhs32;           // 16 floats per off-diagonal block, row-major
  float* lu32;            // 16 floats per position: LU factors, reciprocal pivots
  float* dq32;            // 4 floats per row (1..nn), the sweeps' iterate
  float* dq32b;           // second buffer of the ordered FP32 sweeps (swapped per sweep)
};

// Precision form, chunked order (mode 3).  The reference row order is cut
// into chunks of consecutive rows (at most a set number of rows and of
// dependency levels each), coloured greedily so that chunks of one colour
// share no block; a sweep runs the colours in order, one CTA per chunk, and
// inside a chunk the rows in the reference's order, level by level.  Each
// direction keeps one record per row, in chunk / sub-level order, with all
// the sweep reads of that row; a sub-level is at most kRecRows rows of one
// level.
constexpr int kRecBlocks = 8;  // off-diagonal blocks a record holds

struct __align__(16) SweepRec {
  int4 hdr;                 // row j, off-diagonal block count, 0, 0
  float4 rhs;               // right-hand side (FP32)
  float4 lu[4];             // LU factors of the diagonal block, reciprocal pivots
  int4 cols[2];             // columns of the off-diagonal blocks (0: none)
  float4 a[4 * kRecBlocks]; // the blocks, row-major, block t row r at a[4t + r]
};

struct ChunkTables {
  int nchunks, ncol, maxwin;
  const int* col_ptr;        // ncol+1: chunks of each colour in col_chunks
  const int* col_chunks;
  const int2* window;        // per chunk: first and last row any of its rows touches
  SweepRec* rec[2];          // per direction (0 forward, 1 backward)
  const int* sub_start[2];   // record index of each sub-level, plus the end
  const int* chunk_sub[2];   // first sub-level of each chunk, plus the end
  const int* pos[2];         // record index of each row (1..nn)
  int ring;                  // ring shape of the sub-level tables: rows 64 >> ring
  // one-launch (dataflow) sweeps
  const int* task_chunk[2];  // per direction: chunks in dispensing (colour) order
  const int* colour;         // colour of each chunk
  const int2* nbr;           // per chunk: first and last chunk its window overlaps
  int* done;                 // per chunk: sweep generation + 1 once finished
  unsigned* sync;            // dispenser, chunks finished, sweep generation
};

struct DevState {
  double* Q;
  double* nQ;
  double* pQ;
  double* dQ;       // current dQ (the host swaps it with dQ2 after each ordered sweep)
  double* dQ2;
  double* R;
  double* RHS;
  double* grad;     // 8 per node
  double* phi;      // 8 per node
  double* hess5;    // 20 per node (var-major, 5 derivatives)
  double* pv;       // 4 per node (point values)
  double* dt;
  double* LHS;      // nnz * 16
  double* LUd;      // 16 per node: LU factors of the diagonal block
  double* xn_bedges;// 3 per bedge (mutated by the k=2 boundary pass)
  double* F;        // 4 per subedge
  double* JL;       // 16 per subedge
  double* JR;       // 16 per subedge
  double* Fb;       // 4 per bedge
  double* Jb;       // 16 per bedge
  double* bforce;   // 4 per bedge: lift, drag, is-wall (body-force scratch)
  int* done;        // per row epoch flags for the ordered sweeps
  unsigned int* counter;  // row dispenser for the ordered sweeps
  int* status;      // sticky error bits (FLOW_ERR_*)
  int* skip;        // set when the linear residual dropped below 1e-15
  int* exact;       // set when that test needs the reference's summation order
  int* stop;        // set once the run's density residual dropped below its target
  int* steps_done;  // pseudo-time steps completed since the last reset
  int* citer;       // pseudo-time step index of the step in flight (drives the CFL ramp)
  double* partial;  // reduction partials
  double* scalars;  // [0] rms, [1] dq^2, [2] R_rho^2, [3] cfl, [4] F_lift, [5] F_drag,
                    // [6] R_rho of the run's first step, [7] target drop (0 = none)
};

}  // namespace flow
