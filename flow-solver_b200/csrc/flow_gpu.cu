// flow_gpu.cu - C ABI of the B200 nonlinear iteration (include/flow_gpu.h).
//
// A flow_ctx owns one mesh resident in HBM (the reference GRID/SYS_MEM
// arrays re-laid out for per-face and per-node gathers, see flow_state.h),
// the solver state, and one CUDA stream.  Host work per step is a fixed
// sequence of kernel launches; nothing is copied back unless asked for.
//
// Compiled with --fmad=false: the face and node kernels reproduce the
// reference's double-precision results bit for bit.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <stdint.h>

#include <algorithm>
#include <type_traits>
#include <map>
#include <mutex>
#include <shared_mutex>
#include <string>
#include <vector>

#include "flow_gpu.h"
#include "flow_internal.h"
#include "flow_kernels.cuh"
#include "flow_sweep_cta.cuh"
#include "host/curved.h"

using namespace flow;

namespace {

thread_local std::string g_last_error;

void set_error(const char* msg) { g_last_error = msg; }

std::shared_mutex g_device_gate;

// Exclusive hold of the device gate for a call that may synchronise the device.
using DeviceWide = std::unique_lock<std::shared_mutex>;

}  // namespace

std::shared_mutex& flow::internal::device_gate() { return g_device_gate; }

// One device allocation carved into the buffers of many contexts
// (offset-indexed, 256-byte aligned first fit with coalescing free list).
struct flow_arena {
  int device = 0;
  char* base = nullptr;
  size_t size = 0, used = 0;
  std::map<size_t, size_t> free_blocks;  // offset -> bytes
  std::mutex mu;

  void* alloc(size_t bytes) {
    bytes = (bytes + 255) & ~size_t(255);
    std::lock_guard<std::mutex> lock(mu);
    for (auto it = free_blocks.begin(); it != free_blocks.end(); ++it) {
      if (it->second < bytes) continue;
      size_t off = it->first, rest = it->second - bytes;
      free_blocks.erase(it);
      if (rest) free_blocks[off + bytes] = rest;
      used += bytes;
      sizes[off] = bytes;
      return base + off;
    }
    return nullptr;
  }
  void release(void* p) {
    if (!p) return;
    std::lock_guard<std::mutex> lock(mu);
    size_t off = (size_t)((char*)p - base);
    auto sz = sizes.find(off);
    if (sz == sizes.end()) return;
    size_t bytes = sz->second;
    sizes.erase(sz);
    used -= bytes;
    auto next = free_blocks.lower_bound(off);
    if (next != free_blocks.end() && off + bytes == next->first) {
      bytes += next->second;
      next = free_blocks.erase(next);
    }
    if (next != free_blocks.begin()) {
      auto prev = std::prev(next);
      if (prev->first + prev->second == off) {
        prev->second += bytes;
        return;
      }
    }
    free_blocks[off] = bytes;
  }
  size_t largest_free() {
    std::lock_guard<std::mutex> lock(mu);
    size_t m = 0;
    for (auto& f : free_blocks) m = std::max(m, f.second);
    return m;
  }
  std::map<size_t, size_t> sizes;  // offset -> bytes of live blocks
};

namespace {

// Device buffers of one context: cudaMalloc'ed, or carved from an arena.
// carve_failed records that an allocation found no room (in an arena that is
// a budget refusal, FLOW_ERR_BUDGET, not a CUDA error).
struct Buffers {
  flow_arena* arena = nullptr;
  std::vector<void*> ptrs;
  size_t bytes = 0;
  bool carve_failed = false;
  template <class T>
  T* alloc(size_t n) {
    if (n == 0) n = 1;
    void* p = nullptr;
    if (arena) {
      p = arena->alloc(n * sizeof(T));
      if (!p) {
        carve_failed = true;
        return nullptr;
      }
    } else {
      DeviceWide gate(g_device_gate);
      if (cudaMalloc(&p, n * sizeof(T)) != cudaSuccess) {
        cudaGetLastError();
        carve_failed = true;
        return nullptr;
      }
    }
    ptrs.push_back(p);
    bytes += (n * sizeof(T) + 255) & ~size_t(255);
    return static_cast<T*>(p);
  }
  // Caller holds the device gate when the buffers are cudaMalloc'ed.
  void release() {
    for (void* p : ptrs) {
      if (arena) arena->release(p);
      else cudaFree(p);
    }
    ptrs.clear();
    bytes = 0;
  }
};

}  // namespace

struct flow_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  Buffers buf;
  DevMesh m{};
  DevState s{};
  int order = 1;
  int nsm = 148;
  int epoch = 0;
  int citer = 0;
  int sweep_mode = 0;  // 0 grid-wide ordered sweep, 1 one-CTA ordered sweep
  long launches = 0;
  double last_ms = 0.;
  bool ok = false;
  // host copies needed to answer flow_get in the reference layout
  int nn = 0, ng = 0, ns = 0, nbe = 0, nnz = 0;
  double drop_target = 0.;   // host copy of the pending target (read by reset_run)
  int* h_flags = nullptr;      // pinned: stop flag and status read back by flow_converge_batch
  cudaEvent_t ev_flag = nullptr;
  int* h_run = nullptr;        // pinned: 2 slots of {stop, status, steps done} for a served run
  double* h_runr = nullptr;    // pinned: 2 slots of {R_rho^2 of the last step, R_rho of the first}
  cudaEvent_t ev_run[2] = {nullptr, nullptr};
  // optional per-kernel event timing
  int timing = 0;
  std::vector<cudaEvent_t> event_pool;
  struct Pending { int cls; cudaEvent_t a, b; int weight; };
  std::vector<Pending> pending;
  long kcount[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  double kms[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  // device snapshot of the solution state
  double *snapQ = nullptr, *snapnQ = nullptr, *snappQ = nullptr, *snapXnb = nullptr;
  double* xnb0 = nullptr;  // boundary normals as created (restored by flow_set_state)
  // state at the start of the last two chunks of a served run (by flag slot)
  double* ckpt[2] = {nullptr, nullptr};
  // one-CTA ordered sweep: stage tables (null when the matrix bandwidth is too
  // large for its dQ window, then the multi-CTA sweep is used)
  SweepTables sweep_tb{};
  bool sweep_cta_ok = false;
  double* d_hist = nullptr;  // 2 x hist_cap device history of (dq, r_rho)
  int hist_cap = 0;
  // precision form (flow_set_precision): 0 FP64 reference order, 1 FP32
  // blocks with multicolour sweeps; tables built on first use
  int precision = 0;
  int var[2] = {0, 0};  // kernel variants: k_node_prepare4, k_subedge_flux (autotuner)
  int sched_sweeps = 0, sched_until = 0;  // sweep schedule (flow_set_sweep_schedule)
  MixedTables mt{};
  bool mt_ordered = false;  // tables in reference row order (modes 2, 3) or colour order (mode 1)
  ChunkTables ct{};          // mode 3 tables and sweep records
  std::vector<int> h_col_ptr, h_chunk_start;
  int chunk_rows = 0, chunk_levels = 0;  // requested limits (0: defaults)
  // sub-level tables of each ring shape of the chunk sweep (per direction);
  // ct.sub_start / ct.chunk_sub point at those of the shape in use
  const int* ring_sub_start[kRingShapes][2] = {};
  const int* ring_chunk_sub[kRingShapes][2] = {};
  bool ring_ok[kRingShapes] = {};
  int ring = 0;  // requested shape: sub-levels of ring_rows(ring) rows
  bool grad_written = false;  // the caller wrote the gradient (flow_set "grad")
  int sweep_df = 0;  // 1: one-launch (dataflow) mode 3 sweeps (flow_set_sweep_dataflow)
  bool has_edge_w = false;  // the grid view carried LSQ edge weights
  bool has_stencils = false;  // order 3: the view carried the k=2 stencils and SVD factors
  std::vector<int> h_color_ptr;
  std::vector<int> h_ia, h_ja;  // host copy of the block pattern
  // CUDA graphs of chunks of K steps with the step index advancing on the
  // device, one per chunk length (flow_set_graphs; on by default)
  int use_graphs = 1;
  struct ChunkGraph {
    cudaGraphExec_t exec = nullptr;
    int K = 0, precision = -1, sweep_mode = -1, phase = -1, sweeps = -1;
    flow_params p{};
    long launches = 0;
  };
  std::vector<ChunkGraph> graphs;
  // a chunk whose capture fails is launched eagerly instead (same kernels,
  // same results); capture_fault discards the next captures on purpose
  // (flow_set_capture_fault), capture_fallbacks counts the eager chunks
  int capture_fault = 0;
  long capture_fallbacks = 0;
  int jac_mode = 0;  // face Jacobians of the precision form (flow_set_jacobian)
  bool fused_ok = false;  // every row has at most kRecBlocks off-diagonal blocks
  int exact_rms = 0;      // every b-Ax RMS in the reference's order (flow_set_exact_rms)
  int sweep_pairs = 1;    // mode 3: a colour's two passes in a row as one launch
  // staged node kernel (node_prepare variant 3): largest per-tile slices and
  // whether its shared memory fits, per order of the kernel
  StageCaps stage_caps{};
  bool stage_ok[2] = {false, false};  // [0] the k=1 kernel, [1] the k=2 kernel
};

namespace {

// Host-to-device copy on the context's stream.  The source may be pageable:
// cudaMemcpyAsync returns once it has been staged, so it may be freed after.
// Nothing here touches the legacy default stream or synchronises the device.
bool upload(flow_ctx* c, void* dst, const void* src, size_t bytes) {
  if (bytes == 0) return true;
  return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->stream) == cudaSuccess;
}

// Device-to-host read of a few results on the context's stream, waited for;
// false (with the CUDA message in flow_last_error) when the copy fails.
bool download(flow_ctx* c, void* dst, const void* src, size_t bytes) {
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) set_error(cudaGetErrorString(e));
  return e == cudaSuccess;
}

// Error code of an allocation that failed: a full arena refuses (budget),
// anything else is a CUDA error.
int carve_error(const flow_ctx* c) {
  return c->buf.arena && c->buf.carve_failed ? FLOW_ERR_BUDGET : FLOW_ERR_CUDA;
}

template <class T>
T* upload_vec(flow_ctx* c, const std::vector<T>& v) {
  T* d = c->buf.alloc<T>(v.size());
  if (!d) return nullptr;
  if (!upload(c, d, v.data(), v.size() * sizeof(T))) return nullptr;
  return d;
}

// Build a CSR list: for each node, items appended in call order.
struct Csr {
  std::vector<int> ptr, idx;
  void build(int n, const std::vector<std::pair<int, int>>& items) {
    ptr.assign(n + 2, 0);
    for (auto& it : items) ptr[it.first + 1]++;
    for (int i = 1; i <= n + 1; i++) ptr[i] += ptr[i - 1];
    idx.assign(items.size(), 0);
    std::vector<int> pos(ptr.begin(), ptr.end());
    for (auto& it : items) idx[pos[it.first]++] = it.second;
  }
};

int launch_check(flow_ctx* c) {
  c->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error(cudaGetErrorString(e));
    return FLOW_ERR_CUDA;
  }
  return 0;
}

StepArgs make_args(const flow_params* p, int ts) {
  StepArgs a{};
  a.gamma = p->gamma;
  double angle = p->alpha * M_PI / 180.;
  a.uinf = p->mach * cos(angle);
  a.vinf = p->mach * sin(angle);
  a.pinf = 1. / p->gamma;
  double angle2 = p->alpha * M_PI / 180;  // grid_io.C:1432
  a.cos_a = cos(angle2);
  a.sin_a = sin(angle2);
  const int hi = ts > (p->foits + p->soits);
  a.do_grad = (p->order == 1 && ts > p->foits) || (p->order == 3 && ts > p->foits && !hi);
  a.do_derivs = (p->order == 3 && hi);
  a.do_lim = (p->order == 1 && p->limit > 0 && ts > p->foits) || (p->order == 3 && p->limit > 0 && hi);
  a.recon = (p->order == 1) ? (ts > p->foits ? 1 : 0) : (ts > p->foits && !hi ? 1 : 0);
  a.gauss = (p->order == 3 && hi);
  a.jac = p->method != 0;
  a.steady_diag = 1;
  return a;
}

int check_params(flow_ctx* c, const flow_params* p) {
  if (!p) return FLOW_ERR_ARG;
  if (p->order != c->order) { set_error("params.order differs from the context's"); return FLOW_ERR_ARG; }
  if (p->method != 1) { set_error("only the implicit method (method=1) is supported"); return FLOW_ERR_ARG; }
  if (p->unsteady != 0 || p->tacc != 0) { set_error("only steady runs are supported"); return FLOW_ERR_ARG; }
  if (p->limit != 0 && p->limit != 2) { set_error("only limit=0 or limit=2 is supported"); return FLOW_ERR_ARG; }
  if (p->iter < 1 || p->jufreq < 1 || p->subits < 0) { set_error("bad iter/jufreq/subits"); return FLOW_ERR_ARG; }
  if (p->order == 3 && p->soits > 0 && !c->has_edge_w) {
    set_error("order 3 with soits > 0 needs the LSQ edge weights in the grid view");
    return FLOW_ERR_ARG;
  }
  return 0;
}

int grid_blocks(int n, int t) { return (n + t - 1) / t; }

cudaEvent_t get_event(flow_ctx* c) {
  if (!c->event_pool.empty()) {
    cudaEvent_t e = c->event_pool.back();
    c->event_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

// Brackets the launches of one kernel class with events when timing is on.
struct Timed {
  flow_ctx* c;
  int cls;
  int weight;  // launches of the class the bracket counts as
  cudaEvent_t a = nullptr;
  Timed(flow_ctx* ctx, int k, int w = 1) : c(ctx), cls(k), weight(w) {
    if (c->timing) {
      a = get_event(c);
      cudaEventRecord(a, c->stream);
    }
  }
  ~Timed() {
    if (c->timing) {
      cudaEvent_t b = get_event(c);
      cudaEventRecord(b, c->stream);
      c->pending.push_back({cls, a, b, weight});
    }
  }
};

// Accumulate finished event pairs (call after the stream was synchronised).
void harvest(flow_ctx* c) {
  for (auto& p : c->pending) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
      c->kms[p.cls] += ms;
      c->kcount[p.cls] += p.weight;
    }
    c->event_pool.push_back(p.a);
    c->event_pool.push_back(p.b);
  }
  c->pending.clear();
}

// Kernel variants the autotuner chooses between: minimum resident blocks per
// SM in __launch_bounds__ (which caps the registers per thread).
// k_node_prepare4: variant 0, 1, 2 -> 0 (compiler's choice), 10, 12 blocks.
// k_subedge_flux:  variant 0, 1, 2 -> 4, 5, 3 blocks.
constexpr int kVariants = 3;
// k_node_prepare4 has five more: variant 3 = k_node_stage (gathers staged in
// shared memory), where its shared memory fits the mesh; variant 4 =
// k_node_prepare16 (each node's chains split over 16 lanes); variants 5, 6
// and 7 = variants 0, 1 and 4 with the limiter fold that divides no zero
// and by no zero (venkat_fold_nz), variant 5 with the wave-speed face terms
// in the limiter's face loop too (LIM = 2; variants 6 and 7 LIM = 1).
constexpr int kNodeVariants = 8;
constexpr size_t kStageSmemMax = 110 * 1024;  // two CTAs per SM at most
template <class F>
void launch_variant(int v, F&& f) {
  if (v == 1) f(std::integral_constant<int, 10>());
  else if (v == 2) f(std::integral_constant<int, 12>());
  else f(std::integral_constant<int, 0>());
}
// node variants 5 and 6: (MINB, LIM) = (0, 2) and (10, 1)
template <class F>
void launch_lim_variant(int v, F&& f) {
  if (v == 6) f(std::integral_constant<int, 10>(), std::integral_constant<int, 1>());
  else f(std::integral_constant<int, 0>(), std::integral_constant<int, 2>());
}
template <class F>
void launch_flux_variant(int v, F&& f) {
  if (v == 1) f(std::integral_constant<int, 5>());
  else if (v == 2) f(std::integral_constant<int, 3>());
  else f(std::integral_constant<int, 4>());
}

int launch_node_prepare(flow_ctx* c, const StepArgs& a) {
  if (a.do_derivs && !c->has_stencils) {
    set_error("k=2 derivatives on the device need the stencils and SVD factors in the grid view");
    return FLOW_ERR_ARG;
  }
  Timed tm(c, 0);
  int nb = grid_blocks(4 * c->nn, 128);
  // the LSQ gradient (k=1, or the second-order start-up steps of k=2) is
  // the k=1 kernel's work
  const bool k1 = c->order == 1 || a.do_grad;
  if (c->var[0] == 4 || c->var[0] == 7) {
    const int nb16 = grid_blocks(16 * c->nn, 128);
    if (c->var[0] == 7) {
      if (k1) k_node_prepare16<1, 1><<<nb16, 128, 0, c->stream>>>(c->m, c->s, a);
      else k_node_prepare16<3, 1><<<nb16, 128, 0, c->stream>>>(c->m, c->s, a);
    } else {
      if (k1) k_node_prepare16<1><<<nb16, 128, 0, c->stream>>>(c->m, c->s, a);
      else k_node_prepare16<3><<<nb16, 128, 0, c->stream>>>(c->m, c->s, a);
    }
    return launch_check(c);
  }
  if (c->var[0] == 3 && c->stage_ok[k1 ? 0 : 1]) {
    const int tiles = grid_blocks(c->nn, kStageNodes);
    if (k1)
      k_node_stage<1><<<tiles, 128, stage_smem_bytes(1, c->stage_caps), c->stream>>>(
          c->m, c->s, a, c->stage_caps);
    else
      k_node_stage<3><<<tiles, 128, stage_smem_bytes(3, c->stage_caps), c->stream>>>(
          c->m, c->s, a, c->stage_caps);
    return launch_check(c);
  }
  if (c->var[0] >= 5) {
    if (k1)
      launch_lim_variant(c->var[0], [&](auto W, auto L) {
        k_node_prepare4<1, W.value, L.value><<<nb, 128, 0, c->stream>>>(c->m, c->s, a);
      });
    else
      launch_lim_variant(c->var[0], [&](auto W, auto L) {
        k_node_prepare4<3, W.value, L.value><<<nb, 128, 0, c->stream>>>(c->m, c->s, a);
      });
    return launch_check(c);
  }
  if (k1)
    launch_variant(c->var[0], [&](auto V) {
      k_node_prepare4<1, V.value><<<nb, 128, 0, c->stream>>>(c->m, c->s, a);
    });
  else
    launch_variant(c->var[0], [&](auto V) {
      k_node_prepare4<3, V.value><<<nb, 128, 0, c->stream>>>(c->m, c->s, a);
    });
  return launch_check(c);
}

int launch_residuals(flow_ctx* c, const StepArgs& a, int jac) {
  int rc = 0;
  if (jac && c->jac_mode == 1 && c->precision != 0 && c->fused_ok) {
    // approximate Jacobian: boundary faces first, then the interior faces
    // formed and summed by the nodes (k_faces_assemble)
    const int nbb = grid_blocks(c->nbe, 128);
    if (nbb > 0) {
      Timed t(c, 2);
      k_boundary<true><<<nbb, 128, 0, c->stream>>>(c->m, c->s, a);
      rc |= launch_check(c);
    }
    Timed t(c, 1);
    const int nb = grid_blocks(c->nn, kFusedNodes);
    const MixedTables& mt = c->mt;
    const ChunkTables& ct = c->ct;
    if (c->precision == 3) {
      if (a.recon == 1)
        k_faces_assemble<1, 2><<<nb, 128, kFusedSmem, c->stream>>>(c->m, c->s, a, mt, ct);
      else
        k_faces_assemble<0, 2><<<nb, 128, kFusedSmem, c->stream>>>(c->m, c->s, a, mt, ct);
    } else {
      if (a.recon == 1)
        k_faces_assemble<1, 1><<<nb, 128, kFusedSmem, c->stream>>>(c->m, c->s, a, mt, ct);
      else
        k_faces_assemble<0, 1><<<nb, 128, kFusedSmem, c->stream>>>(c->m, c->s, a, mt, ct);
    }
    rc |= launch_check(c);
    return rc;
  }
  // the approximate Roe Jacobian only in the precision form
  const bool approx = jac && c->jac_mode != 0 && c->precision != 0;
  {
    Timed t(c, 1);
    int nbs = grid_blocks(c->ns, 128);
    if (a.recon == 1) {
      launch_flux_variant(c->var[1], [&](auto V) {
        if (approx) k_subedge_flux<1, true, V.value, 1><<<nbs, 128, 0, c->stream>>>(c->m, c->s, a);
        else if (jac) k_subedge_flux<1, true, V.value><<<nbs, 128, 0, c->stream>>>(c->m, c->s, a);
        else k_subedge_flux<1, false, V.value><<<nbs, 128, 0, c->stream>>>(c->m, c->s, a);
      });
    } else {
      launch_flux_variant(c->var[1], [&](auto V) {
        if (approx) k_subedge_flux<0, true, V.value, 1><<<nbs, 128, 0, c->stream>>>(c->m, c->s, a);
        else if (jac) k_subedge_flux<0, true, V.value><<<nbs, 128, 0, c->stream>>>(c->m, c->s, a);
        else k_subedge_flux<0, false, V.value><<<nbs, 128, 0, c->stream>>>(c->m, c->s, a);
      });
    }
    rc |= launch_check(c);
  }
  int nbb = grid_blocks(c->nbe, 128);
  if (nbb > 0) {
    Timed t(c, 2);
    if (jac) k_boundary<true><<<nbb, 128, 0, c->stream>>>(c->m, c->s, a);
    else k_boundary<false><<<nbb, 128, 0, c->stream>>>(c->m, c->s, a);
    rc |= launch_check(c);
  }
  {
    Timed t(c, 3);
    int nbn = grid_blocks(4 * c->nn, 128);
    const MixedTables& mt = c->mt;
    const ChunkTables& ct = c->ct;
    if (c->precision == 3) {
      if (approx) k_assemble4<true, 2, true><<<nbn, 128, 0, c->stream>>>(c->m, c->s, a, mt, ct);
      else if (jac) k_assemble4<true, 2><<<nbn, 128, 0, c->stream>>>(c->m, c->s, a, mt, ct);
      else k_assemble4<false, 2><<<nbn, 128, 0, c->stream>>>(c->m, c->s, a, mt, ct);
    } else if (c->precision != 0) {
      if (approx) k_assemble4<true, 1, true><<<nbn, 128, 0, c->stream>>>(c->m, c->s, a, mt, ct);
      else if (jac) k_assemble4<true, 1><<<nbn, 128, 0, c->stream>>>(c->m, c->s, a, mt, ct);
      else k_assemble4<false, 1><<<nbn, 128, 0, c->stream>>>(c->m, c->s, a, mt, ct);
    } else {
      if (jac) k_assemble4<true, 0><<<nbn, 128, 0, c->stream>>>(c->m, c->s, a, mt, ct);
      else k_assemble4<false, 0><<<nbn, 128, 0, c->stream>>>(c->m, c->s, a, mt, ct);
    }
    rc |= launch_check(c);
  }
  return rc;
}

// linear_solve (linear_algebra.C:122-401): subits sweeps, alternating
// forward/backward, each followed by the b-Ax RMS that may stop the loop.
// Precision form: p->subits multicolour FP32 sweeps from dQ = 0, colours
// ascending on forward sweeps and descending on backward ones; no b-Ax RMS.
int launch_linear_solve_mixed(flow_ctx* c, const flow_params* p) {
  int rc = 0;
  cudaMemsetAsync(c->s.dQ, 0, sizeof(double) * 4 * (c->nn + 1), c->stream);
  cudaMemsetAsync(c->mt.dq32, 0, sizeof(float) * 4 * (c->nn + 1), c->stream);
  if (c->precision == 3) {
    // coloured chunks of the reference order, in-place FP32 iterate
    const ChunkTables& ct = c->ct;
    const size_t smem = 16 * kRecStride * kRingRecords + sizeof(float4) * ct.maxwin;
    if (c->sweep_pairs && !(c->sweep_df && ct.ring == 0) && p->subits > 1) {
      // the (sweep, colour) passes in order; where one sweep ends with the
      // colour the next begins with, the two passes are one launch
      std::vector<std::pair<int, int>> passes;
      for (int it = 0; it < p->subits; it++)
        for (int ci = 0; ci < ct.ncol; ci++)
          passes.push_back({it, it % 2 == 0 ? ci : ct.ncol - 1 - ci});
      Timed t(c, 4, p->subits);
      for (size_t k = 0; k < passes.size(); k++) {
        const int it = passes[k].first, col = passes[k].second, dir = it % 2;
        const int nb = c->h_col_ptr[col + 1] - c->h_col_ptr[col];
        const bool pair = k + 1 < passes.size() && passes[k + 1].second == col;
        const int last = (pair ? passes[k + 1].first : it) == p->subits - 1;
        if (pair) k++;
        if (nb <= 0) continue;
        if (pair) {
          auto kern = dir == 0 ? (ct.ring == 2 ? k_sweep_chunk_pair<0, 16>
                                  : ct.ring == 1 ? k_sweep_chunk_pair<0, 32>
                                                 : k_sweep_chunk_pair<0, 64>)
                               : (ct.ring == 2 ? k_sweep_chunk_pair<1, 16>
                                  : ct.ring == 1 ? k_sweep_chunk_pair<1, 32>
                                                 : k_sweep_chunk_pair<1, 64>);
          kern<<<nb, 256, smem, c->stream>>>(c->s, ct, c->mt.dq32, col, last);
        } else {
          auto kern = dir == 0 ? (ct.ring == 2 ? k_sweep_chunk<0, 16>
                                  : ct.ring == 1 ? k_sweep_chunk<0, 32> : k_sweep_chunk<0, 64>)
                               : (ct.ring == 2 ? k_sweep_chunk<1, 16>
                                  : ct.ring == 1 ? k_sweep_chunk<1, 32> : k_sweep_chunk<1, 64>);
          kern<<<nb, 256, smem, c->stream>>>(c->s, ct, c->mt.dq32, col, last);
        }
        rc |= launch_check(c);
      }
      return rc;
    }
    for (int it = 0; it < p->subits; it++) {
      Timed t(c, 4);
      const int last = it == p->subits - 1, dir = it % 2;
      if (c->sweep_df && ct.ring == 0) {
        // the whole sweep in one launch, one CTA per chunk
        const long max_spin = 1L << 22;
        if (dir == 0)
          k_sweep_chunk_df<0><<<ct.nchunks, 256, smem, c->stream>>>(c->s, ct, c->mt.dq32, last,
                                                                   max_spin);
        else
          k_sweep_chunk_df<1><<<ct.nchunks, 256, smem, c->stream>>>(c->s, ct, c->mt.dq32, last,
                                                                   max_spin);
        rc |= launch_check(c);
        continue;
      }
      for (int ci = 0; ci < ct.ncol; ci++) {
        const int col = dir == 0 ? ci : ct.ncol - 1 - ci;
        const int nb = c->h_col_ptr[col + 1] - c->h_col_ptr[col];
        if (nb <= 0) continue;
        auto kern = dir == 0 ? (ct.ring == 2 ? k_sweep_chunk<0, 16>
                                : ct.ring == 1 ? k_sweep_chunk<0, 32> : k_sweep_chunk<0, 64>)
                             : (ct.ring == 2 ? k_sweep_chunk<1, 16>
                                : ct.ring == 1 ? k_sweep_chunk<1, 32> : k_sweep_chunk<1, 64>);
        kern<<<nb, 256, smem, c->stream>>>(c->s, ct, c->mt.dq32, col, last);
        rc |= launch_check(c);
      }
    }
    return rc;
  }
  if (c->precision == 2) {
    // reference row order: dispenser sweeps on ping-pong FP32 iterates
    cudaMemsetAsync(c->s.skip, 0, sizeof(int), c->stream);
    const long max_spin = 1L << 21;
    for (int it = 0; it < p->subits; it++) {
      Timed t(c, 4);
      const int last = it == p->subits - 1;
      cudaMemsetAsync(c->s.counter, 0, sizeof(unsigned), c->stream);
      k_prepare_sweep32<<<grid_blocks(4 * (c->nn + 1), 256), 256, 0, c->stream>>>(
          c->s, c->mt.dq32, c->mt.dq32b, 4 * (c->nn + 1));
      rc |= launch_check(c);
      const int blocks = c->nsm * 4;
      if (it % 2 == 0)
        k_sweep_ordered32<true><<<blocks, 128, 0, c->stream>>>(c->s, c->mt, c->nn, c->mt.dq32,
                                                               c->mt.dq32b, last, max_spin);
      else
        k_sweep_ordered32<false><<<blocks, 128, 0, c->stream>>>(c->s, c->mt, c->nn, c->mt.dq32,
                                                                c->mt.dq32b, last, max_spin);
      rc |= launch_check(c);
      std::swap(c->mt.dq32, c->mt.dq32b);
    }
    return rc;
  }
  const int nc = c->mt.ncolors;
  for (int it = 0; it < p->subits; it++) {
    Timed t(c, 4);
    const bool last = it == p->subits - 1;
    for (int ci = 0; ci < nc; ci++) {
      const int col = (it % 2 == 0) ? ci : nc - 1 - ci;
      const int p0 = c->h_color_ptr[col], p1 = c->h_color_ptr[col + 1];
      const int nb = grid_blocks(4 * (p1 - p0), 128);
      if (nb == 0) continue;
      if (last) k_sweep_color32<true><<<nb, 128, 0, c->stream>>>(c->s, c->mt, p0, p1);
      else k_sweep_color32<false><<<nb, 128, 0, c->stream>>>(c->s, c->mt, p0, p1);
      rc |= launch_check(c);
    }
  }
  return rc;
}

int launch_linear_solve(flow_ctx* c, const flow_params* p, bool final_rms) {
  if (c->precision != 0) return launch_linear_solve_mixed(c, p);
  int rc = 0;
  cudaMemsetAsync(c->s.dQ, 0, sizeof(double) * 4 * (c->nn + 1), c->stream);
  cudaMemsetAsync(c->s.skip, 0, sizeof(int), c->stream);
  const long max_spin = 1L << 21;  // ~0.1-0.2 s per wait at most
  for (int it = 0; it < p->subits; it++) {
    cudaMemsetAsync(c->s.counter, 0, sizeof(unsigned), c->stream);
    {
      Timed t(c, 4);
      if (c->sweep_cta_ok && c->sweep_mode == 1) {
        const size_t sm = sizeof(SweepSmem);
        if (it % 2 == 0)
          k_sweep_cta<true><<<1, kSweepThreads, sm, c->stream>>>(c->m, c->s, c->sweep_tb, max_spin);
        else
          k_sweep_cta<false><<<1, kSweepThreads, sm, c->stream>>>(c->m, c->s, c->sweep_tb, max_spin);
        rc |= launch_check(c);
      } else {
        // results go to the other dQ buffer, pre-filled with the not-ready
        // pattern; the buffers swap roles afterwards
        double* dq_new = c->s.dQ2;
        k_prepare_sweep<<<grid_blocks(4 * (c->nn + 1), 256), 256, 0, c->stream>>>(
            c->s, c->s.dQ, dq_new, 4 * (c->nn + 1));
        rc |= launch_check(c);
        int blocks = c->nsm * 4;
        if (it % 2 == 0)
          k_sweep_ordered<true><<<blocks, 128, 0, c->stream>>>(c->m, c->s, c->s.dQ, dq_new, max_spin);
        else
          k_sweep_ordered<false><<<blocks, 128, 0, c->stream>>>(c->m, c->s, c->s.dQ, dq_new, max_spin);
        rc |= launch_check(c);
        std::swap(c->s.dQ, c->s.dQ2);
      }
    }
    if (it < p->subits - 1 || final_rms) {
      Timed t(c, 5);
      k_lin_residual<<<kRedBlocks, kRedThreads, 0, c->stream>>>(c->m, c->s);
      rc |= launch_check(c);
      k_finalize_rms<<<1, kRedThreads, 0, c->stream>>>(c->s, kRedBlocks, c->nn,
                                                       c->exact_rms);
      rc |= launch_check(c);
      k_exact_rms<<<1, 256, 0, c->stream>>>(c->m, c->s);
      rc |= launch_check(c);
    }
  }
  return rc;
}

// Gauss-Seidel sweeps of step ts: the schedule's count up to its last step,
// the parameters' count after.
int sweeps_at(const flow_ctx* c, const flow_params* p, int ts) {
  if (c->sched_sweeps > 0) {
    const int until = c->sched_until > 0 ? c->sched_until : p->ramp;
    if (ts <= until) return c->sched_sweeps;
  }
  return p->subits;
}

// Step index and CFL on the device (k_step_args): citer > 0 sets the index,
// 0 advances the device's own.
int launch_step_args(flow_ctx* c, const flow_params* p, int citer) {
  k_step_args<<<1, 1, 0, c->stream>>>(c->s, citer, p->method, p->ramp, p->CFL);
  return launch_check(c);
}

// What k_begin_step clears at the start of a step (solve.C:298-348: grad and
// hess <- 0, phi <- 1), less what the step's node kernel then writes for
// every node: phi when the limiter runs, the k=2 derivatives when they are
// formed, the gradient when it is formed.  The gradient is cleared on steps
// that do not form it only where some step of the run, or the caller
// (flow_set "grad"), writes it; otherwise it keeps the zeros it was created
// with.
int begin_flags(const flow_ctx* c, const flow_params* p, const StepArgs& a) {
  int f = 0;
  if (!a.do_lim) f |= kBeginResetPhi;
  if (c->order == 3 && !a.do_derivs) f |= kBeginZeroHess;
  if (!a.do_grad && (c->order == 1 || p->soits > 0 || c->grad_written)) f |= kBeginZeroGrad;
  return f;
}

// One solve() call (solve.C:44-933), device-only.  device_ts: the step index
// advances on the device (for captured chunks of steps; ts then only selects
// the order phase, which must be the same for every step of the chunk) and
// the run's first step is recognised on the device.
int enqueue_step(flow_ctx* c, const flow_params* p, int ts, int hist_slot, int first,
                 bool device_ts = false) {
  int rc = 0;
  int total = c->nn + c->ng;
  c->citer = ts;
  if (device_ts) first = -1;
  StepArgs a = make_args(p, ts);
  const int clear = begin_flags(c, p, a);
  // the step index and CFL (k_step_args) by the first thread of the step's
  // first kernel
  k_begin_step<<<grid_blocks(total, 256), 256, 0, c->stream>>>(
      c->m, c->s, kBeginCopyQ | kBeginStepArgs | clear, device_ts ? 0 : ts, p->method, p->ramp,
      p->CFL);
  rc |= launch_check(c);
  for (int mi = 1; mi <= p->iter; mi++) {
    int jac = ((mi - 1) % p->jufreq == 0) || mi == 1;
    if (mi > 1) {
      // phi <- 1 at every Newton iteration (solve.C:344-348)
      k_begin_step<<<grid_blocks(total, 256), 256, 0, c->stream>>>(c->m, c->s, clear);
      rc |= launch_check(c);
    }
    rc |= launch_node_prepare(c, a);
    rc |= launch_residuals(c, a, jac);
    flow_params pe = *p;  // the sweep schedule may lower the sweep count early on
    pe.subits = sweeps_at(c, p, ts);
    rc |= launch_linear_solve(c, &pe, false);
    const bool last = mi == p->iter;
    k_finish_step<<<kRedBlocks, kRedThreads, 0, c->stream>>>(
        c->m, c->s, last, last && hist_slot >= 0 ? c->d_hist : nullptr,
        last && hist_slot >= 0 ? c->d_hist + c->hist_cap : nullptr, hist_slot < 0 ? 0 : hist_slot,
        last ? (first < 0 ? -1 : first) : 0);
    rc |= launch_check(c);
  }
  return rc;
}

bool params_equal(const flow_params& a, const flow_params& b) {
  return a.iter == b.iter && a.jufreq == b.jufreq && a.CFL == b.CFL && a.ramp == b.ramp &&
         a.gamma == b.gamma && a.alpha == b.alpha && a.mach == b.mach && a.subits == b.subits &&
         a.method == b.method && a.order == b.order && a.foits == b.foits && a.soits == b.soits &&
         a.limit == b.limit && a.unsteady == b.unsteady && a.tacc == b.tacc;
}

// Order-phase signature of step ts (which reconstruction/limiter passes run).
int phase_of(const flow_params* p, int ts) {
  StepArgs a = make_args(p, ts);
  return a.do_grad | (a.do_derivs << 1) | (a.do_lim << 2) | (a.recon << 3) | (a.gauss << 6);
}

void drop_graphs(flow_ctx* c) {
  for (auto& g : c->graphs)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  c->graphs.clear();
}

// K steps ts0 .. ts0+K-1 with the step index advancing on the device,
// replayed from a captured CUDA graph when the chunk allows it (one order
// phase throughout; the FP64 ordered sweep's buffer swaps return to their
// start; no per-kernel timing), else launched one by one.
int enqueue_chunk(flow_ctx* c, const flow_params* p, int ts0, int K) {
  int rc = 0;
  const int ph = phase_of(p, ts0);
  const int sw = sweeps_at(c, p, ts0);
  const bool graphable = c->use_graphs && !c->timing && K > 0 && ph == phase_of(p, ts0 + K - 1) &&
                         sw == sweeps_at(c, p, ts0 + K - 1) &&
                         (c->precision == 1 || c->precision == 3 ||
                          (c->precision == 0 && c->sweep_mode == 1) ||
                          p->subits % 2 == 0);
  if (!graphable) {
    for (int i = 0; i < K && !rc; i++) rc |= enqueue_step(c, p, ts0 + i, -1, -1, true);
    return rc;
  }
  flow_ctx::ChunkGraph* g = nullptr;
  for (auto& x : c->graphs)
    if (x.K == K && x.precision == c->precision && x.sweep_mode == c->sweep_mode &&
        x.phase == ph && x.sweeps == sw && params_equal(x.p, *p))
      g = &x;
  if (!g) {
    if (c->graphs.size() >= 4) drop_graphs(c);
    flow_ctx::ChunkGraph ng;
    ng.K = K;
    ng.precision = c->precision;
    ng.sweep_mode = c->sweep_mode;
    ng.phase = ph;
    ng.sweeps = sw;
    ng.p = *p;
    const long l0 = c->launches;
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaSuccess;
    {
      // no device-wide call of this library runs while the capture is open
      std::shared_lock<std::shared_mutex> gate(g_device_gate);
      e = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal);
      if (e == cudaSuccess) {
        for (int i = 0; i < K; i++) rc |= enqueue_step(c, p, ts0 + i, -1, -1, true);
        e = cudaStreamEndCapture(c->stream, &graph);
      }
    }
    if (e == cudaSuccess && !rc && graph) {
      e = cudaGraphInstantiate(&ng.exec, graph, 0);
      if (e != cudaSuccess) ng.exec = nullptr;
    }
    if (graph) cudaGraphDestroy(graph);
    const bool faulted = c->capture_fault > 0;
    if (faulted && ng.exec) {
      cudaGraphExecDestroy(ng.exec);  // a discarded capture (flow_set_capture_fault)
      ng.exec = nullptr;
    }
    if (faulted) c->capture_fault--;
    if (rc || e != cudaSuccess || !ng.exec) {
      // The capture was invalidated (a device-wide call outside this library,
      // from another thread) or could not be instantiated.  Nothing of it ran:
      // launch the chunk eagerly, which does the same work.  A stream that is
      // somehow still capturing, or an eager launch that fails, is an error.
      cudaGetLastError();
      c->launches = l0;
      c->capture_fallbacks++;
      cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
      if (cudaStreamIsCapturing(c->stream, &cs) != cudaSuccess ||
          cs != cudaStreamCaptureStatusNone) {
        set_error("step capture failed and the stream is still capturing");
        return FLOW_ERR_CUDA;
      }
      rc = 0;
      for (int i = 0; i < K && !rc; i++) rc |= enqueue_step(c, p, ts0 + i, -1, -1, true);
      return rc;
    }
    ng.launches = c->launches - l0;
    c->launches = l0;
    c->graphs.push_back(ng);
    g = &c->graphs.back();
  }
  if (cudaGraphLaunch(g->exec, c->stream) != cudaSuccess) {
    set_error("graph launch failed");
    return FLOW_ERR_CUDA;
  }
  c->launches += g->launches;
  c->citer = ts0 + K - 1;
  return 0;
}

// Clear the convergence stop and set the run's target drop (0 = none).
void reset_run(flow_ctx* c, double drop) {
  c->drop_target = drop;
  cudaMemsetAsync(c->s.stop, 0, sizeof(int), c->stream);
  cudaMemsetAsync(c->s.steps_done, 0, sizeof(int), c->stream);
  cudaMemcpyAsync(c->s.scalars + 7, &c->drop_target, sizeof(double), cudaMemcpyHostToDevice,
                  c->stream);
}

int read_status(flow_ctx* c) {
  int st = 0;
  if (cudaMemcpyAsync(&st, c->s.status, sizeof(int), cudaMemcpyDeviceToHost, c->stream) !=
      cudaSuccess)
    return FLOW_ERR_CUDA;
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) {
    set_error(cudaGetErrorString(cudaGetLastError()));
    return FLOW_ERR_CUDA;
  }
  harvest(c);
  return st;
}

// Colour the block pattern greedily in row order (each row takes the
// smallest colour none of its earlier neighbours holds) and lay out the FP32
// tables of the precision form in colour order.
int build_mixed_tables(flow_ctx* c, bool ordered) {
  if (c->mt.lhs32 && c->mt_ordered == ordered) return 0;
  const int nn = c->nn;
  const std::vector<int>& ia = c->h_ia;
  const std::vector<int>& ja = c->h_ja;
  std::vector<int> color(nn + 1, 0);
  int ncol = 0;
  std::vector<char> used;
  for (int j = 1; j <= nn; j++) {
    if (ia[j + 1] <= ia[j] || ja[ia[j + 1] - 1] != j) {
      set_error("precision form: a row's diagonal block is not its last block");
      return FLOW_ERR_ARG;
    }
    used.assign(ncol + 1, 0);
    for (int k = ia[j]; k < ia[j + 1]; k++)
      if (ja[k] < j) used[color[ja[k]]] = 1;
    int col = 0;
    while (!ordered && used[col]) col++;  // ordered: one class, rows in reference order
    color[j] = col;
    ncol = std::max(ncol, col + 1);
  }
  std::vector<int> cptr(ncol + 1, 0), rows(nn), pos(nn + 1, 0), optr(nn + 1, 0), ocol;
  for (int j = 1; j <= nn; j++) cptr[color[j] + 1]++;
  for (int q = 0; q < ncol; q++) cptr[q + 1] += cptr[q];
  std::vector<int> fill(cptr.begin(), cptr.end() - 1);
  for (int j = 1; j <= nn; j++) {
    int pp = fill[color[j]]++;
    rows[pp] = j;
    pos[j] = pp;
  }
  ocol.reserve(ja.size());
  for (int pp = 0; pp < nn; pp++) {
    int j = rows[pp];
    optr[pp] = (int)ocol.size();
    for (int k = ia[j]; k < ia[j + 1] - 1; k++) ocol.push_back(ja[k]);
  }
  optr[nn] = (int)ocol.size();
  MixedTables& mt = c->mt;
  mt.ncolors = ncol;
  mt.color_ptr = upload_vec(c, cptr);
  mt.rows = upload_vec(c, rows);
  mt.pos = upload_vec(c, pos);
  mt.offd_ptr = upload_vec(c, optr);
  mt.offd_col = upload_vec(c, ocol);
  std::vector<int4> rinfo(nn);
  for (int pp = 0; pp < nn; pp++) rinfo[pp] = make_int4(rows[pp], optr[pp], optr[pp + 1], 0);
  mt.rowinfo = upload_vec(c, rinfo);
  mt.lu32 = c->buf.alloc<float>((size_t)16 * nn);
  if (!mt.dq32) mt.dq32 = c->buf.alloc<float>((size_t)4 * (nn + 1));
  if (!mt.dq32b) mt.dq32b = c->buf.alloc<float>((size_t)4 * (nn + 1));
  mt.lhs32 = c->buf.alloc<float>((size_t)16 * std::max<size_t>(ocol.size(), 1));
  if (!mt.color_ptr || !mt.rows || !mt.pos || !mt.offd_ptr || !mt.offd_col || !mt.rowinfo || !mt.lu32 ||
      !mt.dq32 || !mt.dq32b || !mt.lhs32) {
    set_error("precision form: device allocation or upload failed");
    mt.lhs32 = nullptr;
    return carve_error(c);
  }
  if (cudaMemsetAsync(mt.dq32, 0, sizeof(float) * 4 * (nn + 1), c->stream) != cudaSuccess ||
      cudaMemsetAsync(mt.dq32b, 0, sizeof(float) * 4 * (nn + 1), c->stream) != cudaSuccess) {
    set_error("precision form: clearing the FP32 iterates failed");
    mt.lhs32 = nullptr;
    return FLOW_ERR_CUDA;
  }
  c->h_color_ptr = cptr;
  c->mt_ordered = ordered;
  return 0;
}

// Kernel attributes belong to the process and device, not to a context: they
// are set once per device, by the first context that needs them, so that a
// context built while other solves run never changes a kernel that is in
// flight.  The shared-memory caps are the largest any context may use.
//
// The same first call loads every kernel of the step into the device's
// context (cudaFuncGetAttributes forces CUDA's lazy module loading).  Loading
// a module may synchronise the device, so it must not happen at a kernel's
// first launch while another thread captures a chunk of steps into a graph.
bool preload_kernels() {
  cudaFuncAttributes fa;
  bool ok = true;
  for (const void* f :
       {(const void*)k_step_args, (const void*)k_begin_step,
        (const void*)k_node_prepare4<1, 0>, (const void*)k_node_prepare4<1, 10>,
        (const void*)k_node_prepare4<1, 12>, (const void*)k_node_prepare4<3, 0>,
        (const void*)k_node_prepare4<3, 10>, (const void*)k_node_prepare4<3, 12>,
        (const void*)k_node_prepare4<1, 0, 2>, (const void*)k_node_prepare4<1, 10, 1>,
        (const void*)k_node_prepare4<3, 0, 2>, (const void*)k_node_prepare4<3, 10, 1>,
        (const void*)k_assemble4<true, 0>, (const void*)k_assemble4<false, 0>,
        (const void*)k_assemble4<true, 1>, (const void*)k_assemble4<false, 1>,
        (const void*)k_assemble4<true, 2>, (const void*)k_assemble4<false, 2>,
        (const void*)k_assemble4<true, 1, true>, (const void*)k_assemble4<true, 2, true>,
        (const void*)k_boundary_add4<true>, (const void*)k_boundary_add4<false>,
        (const void*)k_node_stage<1>, (const void*)k_node_stage<3>,
        (const void*)k_node_prepare16<1>, (const void*)k_node_prepare16<3>,
        (const void*)k_node_prepare16<1, 1>, (const void*)k_node_prepare16<3, 1>,
        (const void*)k_faces_assemble<0, 1>, (const void*)k_faces_assemble<1, 1>,
        (const void*)k_faces_assemble<0, 2>, (const void*)k_faces_assemble<1, 2>,
        (const void*)k_diag_lu,
        (const void*)k_subedge_flux<0, true, 3>, (const void*)k_subedge_flux<0, true, 4>,
        (const void*)k_subedge_flux<0, true, 5>, (const void*)k_subedge_flux<0, false, 3>,
        (const void*)k_subedge_flux<0, false, 4>, (const void*)k_subedge_flux<0, false, 5>,
        (const void*)k_subedge_flux<1, true, 3>, (const void*)k_subedge_flux<1, true, 4>,
        (const void*)k_subedge_flux<1, true, 5>, (const void*)k_subedge_flux<1, false, 3>,
        (const void*)k_subedge_flux<1, false, 4>, (const void*)k_subedge_flux<1, false, 5>,
        (const void*)k_subedge_flux<0, true, 3, 1>, (const void*)k_subedge_flux<0, true, 4, 1>,
        (const void*)k_subedge_flux<0, true, 5, 1>, (const void*)k_subedge_flux<1, true, 3, 1>,
        (const void*)k_subedge_flux<1, true, 4, 1>, (const void*)k_subedge_flux<1, true, 5, 1>,
        (const void*)k_boundary<true>, (const void*)k_boundary<false>,
        (const void*)k_diag_only, (const void*)k_sweep_ordered<true>,
        (const void*)k_sweep_ordered<false>, (const void*)k_sweep_color32<true>,
        (const void*)k_sweep_color32<false>, (const void*)k_sweep_ordered32<true>,
        (const void*)k_sweep_ordered32<false>, (const void*)k_prepare_sweep32,
        (const void*)k_fill_sweep_records, (const void*)k_prepare_sweep,
        (const void*)k_lin_residual, (const void*)k_finalize_rms, (const void*)k_exact_rms,
        (const void*)k_finish_step,
        (const void*)k_body_forces,
        (const void*)k_body_forces_sum})
    ok = ok && cudaFuncGetAttributes(&fa, f) == cudaSuccess;
  return ok;
}

bool ensure_kernel_attrs(int device) {
  static std::mutex mu;
  static std::vector<char> done;
  std::lock_guard<std::mutex> lock(mu);
  if (device < 0) return false;
  if ((int)done.size() <= device) done.resize(device + 1, 0);
  if (done[device]) return true;
  DeviceWide gate(g_device_gate);
  const int chunk_cap = 227 * 1024 - kChunkStaticSmem;
  const int cta = (int)sizeof(SweepSmem);
  bool ok = preload_kernels();
  for (const void* f : {(const void*)k_sweep_chunk_pair<0, 64>, (const void*)k_sweep_chunk_pair<1, 64>,
                        (const void*)k_sweep_chunk_pair<0, 32>, (const void*)k_sweep_chunk_pair<1, 32>,
                        (const void*)k_sweep_chunk_pair<0, 16>, (const void*)k_sweep_chunk_pair<1, 16>,
                        (const void*)k_sweep_chunk_df<0>, (const void*)k_sweep_chunk_df<1>,
                        (const void*)k_sweep_chunk<0, 64>, (const void*)k_sweep_chunk<1, 64>,
                        (const void*)k_sweep_chunk<0, 32>, (const void*)k_sweep_chunk<1, 32>,
                        (const void*)k_sweep_chunk<0, 16>, (const void*)k_sweep_chunk<1, 16>})
    ok = ok && cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    chunk_cap) == cudaSuccess;
  for (const void* f : {(const void*)k_node_stage<1>, (const void*)k_node_stage<3>})
    ok = ok && cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)kStageSmemMax) == cudaSuccess;
  for (const void* f : {(const void*)k_faces_assemble<0, 1>, (const void*)k_faces_assemble<1, 1>,
                        (const void*)k_faces_assemble<0, 2>, (const void*)k_faces_assemble<1, 2>})
    ok = ok && cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)kFusedSmem) == cudaSuccess;
  for (const void* f : {(const void*)k_sweep_cta<true>, (const void*)k_sweep_cta<false>})
    ok = ok && cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, cta) ==
                   cudaSuccess;
  if (ok) done[device] = 1;
  return ok;
}

// Mode 3 reads none of the mode 1 / 2 tables: only the FP32 iterate.
int build_chunk_iterate(flow_ctx* c) {
  MixedTables& mt = c->mt;
  const size_t n = (size_t)4 * (c->nn + 1);
  if (!mt.dq32) mt.dq32 = c->buf.alloc<float>(n);
  if (!mt.dq32b) mt.dq32b = c->buf.alloc<float>(n);
  if (!mt.dq32 || !mt.dq32b) {
    set_error("precision form: device allocation failed");
    return carve_error(c);
  }
  if (cudaMemsetAsync(mt.dq32, 0, sizeof(float) * n, c->stream) != cudaSuccess ||
      cudaMemsetAsync(mt.dq32b, 0, sizeof(float) * n, c->stream) != cudaSuccess) {
    set_error("precision form: clearing the FP32 iterates failed");
    return FLOW_ERR_CUDA;
  }
  return 0;
}

// Mode 3 tables.  Chunks: consecutive rows of the reference order, closed
// when the next row would exceed the row limit (default twice the matrix
// bandwidth, at most 2048) or the level limit (default 32; a row's level is
// one more than that of its latest in-chunk neighbour upstream, and the
// longest chain is the same in both directions).  Colours: each chunk takes
// the smallest colour no earlier adjacent chunk holds.  Records: per
// direction, chunk by chunk, sub-levels of at most kRecRows rows of one
// level, rows ascending inside a sub-level.
int build_chunks_with(flow_ctx* c, int bw, int cmax, int lmax);

int build_chunk_tables(flow_ctx* c) {
  const int nn = c->nn;
  const std::vector<int>& ia = c->h_ia;
  const std::vector<int>& ja = c->h_ja;
  int bw = 1;
  for (int j = 1; j <= nn; j++) {
    if (ia[j + 1] <= ia[j] || ja[ia[j + 1] - 1] != j) {
      set_error("precision form: a row's diagonal block is not its last block");
      return FLOW_ERR_ARG;
    }
    if (ia[j + 1] - ia[j] - 1 > kRecBlocks) {
      set_error("precision mode 3: a row has more than 8 off-diagonal blocks");
      return FLOW_ERR_ARG;
    }
    for (int k = ia[j]; k < ia[j + 1]; k++) bw = std::max(bw, std::abs(ja[k] - j));
  }
  int cmax = c->chunk_rows > 0 ? c->chunk_rows
                               : std::min(2048, std::max(64, ((2 * bw + 63) / 64) * 64));
  const int lmax = c->chunk_levels > 0 ? c->chunk_levels : 32;
  // an automatic chunk size shrinks (64 rows at a time) until every chunk's
  // window of the iterate fits in shared memory beside the record ring
  for (;;) {
    const int rc = build_chunks_with(c, bw, cmax, lmax);
    if (rc != FLOW_ERR_ARG || c->chunk_rows > 0 || cmax - 64 < std::max(64, bw / 2)) return rc;
    cmax -= 64;
  }
}

// Point the chunk tables at the sub-levels of the requested ring shape (the
// largest shape when the requested one does not fit a chunk).
void apply_ring(flow_ctx* c) {
  const int shape = c->ring_ok[c->ring] ? c->ring : 0;
  for (int dir = 0; dir < 2; dir++) {
    c->ct.sub_start[dir] = c->ring_sub_start[shape][dir];
    c->ct.chunk_sub[dir] = c->ring_chunk_sub[shape][dir];
  }
  c->ct.ring = shape;
}

int build_chunks_with(flow_ctx* c, int bw, int cmax, int lmax) {
  for (int shape = 0; shape < kRingShapes; shape++) c->ring_ok[shape] = true;
  const int nn = c->nn;
  const std::vector<int>& ia = c->h_ia;
  const std::vector<int>& ja = c->h_ja;
  // chunks
  std::vector<int> start, lev(nn + 1, 0), chunk_of(nn + 1, 0);
  start.push_back(1);
  for (int j = 1; j <= nn; j++) {
    int lo = start.back();
    int l = 0;
    for (int k = ia[j]; k < ia[j + 1]; k++)
      if (ja[k] >= lo && ja[k] < j) l = std::max(l, lev[ja[k]] + 1);
    if (j - lo + 1 > cmax || l + 1 > lmax) {
      start.push_back(j);
      l = 0;
    }
    lev[j] = l;
    chunk_of[j] = (int)start.size() - 1;
  }
  const int nch = (int)start.size();
  start.push_back(nn + 1);
  // colours
  std::vector<int> colour(nch, 0);
  int ncol = 1;
  std::vector<char> used;
  for (int q = 0; q < nch; q++) {
    used.assign(ncol + 1, 0);
    for (int j = start[q]; j < start[q + 1]; j++)
      for (int k = ia[j]; k < ia[j + 1]; k++) {
        const int o = chunk_of[ja[k]];
        if (o < q) used[colour[o]] = 1;
      }
    int col = 0;
    while (used[col]) col++;
    colour[q] = col;
    ncol = std::max(ncol, col + 1);
  }
  std::vector<int> cptr(ncol + 1, 0), clist;
  for (int q = 0; q < nch; q++) cptr[colour[q] + 1]++;
  for (int k = 0; k < ncol; k++) cptr[k + 1] += cptr[k];
  clist.assign(nch, 0);
  {
    std::vector<int> fill(cptr.begin(), cptr.end() - 1);
    for (int q = 0; q < nch; q++) clist[fill[colour[q]]++] = q;
  }
  // windows
  std::vector<int2> win(nch);
  int maxwin = 0;
  for (int q = 0; q < nch; q++) {
    int a = start[q], b = start[q + 1] - 1;
    for (int j = start[q]; j < start[q + 1]; j++)
      for (int k = ia[j]; k < ia[j + 1]; k++) {
        a = std::min(a, ja[k]);
        b = std::max(b, ja[k]);
      }
    win[q] = make_int2(a, b);
    maxwin = std::max(maxwin, b - a + 1);
  }
  const size_t smem = 16 * kRecStride * kRingRecords + sizeof(float4) * maxwin;
  if (smem + kChunkStaticSmem > 227 * 1024) {
    set_error("precision mode 3: a chunk's window does not fit in shared memory (bandwidth too large)");
    return FLOW_ERR_ARG;
  }
  ChunkTables& ct = c->ct;
  ct.nchunks = nch;
  ct.ncol = ncol;
  ct.maxwin = maxwin;
  ct.col_ptr = upload_vec(c, cptr);
  ct.col_chunks = upload_vec(c, clist);
  ct.window = upload_vec(c, win);
  {
    // one-launch sweeps: dispensing order per direction (colours ascending
    // forward, descending backward), each chunk's colour, the chunks its
    // window overlaps, and zeroed flags and counters
    std::vector<int> order_f, order_b, nbr_x(nch), nbr_y(nch);
    for (int k = 0; k < ncol; k++)
      for (int t = cptr[k]; t < cptr[k + 1]; t++) order_f.push_back(clist[t]);
    for (int k = ncol - 1; k >= 0; k--)
      for (int t = cptr[k]; t < cptr[k + 1]; t++) order_b.push_back(clist[t]);
    std::vector<int2> nbr(nch);
    for (int q = 0; q < nch; q++) nbr[q] = make_int2(chunk_of[win[q].x], chunk_of[win[q].y]);
    ct.task_chunk[0] = upload_vec(c, order_f);
    ct.task_chunk[1] = upload_vec(c, order_b);
    ct.colour = upload_vec(c, colour);
    ct.nbr = upload_vec(c, nbr);
    ct.done = c->buf.alloc<int>(nch);
    ct.sync = c->buf.alloc<unsigned>(4);
    if (!ct.task_chunk[0] || !ct.task_chunk[1] || !ct.colour || !ct.nbr || !ct.done || !ct.sync) {
      set_error("precision mode 3: table allocation or upload failed");
      return carve_error(c);
    }
    if (cudaMemsetAsync(ct.done, 0, sizeof(int) * nch, c->stream) != cudaSuccess ||
        cudaMemsetAsync(ct.sync, 0, sizeof(unsigned) * 4, c->stream) != cudaSuccess) {
      set_error("precision mode 3: clearing the sweep counters failed");
      return FLOW_ERR_CUDA;
    }
  }
  // per direction: levels, sub-levels, records (static part)
  std::vector<int> levd(nn + 1);
  for (int dir = 0; dir < 2; dir++) {
    std::vector<int> pos(nn + 1, 0), order, lev_start, chunk_lev(nch + 1, 0);
    order.reserve(nn);
    for (int q = 0; q < nch; q++) {
      const int lo = start[q], hi = start[q + 1] - 1;
      int nlev = 0;
      for (int t = 0; t <= hi - lo; t++) {
        const int j = dir == 0 ? lo + t : hi - t;
        int l = 0;
        for (int k = ia[j]; k < ia[j + 1]; k++) {
          const int o = ja[k];
          const bool up = dir == 0 ? (o >= lo && o < j) : (o <= hi && o > j);
          if (up) l = std::max(l, levd[o] + 1);
        }
        levd[j] = l;
        nlev = std::max(nlev, l + 1);
      }
      for (int l = 0; l < nlev; l++) {
        lev_start.push_back((int)order.size());
        for (int j = lo; j <= hi; j++) {
          if (levd[j] != l) continue;
          pos[j] = (int)order.size();
          order.push_back(j);
        }
      }
      chunk_lev[q + 1] = (int)lev_start.size();
    }
    lev_start.push_back((int)order.size());
    // sub-levels of each ring shape: every level cut into runs of at most
    // ring_rows(shape) rows (rows of one level are independent, so the cut
    // changes the barriers, not the arithmetic)
    for (int shape = 0; shape < kRingShapes; shape++) {
      const int rows = ring_rows(shape);
      std::vector<int> ss, cs(nch + 1, 0);
      bool fits = true;
      for (int q = 0; q < nch; q++) {
        cs[q] = (int)ss.size();
        for (int L = chunk_lev[q]; L < chunk_lev[q + 1]; L++)
          for (int x = lev_start[L]; x < lev_start[L + 1]; x += rows) ss.push_back(x);
        if ((int)ss.size() - cs[q] > kChunkSubMax) fits = false;
      }
      cs[nch] = (int)ss.size();
      ss.push_back((int)order.size());
      if (!fits) {
        if (shape == 0) {
          set_error("precision mode 3: a chunk has more sub-levels than the sweep kernel holds");
          return FLOW_ERR_ARG;
        }
        c->ring_ok[shape] = false;
        continue;
      }
      c->ring_sub_start[shape][dir] = upload_vec(c, ss);
      c->ring_chunk_sub[shape][dir] = upload_vec(c, cs);
      if (!c->ring_sub_start[shape][dir] || !c->ring_chunk_sub[shape][dir]) {
        set_error("precision mode 3: table allocation or upload failed");
        return carve_error(c);
      }
    }
    // the records' static part is written on the device from the resident
    // block pattern: only the order (4 bytes a row) crosses from the host
    SweepRec* rec = c->buf.alloc<SweepRec>(nn);
    const int* d_order = upload_vec(c, order);
    if (rec && d_order) {
      const long words = (long)nn * kRecInts;
      k_fill_sweep_records<<<(unsigned)((words + 255) / 256), 256, 0, c->stream>>>(
          rec, d_order, nn, c->m.ia, c->m.ja);
      if (cudaGetLastError() != cudaSuccess) rec = nullptr;
    }
    ct.rec[dir] = rec;
    ct.pos[dir] = upload_vec(c, pos);
    if (!ct.rec[dir] || !ct.pos[dir]) {
      set_error("precision mode 3: table allocation or upload failed");
      return carve_error(c);
    }
  }
  if (!ct.col_ptr || !ct.col_chunks || !ct.window) {
    set_error("precision mode 3: table allocation or upload failed");
    return carve_error(c);
  }
  if (!ensure_kernel_attrs(c->device)) {
    set_error("precision mode 3: cannot reserve shared memory for the sweep");
    return FLOW_ERR_CUDA;
  }
  apply_ring(c);
  c->h_col_ptr = cptr;
  c->h_chunk_start = start;
  return 0;
}

int ensure_hist(flow_ctx* c, int n) {
  if (n <= c->hist_cap) return 0;
  n = std::max(n, 64);
  double* h = c->buf.alloc<double>((size_t)2 * n);  // the old block stays with the context
  if (!h) {
    set_error("history allocation failed");
    return carve_error(c);
  }
  c->d_hist = h;
  c->hist_cap = n;
  return 0;
}

}  // namespace

// ===========================================================================
extern "C" {

const char* flow_last_error(void) { return g_last_error.c_str(); }

static flow_ctx* create_impl(flow_arena* arena, const flow_grid_view* g, const flow_params* p,
                             int device, int* status);

flow_ctx* flow_create(const flow_grid_view* g, const flow_params* p, int device, int* status) {
  return create_impl(nullptr, g, p, device, status);
}

flow_ctx* flow_create_in(flow_arena* arena, const flow_grid_view* g, const flow_params* p,
                         int* status) {
  if (!arena) {
    set_error("null arena");
    if (status) *status = FLOW_ERR_ARG;
    return nullptr;
  }
  return create_impl(arena, g, p, arena->device, status);
}

static flow_ctx* create_impl(flow_arena* arena, const flow_grid_view* g, const flow_params* p,
                             int device, int* status) {
  auto fail = [&](flow_ctx* c, int code, const char* msg) -> flow_ctx* {
    set_error(msg);
    if (status) *status = code;
    if (c) flow_destroy(c);
    return nullptr;
  };
  if (!g || !p) return fail(nullptr, FLOW_ERR_ARG, "null grid or params");
  if (p->order != 1 && p->order != 3) return fail(nullptr, FLOW_ERR_ARG, "order must be 1 or 3");
  const int nn = g->nn, ng = g->nn_ghost, ne = g->nedges, ns = g->nsubedges, nbe = g->nbedges;
  if (nn < 1 || ne < 1 || ns < 1 || !g->edges || !g->subedges || !g->ia || !g->ja || !g->iau ||
      !g->x || !g->cv_area || !g->xn_subedges || !g->bedges || !g->bbc || !g->node_order)
    return fail(nullptr, FLOW_ERR_ARG, "incomplete grid view");
  if (p->order == 1 && !g->edge_weight) return fail(nullptr, FLOW_ERR_ARG, "order 1 needs edge_weight");
  // order 3: the stencils and SVD factors may be left out (all NULL) by a
  // caller that forms the k=2 derivatives itself (the stage entry points);
  // device steps of the k=2 scheme then refuse
  const bool any_st = g->gnsn || g->gnnsn || g->gnnsn1 || g->svd_m || g->svd_off || g->svd_U ||
                      g->svd_VT || g->svd_S;
  const bool all_st = g->gnsn && g->gnnsn && g->gnnsn1 && g->svd_m && g->svd_off && g->svd_U &&
                      g->svd_VT && g->svd_S;
  if (p->order == 3 && (!g->moments || !g->xg_subedges || (any_st && !all_st)))
    return fail(nullptr, FLOW_ERR_ARG,
                "order 3 needs moments and Gauss points, and all or none of the stencils and SVD factors");
  for (int i = 1; i <= nn; i++)
    if (g->node_order[i] != p->order)
      return fail(nullptr, FLOW_ERR_ARG, "mixed node_order is not supported");

  flow_ctx* c = new flow_ctx();
  c->buf.arena = arena;
  c->device = device;
  c->order = p->order;
  c->nn = nn; c->ng = ng; c->ns = ns; c->nbe = nbe;
  c->nnz = g->ia[nn + 1];
  if (cudaSetDevice(device) != cudaSuccess) return fail(c, FLOW_ERR_CUDA, "cudaSetDevice failed");
  cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, device);
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
    return fail(c, FLOW_ERR_CUDA, "stream creation failed");
  cudaEventCreate(&c->ev0);
  cudaEventCreate(&c->ev1);
  // kernel attributes and module loading, once per device, before any work
  if (!ensure_kernel_attrs(device))
    return fail(c, FLOW_ERR_CUDA, "cannot load the kernels or reserve their shared memory");

  if (arena) {
    // the state buffers alone (a lower bound of what the context carves):
    // an arena without that much room refuses now, before the host work
    const size_t nq = (size_t)(nn + ng + 1), n1 = (size_t)(nn + 1);
    const size_t need = 8 * (12 * nq + n1 * (4 * 4 + 8 + 8 + 20 + 4 + 1 + 16)) +
                        8 * (16 * (size_t)c->nnz + 36 * (size_t)(ns + 1));
    size_t room;
    {
      std::lock_guard<std::mutex> lock(arena->mu);
      room = arena->size - arena->used;
    }
    if (room < need) return fail(c, FLOW_ERR_BUDGET, "the arena has no room for this mesh");
  }
  // ---- host-side re-layout ----
  std::vector<std::pair<int, int>> items;
  Csr nsub, nbed, nedg;
  items.reserve(2 * ns);
  std::vector<int2> sub_lr(ns + 1);
  std::vector<double4> sub_geo(ns + 1), sub_dx(ns + 1);
  for (int s = 1; s <= ns; s++) {
    int e = g->subedges[2 * s];
    int L = g->edges[2 * e], R = g->edges[2 * e + 1];
    sub_lr[s] = make_int2(L, R);
    sub_geo[s] = make_double4(g->xn_subedges[3 * s], g->xn_subedges[3 * s + 1],
                              g->xn_subedges[3 * s + 2], 0.);
    // face point of Reconstruct (reconstruct.C:183-197)
    int gel = g->subedges[2 * s + 1];
    double fc0 = (g->el_cent[2 * gel] + g->xm_subedges[2 * s]) * 0.5;
    double fc1 = (g->el_cent[2 * gel + 1] + g->xm_subedges[2 * s + 1]) * 0.5;
    sub_dx[s] = make_double4(fc0 - g->x[2 * L], fc1 - g->x[2 * L + 1], fc0 - g->x[2 * R],
                             fc1 - g->x[2 * R + 1]);
    items.push_back({L, s << 1});
    items.push_back({R, (s << 1) | 1});
  }
  nsub.build(nn, items);
  items.clear();
  for (int b = 1; b <= nbe; b++) items.push_back({g->bedges[5 * b], b});
  nbed.build(nn, items);
  items.clear();
  std::vector<int2> edge_lr(ne + 1);
  std::vector<double4> edge_w(ne + 1, make_double4(0, 0, 0, 0));
  c->has_edge_w = g->edge_weight != nullptr;
  for (int e = 1; e <= ne; e++) {
    int L = g->edges[2 * e], R = g->edges[2 * e + 1];
    edge_lr[e] = make_int2(L, R);
    if (g->edge_weight)
      edge_w[e] = make_double4(g->edge_weight[4 * e], g->edge_weight[4 * e + 1],
                               g->edge_weight[4 * e + 2], g->edge_weight[4 * e + 3]);
    items.push_back({L, e << 1});
    items.push_back({R, (e << 1) | 1});
  }
  nedg.build(nn, items);
  std::vector<int> nedg_nbr(nedg.idx.size());
  for (size_t k = 0; k < nedg.idx.size(); k++) {
    const int e = nedg.idx[k] >> 1, side = nedg.idx[k] & 1;
    nedg_nbr[k] = side ? edge_lr[e].x : edge_lr[e].y;
  }
  // subedges of each edge, ascending
  std::vector<int2> edge_sub(ne + 1, make_int2(-1, -1));
  for (int s = 1; s <= ns; s++) {
    int e = g->subedges[2 * s];
    if (edge_sub[e].x < 0) edge_sub[e].x = s;
    else if (edge_sub[e].y < 0) edge_sub[e].y = s;
    else return fail(c, FLOW_ERR_ARG, "an edge has more than two subedges");
  }
  // per CSR block: the edge's subedges and the row's role
  const int nnz = c->nnz;
  std::vector<int4> csr_sub(nnz, make_int4(-1, -1, 0, 0));
  for (int n = 1; n <= nn; n++) {
    for (int k = g->ia[n]; k < g->ia[n + 1]; k++) {
      int col = g->ja[k];
      if (col == n) continue;
      int found = -1, role = 0;
      for (int q = nedg.ptr[n]; q < nedg.ptr[n + 1]; q++) {
        int e = nedg.idx[q] >> 1, side = nedg.idx[q] & 1;
        int other = side ? edge_lr[e].x : edge_lr[e].y;
        if (other == col) { found = e; role = side; break; }
      }
      if (found < 0) return fail(c, FLOW_ERR_ARG, "CSR block without an edge");
      csr_sub[k] = make_int4(edge_sub[found].x, edge_sub[found].y, role, 0);
    }
  }
  // per subedge incidence: the row position of the block (node, other end)
  std::vector<int> nsub_slot(nsub.idx.size(), 0);
  c->fused_ok = true;
  for (int n = 1; n <= nn; n++) {
    if (g->ia[n + 1] - g->ia[n] - 1 > kRecBlocks) c->fused_ok = false;
    for (int k = nsub.ptr[n]; k < nsub.ptr[n + 1]; k++) {
      const int sub = nsub.idx[k] >> 1, side = nsub.idx[k] & 1;
      const int other = side ? sub_lr[sub].x : sub_lr[sub].y;
      int pos = -1;
      for (int b = g->ia[n]; b < g->ia[n + 1]; b++)
        if (g->ja[b] == other) pos = b - g->ia[n];
      if (pos < 0 || pos >= kRecBlocks) c->fused_ok = false;
      nsub_slot[k] = pos < 0 ? 0 : std::min(pos, kRecBlocks - 1);
    }
  }
  std::vector<int4> bed_info(nbe + 1, make_int4(0, 0, 0, 0));
  std::vector<double2> bed_cnrm(nbe + 1, make_double2(0., 0.));
  for (int b = 1; b <= nbe; b++) {
    int rn = g->bedges[5 * b], gn = g->bedges[5 * b + 1] + nn;
    int bc = g->bbc[g->bedges[5 * b + 3]];
    int wall = !(bc == 0 || (bc % 2 == 0));
    bed_info[b] = make_int4(rn, gn, bc, wall);
    if (bc > 10) {
      double nx, ny;
      flow_curved_normal(bc, &g->x[2 * rn], &nx, &ny);
      bed_cnrm[b] = make_double2(nx, ny);
    }
  }
  // k=2 stencils: node i uses gnsn[gnnsn[gnnsn1[i]+1] .. gnnsn[gnnsn1[i+1]])
  std::vector<int> st_ptr(nn + 2, 0), st_idx;
  std::vector<double> st_w, U1, VT((size_t)(nn + 1) * 25, 0.), S((size_t)(nn + 1) * 5, 1.);
  int stencil_max = 0;
  c->has_stencils = p->order == 3 && all_st;
  if (c->has_stencils) {
    for (int i = 1; i <= nn; i++) {
      int a0 = g->gnnsn[g->gnnsn1[i] + 1], a1 = g->gnnsn[g->gnnsn1[i + 1]];
      int mrows = a1 - a0;
      if (mrows != g->svd_m[i]) return fail(c, FLOW_ERR_ARG, "stencil size differs from svd_m");
      if (mrows < 5 || mrows > 64) return fail(c, FLOW_ERR_ARG, "stencil size out of range");
      stencil_max = std::max(stencil_max, mrows);
      st_ptr[i] = (int)st_idx.size();
      for (int j = a0; j < a1; j++) {
        int nb = g->gnsn[j];
        double dx0 = g->x[2 * nb] - g->x[2 * i];
        double dx1 = g->x[2 * nb + 1] - g->x[2 * i + 1];
        double dist = sqrt(dx0 * dx0 + dx1 * dx1);
        st_idx.push_back(nb);
        st_w.push_back(1.0 / pow(dist, 1.0));  // compute_derivatives.C:1470 (GEOM_WEIGHT 1)
      }
      const double* Ui = g->svd_U + g->svd_off[i];
      // the first 5 columns of U, re-laid row by row (U1[k][c] = U[c*m + k])
      for (int k = 0; k < mrows; k++)
        for (int q = 0; q < 5; q++) U1.push_back(Ui[q * mrows + k]);
      for (int q = 0; q < 25; q++) VT[(size_t)i * 25 + q] = g->svd_VT[(size_t)i * 25 + q];
      for (int q = 0; q < 5; q++) S[(size_t)i * 5 + q] = g->svd_S[(size_t)i * 5 + q];
    }
    st_ptr[nn + 1] = (int)st_idx.size();
  }

  // ---- staged node kernel: the largest slice of each list any tile holds ----
  {
    StageCaps cap{0, 0, 0};
    for (int n0 = 1; n0 <= nn; n0 += kStageNodes) {
      const int n1 = std::min(n0 + kStageNodes, nn + 1);
      cap.sub = std::max(cap.sub, nsub.ptr[n1] - nsub.ptr[n0]);
      cap.edg = std::max(cap.edg, nedg.ptr[n1] - nedg.ptr[n0]);
      if (c->has_stencils) cap.sten = std::max(cap.sten, st_ptr[n1] - st_ptr[n0]);
    }
    c->stage_caps = cap;
    c->stage_ok[0] = stage_smem_bytes(1, cap) <= kStageSmemMax;
    c->stage_ok[1] = c->has_stencils && stage_smem_bytes(3, cap) <= kStageSmemMax;
  }

  // ---- device mesh ----
  DevMesh& m = c->m;
  m.nn = nn; m.ng = ng; m.ne = ne; m.ns = ns; m.nbe = nbe; m.nnz = nnz; m.order = p->order;
  m.stencil_max = stencil_max;
  bool okk = true;
#define UP(field, vec) do { auto* d = upload_vec(c, vec); okk = okk && d; m.field = d; } while (0)
  UP(nsub_ptr, nsub.ptr); UP(nsub, nsub.idx); UP(nsub_slot, nsub_slot);
  UP(nbed_ptr, nbed.ptr); UP(nbed, nbed.idx);
  UP(nedg_ptr, nedg.ptr); UP(nedg, nedg.idx); UP(nedg_nbr, nedg_nbr);
  UP(sub_lr, sub_lr); UP(sub_geo, sub_geo); UP(sub_dx, sub_dx);
  UP(edge_lr, edge_lr); UP(edge_w, edge_w);
  UP(csr_sub, csr_sub);
  UP(bed_info, bed_info); UP(bed_cnrm, bed_cnrm);
  {
    std::vector<int> ia(g->ia, g->ia + nn + 2), iau(g->iau, g->iau + nn + 1), ja(g->ja, g->ja + nnz);
    UP(ia, ia); UP(iau, iau); UP(ja, ja);
    c->h_ia = ia;
    c->h_ja = ja;
    std::vector<double> x(g->x, g->x + (size_t)(nn + ng + 1) * 2), cv(g->cv_area, g->cv_area + nn + 1);
    UP(x, x); UP(cv_area, cv);
    std::vector<int> no(g->node_order, g->node_order + nn + ng + 1);
    UP(node_order, no);
    std::vector<double> xg((size_t)(ns + 1) * 6, 0.);
    if (g->xg_subedges) std::copy(g->xg_subedges, g->xg_subedges + xg.size(), xg.begin());
    UP(sub_xg, xg);
    std::vector<double> xgb((size_t)(nbe + 1) * 6, 0.), xgnb((size_t)(nbe + 1) * 9, 0.);
    if (g->xg_bedges) std::copy(g->xg_bedges, g->xg_bedges + xgb.size(), xgb.begin());
    if (g->xgn_bedges) std::copy(g->xgn_bedges, g->xgn_bedges + xgnb.size(), xgnb.begin());
    UP(xg_bedges, xgb); UP(xgn_bedges, xgnb);
    std::vector<double> mo((size_t)(nn + 1) * 9, 0.);
    if (g->moments) std::copy(g->moments, g->moments + mo.size(), mo.begin());
    UP(moments, mo);
  }
  if (c->has_stencils) {
    UP(st_ptr, st_ptr); UP(st_idx, st_idx); UP(st_w, st_w);
    UP(svd_U1, U1); UP(svd_VT, VT); UP(svd_S, S);
  }
#undef UP
  if (!okk) return fail(c, carve_error(c), "device allocation or upload failed");

  // ---- stage tables of the one-CTA ordered sweep ----
  {
    int bw = 0;
    for (int n = 1; n <= nn; n++)
      for (int k = g->ia[n]; k < g->ia[n + 1]; k++) bw = std::max(bw, std::abs(g->ja[k] - n));
    std::vector<int> rs, row_stage(nn + 1, 0);
    bool fits = bw <= kWindow - kStages * kStageRows - 1;
    rs.push_back(1);
    int rows = 0, blocks = 0;
    for (int n = 1; n <= nn && fits; n++) {
      int nb = g->ia[n + 1] - g->ia[n];
      if (nb > kStageBlocks) { fits = false; break; }
      if (rows + 1 > kStageRows || blocks + nb > kStageBlocks) {
        rs.push_back(n);
        rows = 0;
        blocks = 0;
      }
      rows++;
      blocks += nb;
      row_stage[n] = (int)rs.size() - 1;
    }
    rs.push_back(nn + 1);
    if (fits) {
      std::vector<int> japad(g->ja, g->ja + nnz);
      japad.resize((size_t)nnz + 16, 0);
      int* d_rs = upload_vec(c, rs);
      int* d_row = upload_vec(c, row_stage);
      int* d_ja = upload_vec(c, japad);
      if (!d_rs || !d_row || !d_ja) return fail(c, carve_error(c), "sweep table upload failed");
      c->sweep_tb.stage_row0 = d_rs;
      c->sweep_tb.row_stage = d_row;
      c->sweep_tb.ja_pad = d_ja;
      c->sweep_tb.nstages = (int)rs.size() - 1;
      c->sweep_cta_ok = true;
    }
  }

  // ---- device state ----
  DevState& s = c->s;
  size_t nq = (size_t)(nn + ng + 1) * 4;
  s.Q = c->buf.alloc<double>(nq);
  s.nQ = c->buf.alloc<double>(nq);
  s.pQ = c->buf.alloc<double>(nq);
  s.dQ = c->buf.alloc<double>((size_t)(nn + 1) * 4);
  s.dQ2 = c->buf.alloc<double>((size_t)(nn + 1) * 4);
  s.R = c->buf.alloc<double>((size_t)(nn + 1) * 4);
  s.RHS = c->buf.alloc<double>((size_t)(nn + 1) * 4);
  s.grad = c->buf.alloc<double>((size_t)(nn + 1) * 8);
  s.phi = c->buf.alloc<double>((size_t)(nn + 1) * 8);
  s.hess5 = c->buf.alloc<double>((size_t)(nn + 1) * 20);
  s.pv = c->buf.alloc<double>((size_t)(nn + 1) * 4);
  s.dt = c->buf.alloc<double>((size_t)(nn + 1));
  s.LHS = c->buf.alloc<double>((size_t)nnz * 16);
  s.LUd = c->buf.alloc<double>((size_t)(nn + 1) * 16);
  s.xn_bedges = c->buf.alloc<double>((size_t)(nbe + 1) * 3);
  s.F = c->buf.alloc<double>((size_t)(ns + 1) * 4);
  s.JL = c->buf.alloc<double>((size_t)(ns + 1) * 16);
  s.JR = c->buf.alloc<double>((size_t)(ns + 1) * 16);
  s.Fb = c->buf.alloc<double>((size_t)(nbe + 1) * 4);
  s.Jb = c->buf.alloc<double>((size_t)(nbe + 1) * 16);
  s.bforce = c->buf.alloc<double>((size_t)(nbe + 1) * 4);
  s.done = c->buf.alloc<int>((size_t)(nn + 1));
  s.counter = c->buf.alloc<unsigned>(4);
  s.status = c->buf.alloc<int>(1);
  s.skip = c->buf.alloc<int>(1);
  s.exact = c->buf.alloc<int>(1);
  s.stop = c->buf.alloc<int>(1);
  s.steps_done = c->buf.alloc<int>(1);
  s.citer = c->buf.alloc<int>(1);
  // the partial sums of the step's reductions, then k_finish_step's block count
  s.partial = c->buf.alloc<double>(2 * kRedBlocks + 2);
  s.scalars = c->buf.alloc<double>(8);
  if (!s.Q || !s.nQ || !s.pQ || !s.dQ || !s.dQ2 || !s.R || !s.RHS || !s.grad || !s.phi || !s.hess5 ||
      !s.pv || !s.dt || !s.LHS || !s.LUd || !s.xn_bedges || !s.F || !s.JL || !s.JR || !s.Fb ||
      !s.Jb || !s.bforce || !s.done || !s.counter || !s.status || !s.skip || !s.partial ||
      !s.scalars || !s.stop || !s.steps_done || !s.citer || !s.exact)
    return fail(c, carve_error(c), "device state allocation failed");
  bool zero_ok = true;
  auto zero = [&](void* ptr, size_t bytes) {
    zero_ok = zero_ok && cudaMemsetAsync(ptr, 0, bytes, c->stream) == cudaSuccess;
  };
  zero(s.Q, nq * 8);
  zero(s.nQ, nq * 8);
  zero(s.pQ, nq * 8);
  zero(s.dQ, (size_t)(nn + 1) * 32);
  zero(s.dQ2, (size_t)(nn + 1) * 32);
  zero(s.R, (size_t)(nn + 1) * 32);
  zero(s.RHS, (size_t)(nn + 1) * 32);
  zero(s.grad, (size_t)(nn + 1) * 64);
  zero(s.phi, (size_t)(nn + 1) * 64);
  zero(s.hess5, (size_t)(nn + 1) * 160);
  zero(s.pv, (size_t)(nn + 1) * 32);
  zero(s.dt, (size_t)(nn + 1) * 8);
  zero(s.LHS, (size_t)nnz * 128);
  zero(s.done, (size_t)(nn + 1) * 4);
  zero(s.status, 4);
  zero(s.skip, 4);
  zero(s.exact, 4);
  zero(s.stop, 4);
  zero(s.steps_done, 4);
  zero(s.citer, 4);
  zero(s.scalars, 64);
  zero(s.partial, (2 * kRedBlocks + 2) * 8);
  if (!zero_ok) return fail(c, FLOW_ERR_CUDA, "clearing the device state failed");
  std::vector<double> xnb((size_t)(nbe + 1) * 3, 0.);
  std::copy(g->xn_bedges, g->xn_bedges + xnb.size(), xnb.begin());
  c->xnb0 = c->buf.alloc<double>(xnb.size());
  if (!c->xnb0) return fail(c, carve_error(c), "device allocation failed");
  if (!upload(c, s.xn_bedges, xnb.data(), xnb.size() * 8) ||
      !upload(c, c->xnb0, xnb.data(), xnb.size() * 8))
    return fail(c, FLOW_ERR_CUDA, "upload failed");
  // the context's own stream only: a device-wide synchronisation here would
  // invalidate a graph capture another thread has open
  if (cudaStreamSynchronize(c->stream) != cudaSuccess)
    return fail(c, FLOW_ERR_CUDA, "device error at set-up");
  c->ok = true;
  if (status) *status = 0;
  return c;
}

void flow_destroy(flow_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  harvest(c);
  // pinned frees and cudaFree synchronise the device: not while a capture is open
  DeviceWide gate(g_device_gate);
  drop_graphs(c);
  for (cudaEvent_t e : c->event_pool) cudaEventDestroy(e);
  if (c->ev_flag) cudaEventDestroy(c->ev_flag);
  if (c->h_flags) cudaFreeHost(c->h_flags);
  for (cudaEvent_t e : c->ev_run)
    if (e) cudaEventDestroy(e);
  if (c->h_run) cudaFreeHost(c->h_run);
  if (c->h_runr) cudaFreeHost(c->h_runr);
  c->buf.release();
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

int flow_set_state(flow_ctx* c, const double* Q) {
  if (!c || !c->ok || !Q) return FLOW_ERR_ARG;
  cudaSetDevice(c->device);
  size_t bytes = sizeof(double) * 4 * (size_t)(c->nn + c->ng + 1);
  size_t xbytes = sizeof(double) * 3 * (size_t)(c->nbe + 1);
  if (cudaMemcpyAsync(c->s.Q, Q, bytes, cudaMemcpyHostToDevice, c->stream) != cudaSuccess ||
      cudaMemcpyAsync(c->s.nQ, c->s.Q, bytes, cudaMemcpyDeviceToDevice, c->stream) !=
          cudaSuccess ||
      cudaMemcpyAsync(c->s.xn_bedges, c->xnb0, xbytes, cudaMemcpyDeviceToDevice, c->stream) !=
          cudaSuccess ||
      cudaStreamSynchronize(c->stream) != cudaSuccess)
    return FLOW_ERR_CUDA;
  return 0;
}

int flow_set_sweep_mode(flow_ctx* c, int mode) {
  if (!c || mode < 0 || mode > 1) return FLOW_ERR_ARG;
  if (mode == 1 && !c->sweep_cta_ok) {
    set_error("matrix bandwidth too large for the one-CTA sweep window");
    return FLOW_ERR_ARG;
  }
  c->sweep_mode = mode;
  return 0;
}

int flow_set_precision(flow_ctx* c, int mode) {
  if (!c || !c->ok || mode < 0 || mode > 3) {
    set_error("flow_set_precision: null context or mode not 0..3");
    return FLOW_ERR_ARG;
  }
  cudaSetDevice(c->device);
  if (mode != 0) {
    cudaStreamSynchronize(c->stream);
    drop_graphs(c);
    int rc = mode == 3 ? build_chunk_iterate(c) : build_mixed_tables(c, mode >= 2);
    if (!rc && mode == 3) rc = build_chunk_tables(c);
    if (rc) return rc;
  }
  c->precision = mode;
  return 0;
}

int flow_set_sweep_ring(flow_ctx* c, int rows) {
  int shape = -1;
  for (int k = 0; k < kRingShapes; k++)
    if (rows == ring_rows(k)) shape = k;
  if (rows == 0) shape = 0;
  if (!c || !c->ok || shape < 0) {
    set_error("flow_set_sweep_ring: null context or rows not 0, 16, 32 or 64");
    return FLOW_ERR_ARG;
  }
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  c->ring = shape;
  if (c->precision == 3) {
    if (!c->ring_ok[shape]) {
      c->ring = 0;
      set_error("flow_set_sweep_ring: a chunk has more sub-levels of that size than the kernel holds");
      return FLOW_ERR_ARG;
    }
    drop_graphs(c);
    apply_ring(c);
  }
  return 0;
}

int flow_set_sweep_dataflow(flow_ctx* c, int on) {
  if (!c || !c->ok) {
    set_error("flow_set_sweep_dataflow: null context");
    return FLOW_ERR_ARG;
  }
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  drop_graphs(c);
  c->sweep_df = on ? 1 : 0;
  return 0;
}

int flow_set_chunk(flow_ctx* c, int rows, int levels) {
  if (!c || !c->ok || rows < 0 || rows > 2048 || levels < 0) {
    set_error("flow_set_chunk: null context, rows outside 0..2048 or negative levels");
    return FLOW_ERR_ARG;
  }
  c->chunk_rows = rows;
  c->chunk_levels = levels;
  if (c->precision == 3) {
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    drop_graphs(c);
    return build_chunk_tables(c);
  }
  return 0;
}

int flow_chunk_starts(flow_ctx* c, int* starts, int cap, int* nchunks, int* ncolours) {
  if (!c || !c->ok || c->h_chunk_start.empty()) return FLOW_ERR_ARG;
  const int n = (int)c->h_chunk_start.size() - 1;
  if (nchunks) *nchunks = n;
  if (ncolours) *ncolours = c->ct.ncol;
  if (starts)
    for (int i = 0; i <= n && i < cap; i++) starts[i] = c->h_chunk_start[i];
  return 0;
}

int flow_set_sweep_schedule(flow_ctx* c, int sweeps, int until_step) {
  if (!c || !c->ok || sweeps < 0 || until_step < 0) {
    set_error("flow_set_sweep_schedule: null context or negative argument");
    return FLOW_ERR_ARG;
  }
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  drop_graphs(c);
  c->sched_sweeps = sweeps;
  c->sched_until = until_step;
  return 0;
}

int flow_set_stream_priority(flow_ctx* c, int priority) {
  if (!c || !c->ok) return FLOW_ERR_ARG;
  cudaSetDevice(c->device);
  int lo = 0, hi = 0;  // hi is the greatest priority (numerically lowest)
  cudaDeviceGetStreamPriorityRange(&lo, &hi);
  const int pr = std::max(hi, std::min(lo, priority));
  cudaStream_t st = nullptr;
  if (cudaStreamSynchronize(c->stream) != cudaSuccess ||
      cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, pr) != cudaSuccess) {
    set_error("flow_set_stream_priority: stream creation failed");
    return FLOW_ERR_CUDA;
  }
  harvest(c);
  DeviceWide gate(g_device_gate);
  cudaStreamDestroy(c->stream);
  c->stream = st;
  return 0;
}

int flow_set_graphs(flow_ctx* c, int on) {
  if (!c || !c->ok) return FLOW_ERR_ARG;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  if (!on) drop_graphs(c);
  c->use_graphs = on ? 1 : 0;
  return 0;
}

int flow_set_jacobian(flow_ctx* c, int mode) {
  if (!c || !c->ok || mode < 0 || mode > 2) {
    set_error("flow_set_jacobian: null context or mode not 0..2");
    return FLOW_ERR_ARG;
  }
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  drop_graphs(c);
  c->jac_mode = mode;
  return 0;
}

int flow_set_sweep_pairs(flow_ctx* c, int on) {
  if (!c || !c->ok) {
    set_error("flow_set_sweep_pairs: null context");
    return FLOW_ERR_ARG;
  }
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  drop_graphs(c);
  c->sweep_pairs = on ? 1 : 0;
  return 0;
}

int flow_set_exact_rms(flow_ctx* c, int on) {
  if (!c || !c->ok) {
    set_error("flow_set_exact_rms: null context");
    return FLOW_ERR_ARG;
  }
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  drop_graphs(c);
  c->exact_rms = on ? 1 : 0;
  return 0;
}

int flow_set_capture_fault(flow_ctx* c, int count) {
  if (!c || !c->ok || count < 0) {
    set_error("flow_set_capture_fault: null context or negative count");
    return FLOW_ERR_ARG;
  }
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  drop_graphs(c);  // the next chunk captures again
  c->capture_fault = count;
  return 0;
}

long flow_capture_fallbacks(flow_ctx* c) { return c ? c->capture_fallbacks : -1; }

int flow_precision_of(flow_ctx* c) { return c ? c->precision : -1; }

int flow_solve(flow_ctx* c, const flow_params* p, int ts, double* dq_norm, double* r_rho) {
  if (!c || !c->ok) return FLOW_ERR_ARG;
  int rc = check_params(c, p);
  if (rc) return rc;
  cudaSetDevice(c->device);
  if ((rc = ensure_hist(c, 1))) return rc;
  cudaEventRecord(c->ev0, c->stream);
  reset_run(c, 0.);
  rc = enqueue_step(c, p, ts, 0, 1);
  cudaEventRecord(c->ev1, c->stream);
  if (rc) return rc;
  int st = read_status(c);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, c->ev0, c->ev1);
  c->last_ms = ms;
  double h[2] = {0., 0.};
  if (!download(c, &h[0], c->d_hist, sizeof(double)) ||
      !download(c, &h[1], c->d_hist + c->hist_cap, sizeof(double)))
    return st | FLOW_ERR_CUDA;
  if (dq_norm) *dq_norm = h[0];
  if (r_rho) *r_rho = h[1];
  return st;
}

int flow_run(flow_ctx* c, const flow_params* p, int ts0, int nsteps, double* r_hist,
             double* dq_hist) {
  if (!c || !c->ok || nsteps < 0) return FLOW_ERR_ARG;
  int rc = check_params(c, p);
  if (rc) return rc;
  cudaSetDevice(c->device);
  if ((rc = ensure_hist(c, std::max(nsteps, 1)))) return rc;
  cudaEventRecord(c->ev0, c->stream);
  reset_run(c, 0.);
  for (int i = 0; i < nsteps && !rc; i++) rc |= enqueue_step(c, p, ts0 + i, i, i == 0);
  cudaEventRecord(c->ev1, c->stream);
  if (rc) return rc;
  int st = read_status(c);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, c->ev0, c->ev1);
  c->last_ms = ms;
  if (dq_hist && !download(c, dq_hist, c->d_hist, sizeof(double) * nsteps)) st |= FLOW_ERR_CUDA;
  if (r_hist && !download(c, r_hist, c->d_hist + c->hist_cap, sizeof(double) * nsteps))
    st |= FLOW_ERR_CUDA;
  return st;
}

int flow_converge(flow_ctx* c, const flow_params* p, int ts0, int max_steps, double drop,
                  int chunk, int* steps, double* r_first, double* r_last) {
  if (!c || !c->ok || max_steps < 1 || !(drop > 0.)) return FLOW_ERR_ARG;
  int rc = check_params(c, p);
  if (rc) return rc;
  cudaSetDevice(c->device);
  if (chunk < 1) chunk = 64;
  if ((rc = ensure_hist(c, 1))) return rc;
  reset_run(c, drop);
  cudaEventRecord(c->ev0, c->stream);
  int done = 0, stop = 0, issued = 0;
  while (!rc && issued < max_steps) {
    int n = std::min(chunk, max_steps - issued);
    if (issued == 0 || n < chunk) {
      for (int i = 0; i < n && !rc; i++, issued++)
        rc |= enqueue_step(c, p, ts0 + issued, -1, issued == 0);
    } else {
      rc |= enqueue_chunk(c, p, ts0 + issued, n);
      issued += n;
    }
    if (rc) break;
    int st = 0;
    if (!download(c, &stop, c->s.stop, sizeof(int)) ||
        !download(c, &done, c->s.steps_done, sizeof(int)) ||
        !download(c, &st, c->s.status, sizeof(int))) {
      rc |= FLOW_ERR_CUDA;  // the clean-up below still runs
      break;
    }
    harvest(c);
    if (stop || st) break;
  }
  cudaEventRecord(c->ev1, c->stream);
  if (rc) {
    // leave the device in the no-target state for later calls
    reset_run(c, 0.);
    cudaStreamSynchronize(c->stream);
    harvest(c);
    return rc;
  }
  int st = read_status(c);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, c->ev0, c->ev1);
  c->last_ms = ms;
  double sc[8] = {0., 0., 0., 0., 0., 0., 0., 0.};
  if (!download(c, sc, c->s.scalars, sizeof(sc)) || !download(c, &done, c->s.steps_done, sizeof(int)) ||
      !download(c, &stop, c->s.stop, sizeof(int)))
    st |= FLOW_ERR_CUDA;
  // leave the device in the no-target state for later calls
  reset_run(c, 0.);
  cudaStreamSynchronize(c->stream);
  if (steps) *steps = done;
  if (r_first) *r_first = sc[6];
  if (r_last) *r_last = sqrt(sc[2]);
  if (st) return st;
  return stop ? 0 : FLOW_ERR_NOT_CONVERGED;
}

int flow_converge_batch(flow_ctx** ctxs, int n, const flow_params* p, int ts0, int max_steps,
                        double drop, int chunk, int* steps, int* status) {
  if (!ctxs || n < 1 || max_steps < 1 || !(drop > 0.)) return FLOW_ERR_ARG;
  if (chunk < 1) chunk = 64;
  int rc_all = 0;
  for (int i = 0; i < n; i++) {
    flow_ctx* c = ctxs[i];
    if (!c || !c->ok) return FLOW_ERR_ARG;
    int rc = check_params(c, p);
    if (rc) return rc;
    cudaSetDevice(c->device);
    if ((rc = ensure_hist(c, 1))) return rc;
    if (!c->h_flags) {
      DeviceWide gate(g_device_gate);
      if (cudaHostAlloc(&c->h_flags, 2 * sizeof(int), cudaHostAllocDefault) != cudaSuccess)
        return FLOW_ERR_CUDA;
    }
    if (!c->ev_flag) cudaEventCreateWithFlags(&c->ev_flag, cudaEventDisableTiming);
    c->h_flags[0] = 0;
    c->h_flags[1] = 0;
    reset_run(c, drop);
    cudaEventRecord(c->ev0, c->stream);
  }
  std::vector<int> issued(n, 0), active(n, 1), pending(n, 0);
  int nactive = n;
  while (nactive > 0) {
    // issue one chunk per active context, then read back the previous round
    for (int i = 0; i < n; i++) {
      if (!active[i]) continue;
      flow_ctx* c = ctxs[i];
      cudaSetDevice(c->device);
      int k = std::min(chunk, max_steps - issued[i]);
      int rc = 0;
      if (issued[i] == 0 || k < chunk) {
        for (int q = 0; q < k && !rc; q++, issued[i]++)
          rc |= enqueue_step(c, p, ts0 + issued[i], -1, issued[i] == 0);
      } else {
        rc |= enqueue_chunk(c, p, ts0 + issued[i], k);
        issued[i] += k;
      }
      if (rc) { rc_all |= rc; active[i] = 0; nactive--; continue; }
      if (pending[i]) {
        // the flags of the previous round are ready once its event completed
        if (cudaEventSynchronize(c->ev_flag) != cudaSuccess) {
          rc_all |= FLOW_ERR_CUDA;
          active[i] = 0;
          nactive--;
          continue;
        }
        harvest(c);
        if (c->h_flags[0] || c->h_flags[1]) { active[i] = 0; nactive--; continue; }
      }
      cudaMemcpyAsync(&c->h_flags[0], c->s.stop, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
      cudaMemcpyAsync(&c->h_flags[1], c->s.status, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
      cudaEventRecord(c->ev_flag, c->stream);
      pending[i] = 1;
      if (issued[i] >= max_steps) { active[i] = 0; nactive--; }
    }
  }
  for (int i = 0; i < n; i++) {
    flow_ctx* c = ctxs[i];
    cudaSetDevice(c->device);
    cudaEventRecord(c->ev1, c->stream);
    int st = read_status(c);
    int done = 0, stop = 0;
    if (!download(c, &done, c->s.steps_done, sizeof(int)) || !download(c, &stop, c->s.stop, sizeof(int)))
      st |= FLOW_ERR_CUDA;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    c->last_ms = ms;
    reset_run(c, 0.);
    cudaStreamSynchronize(c->stream);
    if (steps) steps[i] = done;
    if (!stop && !st) st = FLOW_ERR_NOT_CONVERGED;
    if (status) status[i] = st;
    rc_all |= st;
  }
  return rc_all;
}

int flow_build_matrix(flow_ctx* c, const flow_params* p, int citer) {
  if (!c || !c->ok) return FLOW_ERR_ARG;
  int rc = check_params(c, p);
  if (rc) return rc;
  cudaSetDevice(c->device);
  reset_run(c, 0.);
  StepArgs a = make_args(p, citer);
  a.do_grad = a.do_derivs = a.do_lim = 0;
  c->citer = citer;
  rc = launch_step_args(c, p, citer);
  rc |= launch_node_prepare(c, a);
  k_diag_only<<<grid_blocks(c->nn, 128), 128, 0, c->stream>>>(c->m, c->s);
  rc |= launch_check(c);
  if (rc) return rc;
  return read_status(c);
}

int flow_reconstruct(flow_ctx* c, const flow_params* p, int ts) {
  if (!c || !c->ok) return FLOW_ERR_ARG;
  int rc = check_params(c, p);
  if (rc) return rc;
  cudaSetDevice(c->device);
  reset_run(c, 0.);
  StepArgs a = make_args(p, ts);
  c->citer = ts;
  rc |= launch_step_args(c, p, ts);
  // grad, hess <- 0 and phi <- 1 (solve.C:298-348), keeping the current nQ
  k_begin_step<<<grid_blocks(c->nn + c->ng, 256), 256, 0, c->stream>>>(
      c->m, c->s, kBeginResetPhi | kBeginZeroGrad | kBeginZeroHess);
  rc |= launch_check(c);
  rc |= launch_node_prepare(c, a);
  if (rc) return rc;
  return read_status(c);
}

int flow_residuals(flow_ctx* c, const flow_params* p, int jupdate, int ts) {
  if (!c || !c->ok) return FLOW_ERR_ARG;
  int rc = check_params(c, p);
  if (rc) return rc;
  cudaSetDevice(c->device);
  reset_run(c, 0.);
  StepArgs a = make_args(p, ts);
  c->citer = ts;
  rc = launch_residuals(c, a, jupdate);
  if (rc) return rc;
  return read_status(c);
}

int flow_linear_solve(flow_ctx* c, const flow_params* p, double* rms) {
  if (!c || !c->ok) return FLOW_ERR_ARG;
  int rc = check_params(c, p);
  if (rc) return rc;
  cudaSetDevice(c->device);
  reset_run(c, 0.);
  rc = launch_linear_solve(c, p, true);
  if (rc) return rc;
  int st = read_status(c);
  if (rms) {
    double v = 10.;
    if (c->precision != 0) v = -1.;  // the precision form forms no b-Ax RMS
    else if (p->subits > 0 && !download(c, &v, c->s.scalars, sizeof(double))) st |= FLOW_ERR_CUDA;
    *rms = v;
  }
  return st;
}

int flow_selftest_sweep_timeout(flow_ctx* c, long max_spin, int* status) {
  if (!c || !c->ok || max_spin < 1 || max_spin > (1L << 21) || !status) {
    set_error("flow_selftest_sweep_timeout: null context/status or max_spin outside 1..2^21");
    return FLOW_ERR_ARG;
  }
  cudaSetDevice(c->device);
  static const unsigned kFirst = 1;  // the dispenser starts at row 2: row 1 never runs
  reset_run(c, 0.);
  cudaMemsetAsync(c->s.status, 0, sizeof(int), c->stream);
  cudaMemsetAsync(c->s.skip, 0, sizeof(int), c->stream);
  cudaMemcpyAsync(c->s.counter, &kFirst, sizeof(unsigned), cudaMemcpyHostToDevice, c->stream);
  double* dq_new = c->s.dQ2;
  k_prepare_sweep<<<grid_blocks(4 * (c->nn + 1), 256), 256, 0, c->stream>>>(
      c->s, c->s.dQ, dq_new, 4 * (c->nn + 1));
  int rc = launch_check(c);
  k_sweep_ordered<true><<<c->nsm * 4, 128, 0, c->stream>>>(c->m, c->s, c->s.dQ, dq_new, max_spin);
  rc |= launch_check(c);
  if (rc) return rc;
  *status = read_status(c);
  // the sweep's output buffer is scratch (the buffers were not swapped); the
  // context goes on from its state with a clear status
  cudaMemsetAsync(c->s.status, 0, sizeof(int), c->stream);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) return FLOW_ERR_CUDA;
  return 0;
}

int flow_body_forces(flow_ctx* c, const flow_params* p, double* forces) {
  if (!c || !c->ok || !forces) return FLOW_ERR_ARG;
  cudaSetDevice(c->device);
  StepArgs a = make_args(p, 1);
  // Reconstruct_Gauss_Boundary's order at the current step (reconstruct.C:1725-1760)
  int citer = c->citer;
  int ro = 0;
  if (p->order == 1) ro = citer > p->foits ? 1 : 0;
  if (p->order == 3) ro = citer > p->foits + p->soits ? 3 : (citer > p->foits ? 1 : 0);
  int rc = 0;
  if (c->nbe > 0) {
    k_body_forces<<<grid_blocks(c->nbe, 128), 128, 0, c->stream>>>(c->m, c->s, a, ro);
    rc |= launch_check(c);
  }
  k_body_forces_sum<<<1, 32, 0, c->stream>>>(c->m, c->s);
  rc |= launch_check(c);
  if (rc) return rc;
  double f[2];
  cudaMemcpyAsync(f, c->s.scalars + 4, sizeof(f), cudaMemcpyDeviceToHost, c->stream);
  int st = read_status(c);
  forces[0] = f[0];
  forces[1] = f[1];
  return st;
}

long flow_size(flow_ctx* c, const char* name) {
  if (!c || !name) return -1;
  long nn = c->nn, ng = c->ng;
  std::string n(name);
  if (n == "Q" || n == "nQ" || n == "pQ") return (nn + ng + 1) * 4;
  if (n == "dQ" || n == "R" || n == "RHS" || n == "point_value") return (nn + 1) * 4;
  if (n == "grad" || n == "phi") return (nn + 1) * 8;
  if (n == "hess") return (nn + 1) * 36;
  if (n == "dt") return nn + 1;
  if (n == "LHS") return (long)c->nnz * 16;
  if (n == "xn_bedges") return (long)(c->nbe + 1) * 3;
  if (n == "cfl") return 1;
  return -1;
}

int flow_get(flow_ctx* c, const char* name, double* out, long n) {
  if (!c || !c->ok || !name || !out) return FLOW_ERR_ARG;
  long need = flow_size(c, name);
  if (need < 0) return FLOW_ERR_NOT_FOUND;
  if (n < need) return FLOW_ERR_ARG;
  cudaSetDevice(c->device);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) return FLOW_ERR_CUDA;
  std::string nm(name);
  const double* src = nullptr;
  if (nm == "Q") src = c->s.Q;
  else if (nm == "nQ") src = c->s.nQ;
  else if (nm == "pQ") src = c->s.pQ;
  else if (nm == "dQ") src = c->s.dQ;
  else if (nm == "R") src = c->s.R;
  else if (nm == "RHS") src = c->s.RHS;
  else if (nm == "grad") src = c->s.grad;
  else if (nm == "phi") src = c->s.phi;
  else if (nm == "dt") src = c->s.dt;
  else if (nm == "LHS") src = c->s.LHS;
  else if (nm == "xn_bedges") src = c->s.xn_bedges;
  else if (nm == "point_value") src = c->s.pv;
  if (src) {
    if (cudaMemcpyAsync(out, src, sizeof(double) * need, cudaMemcpyDeviceToHost, c->stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(c->stream) != cudaSuccess)
      return FLOW_ERR_CUDA;
    return 0;
  }
  if (nm == "cfl") return download(c, out, c->s.scalars + 3, sizeof(double)) ? 0 : FLOW_ERR_CUDA;
  if (nm == "hess") {
    std::vector<double> h((size_t)(c->nn + 1) * 20);
    if (!download(c, h.data(), c->s.hess5, h.size() * 8)) return FLOW_ERR_CUDA;
    std::fill(out, out + need, 0.);
    for (long i = 0; i <= c->nn; i++)
      for (int v = 0; v < 4; v++)
        for (int k = 0; k < 5; k++) out[i * 36 + v * 9 + k] = h[i * 20 + v * 5 + k];
    return 0;
  }
  return FLOW_ERR_NOT_FOUND;
}

int flow_set(flow_ctx* c, const char* name, const double* in, long n) {
  if (!c || !c->ok || !name || !in) return FLOW_ERR_ARG;
  const std::string nm(name);
  const long need = flow_size(c, name);
  if (need < 0 || nm == "cfl") return FLOW_ERR_NOT_FOUND;
  if (n < need) {
    set_error("flow_set: fewer values than the array holds");
    return FLOW_ERR_ARG;
  }
  cudaSetDevice(c->device);
  double* dst = nullptr;
  if (nm == "Q") dst = c->s.Q;
  else if (nm == "nQ") dst = c->s.nQ;
  else if (nm == "pQ") dst = c->s.pQ;
  else if (nm == "dQ") dst = c->s.dQ;
  else if (nm == "R") dst = c->s.R;
  else if (nm == "RHS") dst = c->s.RHS;
  else if (nm == "grad") {
    dst = c->s.grad;
    if (!c->grad_written) {
      // from now on the steps that do not form a gradient clear it again
      cudaStreamSynchronize(c->stream);
      drop_graphs(c);
      c->grad_written = true;
    }
  }
  else if (nm == "phi") dst = c->s.phi;
  else if (nm == "dt") dst = c->s.dt;
  else if (nm == "LHS") dst = c->s.LHS;
  else if (nm == "xn_bedges") dst = c->s.xn_bedges;
  else if (nm == "point_value") dst = c->s.pv;
  int rc = 0;
  if (dst) {
    if (!upload(c, dst, in, sizeof(double) * need)) rc = FLOW_ERR_CUDA;
  } else if (nm == "hess") {
    // the five derivatives of each variable the k=2 scheme keeps
    std::vector<double> h((size_t)(c->nn + 1) * 20);
    for (long i = 0; i <= c->nn; i++)
      for (int v = 0; v < 4; v++)
        for (int k = 0; k < 5; k++) h[i * 20 + v * 5 + k] = in[i * 36 + v * 9 + k];
    if (!upload(c, c->s.hess5, h.data(), h.size() * 8)) rc = FLOW_ERR_CUDA;
    else if (cudaStreamSynchronize(c->stream) != cudaSuccess) rc = FLOW_ERR_CUDA;
  } else {
    return FLOW_ERR_NOT_FOUND;
  }
  if (!rc && nm == "LHS") {
    // the sweeps read the LU factors of the diagonal blocks: form them anew
    k_diag_lu<<<grid_blocks(c->nn, 128), 128, 0, c->stream>>>(c->m, c->s);
    rc |= launch_check(c);
  }
  if (!rc && cudaStreamSynchronize(c->stream) != cudaSuccess) rc = FLOW_ERR_CUDA;
  if (rc & FLOW_ERR_CUDA) set_error("flow_set: copy to the device failed");
  return rc;
}

int flow_residual_stage(flow_ctx* c, const flow_params* p, int jupdate, int ts, int stage) {
  if (!c || !c->ok) return FLOW_ERR_ARG;
  if (stage != FLOW_STAGE_INTERIOR && stage != FLOW_STAGE_BOUNDARY) {
    set_error("flow_residual_stage: stage must be FLOW_STAGE_INTERIOR or FLOW_STAGE_BOUNDARY");
    return FLOW_ERR_ARG;
  }
  if (c->precision != 0) {
    set_error("flow_residual_stage: the FP64 drop-in only (precision mode 0)");
    return FLOW_ERR_ARG;
  }
  int rc = check_params(c, p);
  if (rc) return rc;
  cudaSetDevice(c->device);
  reset_run(c, 0.);
  StepArgs a = make_args(p, ts);
  c->citer = ts;
  if (stage == FLOW_STAGE_INTERIOR) {
    // faces, then the per-node sums of the interior faces only
    a.skip_bnd = 1;
    {
      Timed t(c, 1);
      const int nbs = grid_blocks(c->ns, 128);
      launch_flux_variant(c->var[1], [&](auto V) {
        if (a.recon == 1) {
          if (jupdate) k_subedge_flux<1, true, V.value><<<nbs, 128, 0, c->stream>>>(c->m, c->s, a);
          else k_subedge_flux<1, false, V.value><<<nbs, 128, 0, c->stream>>>(c->m, c->s, a);
        } else {
          if (jupdate) k_subedge_flux<0, true, V.value><<<nbs, 128, 0, c->stream>>>(c->m, c->s, a);
          else k_subedge_flux<0, false, V.value><<<nbs, 128, 0, c->stream>>>(c->m, c->s, a);
        }
      });
      rc |= launch_check(c);
    }
    Timed t(c, 3);
    const MixedTables& mt = c->mt;
    const ChunkTables& ct = c->ct;
    const int nbn = grid_blocks(4 * c->nn, 128);
    if (jupdate) k_assemble4<true, 0><<<nbn, 128, 0, c->stream>>>(c->m, c->s, a, mt, ct);
    else k_assemble4<false, 0><<<nbn, 128, 0, c->stream>>>(c->m, c->s, a, mt, ct);
    rc |= launch_check(c);
  } else if (c->nbe > 0) {
    // ghost states, boundary fluxes and Jacobians, added onto the interior sums
    {
      Timed t(c, 2);
      const int nbb = grid_blocks(c->nbe, 128);
      if (jupdate) k_boundary<true><<<nbb, 128, 0, c->stream>>>(c->m, c->s, a);
      else k_boundary<false><<<nbb, 128, 0, c->stream>>>(c->m, c->s, a);
      rc |= launch_check(c);
    }
    Timed t(c, 3);
    const int nbn = grid_blocks(4 * c->nn, 128);
    if (jupdate) k_boundary_add4<true><<<nbn, 128, 0, c->stream>>>(c->m, c->s);
    else k_boundary_add4<false><<<nbn, 128, 0, c->stream>>>(c->m, c->s);
    rc |= launch_check(c);
  }
  if (rc) return rc;
  return read_status(c);
}

int flow_save_state(flow_ctx* c) {
  if (!c || !c->ok) return FLOW_ERR_ARG;
  cudaSetDevice(c->device);
  size_t nq = (size_t)(c->nn + c->ng + 1) * 4, nx = (size_t)(c->nbe + 1) * 3;
  if (!c->snapQ) {
    c->snapQ = c->buf.alloc<double>(nq);
    c->snapnQ = c->buf.alloc<double>(nq);
    c->snappQ = c->buf.alloc<double>(nq);
    c->snapXnb = c->buf.alloc<double>(nx);
    if (!c->snapQ || !c->snapnQ || !c->snappQ || !c->snapXnb) return FLOW_ERR_CUDA;
  }
  cudaMemcpyAsync(c->snapQ, c->s.Q, nq * 8, cudaMemcpyDeviceToDevice, c->stream);
  cudaMemcpyAsync(c->snapnQ, c->s.nQ, nq * 8, cudaMemcpyDeviceToDevice, c->stream);
  cudaMemcpyAsync(c->snappQ, c->s.pQ, nq * 8, cudaMemcpyDeviceToDevice, c->stream);
  cudaMemcpyAsync(c->snapXnb, c->s.xn_bedges, nx * 8, cudaMemcpyDeviceToDevice, c->stream);
  return read_status(c);
}

int flow_restore_state(flow_ctx* c) {
  if (!c || !c->ok || !c->snapQ) return FLOW_ERR_ARG;
  cudaSetDevice(c->device);
  size_t nq = (size_t)(c->nn + c->ng + 1) * 4, nx = (size_t)(c->nbe + 1) * 3;
  cudaMemcpyAsync(c->s.Q, c->snapQ, nq * 8, cudaMemcpyDeviceToDevice, c->stream);
  cudaMemcpyAsync(c->s.nQ, c->snapnQ, nq * 8, cudaMemcpyDeviceToDevice, c->stream);
  cudaMemcpyAsync(c->s.pQ, c->snappQ, nq * 8, cudaMemcpyDeviceToDevice, c->stream);
  cudaMemcpyAsync(c->s.xn_bedges, c->snapXnb, nx * 8, cudaMemcpyDeviceToDevice, c->stream);
  return read_status(c);
}

int flow_set_variants(flow_ctx* c, int node_prepare, int flux) {
  if (!c || !c->ok || node_prepare < 0 || node_prepare >= kNodeVariants || flux < 0 ||
      flux >= kVariants) {
    set_error("flow_set_variants: null context, node variant outside 0..7 or flux outside 0..2");
    return FLOW_ERR_ARG;
  }
  if (node_prepare == 3 && !c->stage_ok[0] && !c->stage_ok[1]) {
    set_error("flow_set_variants: the staged node kernel's shared memory does not fit this mesh");
    return FLOW_ERR_ARG;
  }
  if (c->var[0] != node_prepare || c->var[1] != flux) {
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    drop_graphs(c);
  }
  c->var[0] = node_prepare;
  c->var[1] = flux;
  return 0;
}

int flow_autotune(flow_ctx* c, const flow_params* p, int ts, int steps, int* variants,
                  double* ms) {
  if (!c || !c->ok || ts < 1) return FLOW_ERR_ARG;
  int rc = check_params(c, p);
  if (rc) return rc;
  cudaSetDevice(c->device);
  if (steps < 1) steps = 4;
  if ((rc = flow_save_state(c))) return rc;
  if ((rc = ensure_hist(c, 1))) return rc;
  const int saved_timing = c->timing;
  long kc[8];
  double km[8];
  std::copy(c->kcount, c->kcount + 8, kc);
  std::copy(c->kms, c->kms + 8, km);
  for (int k = 0; k < 2 && !rc; k++) {  // class 0: k_node_prepare4, class 1: k_subedge_flux
    int best = c->var[k];
    double best_ms = 1e30;
    const int nv = k == 0 ? kNodeVariants : kVariants;
    for (int v = 0; v < nv && !rc; v++) {
      if (k == 0 && v == 3 && !c->stage_ok[0] && !c->stage_ok[1]) {
        if (ms) ms[v] = 1e30;  // the staged kernel does not fit this mesh
        continue;
      }
      c->var[k] = v;
      rc |= flow_restore_state(c);
      reset_run(c, 0.);
      c->timing = 0;
      rc |= enqueue_step(c, p, ts, -1, 1);  // warm-up, untimed
      cudaStreamSynchronize(c->stream);
      harvest(c);
      c->kcount[k] = 0;
      c->kms[k] = 0.;
      c->timing = 1;
      for (int i = 0; i < steps && !rc; i++) rc |= enqueue_step(c, p, ts + 1 + i, -1, 0);
      if (cudaStreamSynchronize(c->stream) != cudaSuccess) rc |= FLOW_ERR_CUDA;
      harvest(c);
      const double t = c->kcount[k] ? c->kms[k] / c->kcount[k] : 1e30;
      if (ms) ms[(k == 0 ? 0 : kNodeVariants) + v] = t;
      if (t < best_ms) {
        best_ms = t;
        best = v;
      }
    }
    c->var[k] = best;
  }
  c->timing = saved_timing;
  std::copy(kc, kc + 8, c->kcount);
  std::copy(km, km + 8, c->kms);
  // the timing steps may have run into a non-physical state; the solve that
  // follows starts from the restored state with a clear status
  cudaMemsetAsync(c->s.status, 0, sizeof(int), c->stream);
  rc |= flow_restore_state(c);
  reset_run(c, 0.);
  drop_graphs(c);
  if (variants) {
    variants[0] = c->var[0];
    variants[1] = c->var[1];
  }
  return rc & FLOW_ERR_CUDA ? rc : read_status(c);
}

int flow_autotune_sweep(flow_ctx* c, const flow_params* p, int ts, int steps, int allow_df,
                        int* choice, double* ms) {
  if (!c || !c->ok || ts < 1) return FLOW_ERR_ARG;
  if (c->precision != 3) {
    set_error("flow_autotune_sweep: precision mode 3 only");
    return FLOW_ERR_ARG;
  }
  int rc = check_params(c, p);
  if (rc) return rc;
  cudaSetDevice(c->device);
  if (steps < 1) steps = 4;
  if ((rc = flow_save_state(c))) return rc;
  if ((rc = ensure_hist(c, 1))) return rc;
  const int saved_timing = c->timing, saved_ring = c->ring, saved_df = c->sweep_df;
  long kc[8];
  double km[8];
  std::copy(c->kcount, c->kcount + 8, kc);
  std::copy(c->kms, c->kms + 8, km);
  // candidates: the three ring shapes with one launch per colour, and the
  // 64-row shape with one launch per sweep (allow_df)
  const int nc = kRingShapes + 1;
  int best = -1;
  double best_ms = 1e30;
  for (int k = 0; k < nc && !rc; k++) {
    const int shape = k < kRingShapes ? k : 0, df = k < kRingShapes ? 0 : 1;
    if (ms) ms[k] = 1e30;
    if (!c->ring_ok[shape] || (df && !allow_df)) continue;
    c->ring = shape;
    c->sweep_df = df;
    apply_ring(c);
    rc |= flow_restore_state(c);
    reset_run(c, 0.);
    c->timing = 0;
    rc |= enqueue_step(c, p, ts, -1, 1);  // warm-up, untimed
    cudaStreamSynchronize(c->stream);
    harvest(c);
    c->kcount[4] = 0;
    c->kms[4] = 0.;
    c->timing = 1;
    for (int i = 0; i < steps && !rc; i++) rc |= enqueue_step(c, p, ts + 1 + i, -1, 0);
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) rc |= FLOW_ERR_CUDA;
    harvest(c);
    const double t = c->kcount[4] ? c->kms[4] / c->kcount[4] : 1e30;
    if (ms) ms[k] = t;
    if (t < best_ms) {
      best_ms = t;
      best = k;
    }
  }
  if (best < 0) {
    c->ring = saved_ring;
    c->sweep_df = saved_df;
  } else {
    c->ring = best < kRingShapes ? best : 0;
    c->sweep_df = best < kRingShapes ? 0 : 1;
  }
  apply_ring(c);
  c->timing = saved_timing;
  std::copy(kc, kc + 8, c->kcount);
  std::copy(km, km + 8, c->kms);
  cudaMemsetAsync(c->s.status, 0, sizeof(int), c->stream);
  rc |= flow_restore_state(c);
  reset_run(c, 0.);
  drop_graphs(c);
  if (choice) *choice = ring_rows(c->ring) + (c->sweep_df ? 1000 : 0);
  return rc & FLOW_ERR_CUDA ? rc : read_status(c);
}

int flow_set_timing(flow_ctx* c, int on) {
  if (!c || !c->ok) return FLOW_ERR_ARG;
  cudaStreamSynchronize(c->stream);
  harvest(c);
  c->timing = on ? 1 : 0;
  for (int i = 0; i < 8; i++) { c->kcount[i] = 0; c->kms[i] = 0.; }
  return 0;
}

int flow_kernel_times(flow_ctx* c, long* launches, double* ms, int nclasses) {
  if (!c || !c->ok) return FLOW_ERR_ARG;
  cudaStreamSynchronize(c->stream);
  harvest(c);
  for (int i = 0; i < nclasses && i < 8; i++) {
    if (launches) launches[i] = c->kcount[i];
    if (ms) ms[i] = c->kms[i];
  }
  return 0;
}

void* flow_stream(flow_ctx* c) { return c ? (void*)c->stream : nullptr; }

int flow_status(flow_ctx* c) {
  if (!c || !c->ok) return FLOW_ERR_ARG;
  cudaSetDevice(c->device);
  return read_status(c);
}

void flow_clear_status(flow_ctx* c) {
  if (!c || !c->ok) return;
  cudaSetDevice(c->device);
  cudaMemsetAsync(c->s.status, 0, sizeof(int), c->stream);
  cudaStreamSynchronize(c->stream);
}

flow_arena* flow_arena_create(int device, long long bytes, int* status) {
  if (bytes <= 0) {
    set_error("arena size must be positive");
    if (status) *status = FLOW_ERR_ARG;
    return nullptr;
  }
  if (cudaSetDevice(device) != cudaSuccess) {
    set_error("cudaSetDevice failed");
    if (status) *status = FLOW_ERR_CUDA;
    return nullptr;
  }
  flow_arena* a = new flow_arena();
  a->device = device;
  a->size = ((size_t)bytes + 255) & ~size_t(255);
  DeviceWide gate(g_device_gate);
  if (cudaMalloc((void**)&a->base, a->size) != cudaSuccess) {
    cudaGetLastError();
    delete a;
    set_error("arena allocation failed (not enough device memory)");
    if (status) *status = FLOW_ERR_CUDA;
    return nullptr;
  }
  a->free_blocks[0] = a->size;
  if (status) *status = 0;
  return a;
}

void flow_arena_destroy(flow_arena* a) {
  if (!a) return;
  cudaSetDevice(a->device);
  DeviceWide gate(g_device_gate);
  cudaFree(a->base);
  delete a;
}

long long flow_arena_free_bytes(flow_arena* a) {
  if (!a) return -1;
  std::lock_guard<std::mutex> lock(a->mu);
  return (long long)(a->size - a->used);
}

long long flow_arena_largest_free(flow_arena* a) { return a ? (long long)a->largest_free() : -1; }

long long flow_ctx_device_bytes(flow_ctx* c) { return c ? (long long)c->buf.bytes : -1; }

long flow_launch_count(flow_ctx* c) { return c ? c->launches : 0; }

double flow_last_device_ms(flow_ctx* c) { return c ? c->last_ms : 0.; }

}  // extern "C"

// ===========================================================================
// b - A x RMS of a caller-held BCSR system, with no device allocation.
//
// For callers that cannot allocate device memory: host applications that
// hand all of a GPU's memory to their own arena or caching allocator at
// start-up (a cudaMalloc behind the arena's back fails once it holds the
// GPU, or fragments it), and time-step loops that must not take the implicit
// device-wide synchronisation that cudaMalloc and cudaFree can cause.  The
// kernels below are the per-sweep residual of flow_linear_solve
// (k_lin_residual + k_finalize_rms) with their scratch moved into one
// file-scope __device__ array: the squared residual of each row, the block
// partial sums, the RMS and an error word.  The partial sums follow
// k_lin_residual's order, so the RMS is the one flow_linear_solve returns for
// the same matrix, right-hand side and dQ.
// ===========================================================================
namespace flow {
namespace noalloc {
constexpr long kRowOff = 0;                                 // [1, nn]: |r_j|^2
constexpr long kPartOff = (long)FLOW_NOALLOC_MAX_ROWS + 1;  // kRedBlocks block sums
constexpr long kOutOff = kPartOff + kRedBlocks;             // RMS, then the error word
constexpr long kWords = ((kOutOff + 2 + 31) / 32) * 32;
constexpr int kMaxDevices = 64;
constexpr unsigned long long kBadRowPtr = 1ull, kBadColumn = 2ull;
}  // namespace noalloc
}  // namespace flow

// The scratch of flow_linear_residual_noalloc: about 2 MB per device, shared
// by every call on that device.
static __device__ __align__(256) double g_noalloc_scratch[flow::noalloc::kWords];

namespace flow {
namespace noalloc {

// Squared residual of every row; the residual itself is formed exactly as in
// k_lin_residual.  Row pointers and columns outside the system are reported
// in the error word and never dereferenced.
__global__ void __launch_bounds__(kRedThreads)
    k_rows(const int* ia, const int* ja, const double* lhs, const double* rhs, const double* x,
           int nn, long nnz, double* scratch) {
  unsigned long long* err = reinterpret_cast<unsigned long long*>(scratch + kOutOff + 1);
  for (int j = blockIdx.x * blockDim.x + threadIdx.x + 1; j <= nn;
       j += gridDim.x * blockDim.x) {
    double r[4] = {rhs[4 * (long)j], rhs[4 * (long)j + 1], rhs[4 * (long)j + 2],
                   rhs[4 * (long)j + 3]};
    const int k0 = ia[j], k1 = ia[j + 1];
    if (k0 < 0 || k1 < k0 || (long)k1 > nnz) {
      atomicOr(err, kBadRowPtr);
      scratch[kRowOff + j] = 0.;
      continue;
    }
    for (int k = k0; k < k1; k++) {
      const int c = ja[k];
      if (c < 1 || c > nn) {
        atomicOr(err, kBadColumn);
        continue;
      }
      const double d[4] = {x[4 * (long)c], x[4 * (long)c + 1], x[4 * (long)c + 2],
                           x[4 * (long)c + 3]};
      const double* A = lhs + 16 * (long)k;
#pragma unroll
      for (int q = 0; q < 4; q++) r[q] -= row_dot(A, q, d);
    }
    scratch[kRowOff + j] = (r[0] * r[0] + r[1] * r[1] + r[2] * r[2] + r[3] * r[3]);
  }
}

// Block partial sums over the same rows, in the same order, as k_lin_residual.
__global__ void __launch_bounds__(kRedThreads) k_partials(int nn, double* scratch) {
  __shared__ double sh[kRedThreads];
  double acc = 0.;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x + 1; j <= nn;
       j += gridDim.x * blockDim.x)
    acc += scratch[kRowOff + j];
  double tot = block_sum(acc, sh);
  if (threadIdx.x == 0) scratch[kPartOff + blockIdx.x] = tot;
}

// The RMS from the partials, as k_finalize_rms forms it.
__global__ void __launch_bounds__(kRedThreads) k_rms(int nn, double* scratch) {
  __shared__ double sh[kRedThreads];
  double v = 0.;
  for (int i = threadIdx.x; i < kRedBlocks; i += blockDim.x) v += scratch[kPartOff + i];
  double tot = block_sum(v, sh);
  if (threadIdx.x == 0) {
    double rms = tot / (1. * nn);
    rms = sqrt(rms);
    scratch[kOutOff] = rms;
  }
}

std::mutex g_mu;
bool g_loaded[kMaxDevices] = {};

// Device address of the scratch array on device `dev` (the current device).
// It is looked up on every call, so a module reloaded after cudaDeviceReset
// is followed; the first call on a device loads the module, under the device
// gate (loading may synchronise the device), later lookups allocate nothing.
double* scratch_for(int dev, int* rc) {
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("flow_linear_residual_noalloc: device ordinal outside 0..63");
    *rc = FLOW_ERR_ARG;
    return nullptr;
  }
  double* ptr = nullptr;
  cudaError_t e = cudaSuccess;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_loaded[dev]) {
      DeviceWide gate(g_device_gate);
      e = cudaGetSymbolAddress((void**)&ptr, g_noalloc_scratch);
      g_loaded[dev] = e == cudaSuccess;
    }
  }
  if (e == cudaSuccess && !ptr) e = cudaGetSymbolAddress((void**)&ptr, g_noalloc_scratch);
  if (e != cudaSuccess || !ptr) {
    set_error((std::string("flow_linear_residual_noalloc: cudaGetSymbolAddress failed: ") +
               cudaGetErrorString(e)).c_str());
    *rc = FLOW_ERR_CUDA;
    return nullptr;
  }
  return ptr;
}

}  // namespace noalloc
}  // namespace flow

extern "C" int flow_linear_residual_noalloc(const int* ia, const int* ja, const double* lhs,
                                            const double* rhs, const double* x, int nn,
                                            long nnz, void* stream, double* rms) {
  using namespace flow::noalloc;
  if (!ia || !ja || !lhs || !rhs || !x || !rms) {
    set_error("flow_linear_residual_noalloc: null argument");
    return FLOW_ERR_ARG;
  }
  if (nn < 1 || nn > FLOW_NOALLOC_MAX_ROWS) {
    char msg[160];
    snprintf(msg, sizeof msg,
             "flow_linear_residual_noalloc: nn = %d rows is outside 1..%d, the rows its static "
             "scratch holds",
             nn, FLOW_NOALLOC_MAX_ROWS);
    set_error(msg);
    return FLOW_ERR_ARG;
  }
  if (nnz < 0 || nnz > 0x7fffffffL) {
    set_error("flow_linear_residual_noalloc: nnz outside 0..2^31-1");
    return FLOW_ERR_ARG;
  }
  if (((uintptr_t)ia | (uintptr_t)ja) % sizeof(int) ||
      ((uintptr_t)lhs | (uintptr_t)rhs | (uintptr_t)x) % sizeof(double)) {
    set_error("flow_linear_residual_noalloc: misaligned device pointer");
    return FLOW_ERR_ARG;
  }
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    set_error(cudaGetErrorString(e));
    return FLOW_ERR_CUDA;
  }
  int rc = 0;
  double* scratch = scratch_for(dev, &rc);
  if (!scratch) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // The error word must start at zero; every other word this call reads, it
  // writes first.
  e = cudaMemsetAsync(scratch + kOutOff + 1, 0, sizeof(double), st);
  if (e == cudaSuccess) {
    k_rows<<<flow::kRedBlocks, flow::kRedThreads, 0, st>>>(ia, ja, lhs, rhs, x, nn, nnz,
                                                           scratch);
    k_partials<<<flow::kRedBlocks, flow::kRedThreads, 0, st>>>(nn, scratch);
    k_rms<<<1, flow::kRedThreads, 0, st>>>(nn, scratch);
    e = cudaGetLastError();
  }
  double out[2] = {0., 0.};
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, scratch + kOutOff, sizeof out,
                                            cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    set_error((std::string("flow_linear_residual_noalloc: ") + cudaGetErrorString(e)).c_str());
    return FLOW_ERR_CUDA;
  }
  unsigned long long err = 0;
  memcpy(&err, &out[1], sizeof err);
  if (err) {
    set_error(err & kBadRowPtr
                  ? "flow_linear_residual_noalloc: a row pointer ia[j] lies outside 0..nnz"
                  : "flow_linear_residual_noalloc: a column index ja[k] lies outside 1..nn");
    return FLOW_ERR_ARG;
  }
  *rms = out[0];
  return FLOW_OK;
}

// ===========================================================================
// Hooks for the serving engine (flow_internal.h).
// ===========================================================================
namespace flow {
namespace internal {

int begin_run(flow_ctx* c, const flow_params* p, double drop) {
  if (!c || !c->ok) return FLOW_ERR_ARG;
  int rc = check_params(c, p);
  if (rc) return rc;
  cudaSetDevice(c->device);
  if ((rc = ensure_hist(c, 1))) return rc;
  if (!c->h_run) {
    DeviceWide gate(g_device_gate);
    if (cudaHostAlloc(&c->h_run, 6 * sizeof(int), cudaHostAllocDefault) != cudaSuccess ||
        cudaHostAlloc(&c->h_runr, 4 * sizeof(double), cudaHostAllocDefault) != cudaSuccess) {
      set_error("pinned flag allocation failed");
      return FLOW_ERR_CUDA;
    }
    for (auto& e : c->ev_run)
      if (cudaEventCreate(&e) != cudaSuccess) return FLOW_ERR_CUDA;
  }
  for (int i = 0; i < 6; i++) c->h_run[i] = 0;
  reset_run(c, drop);
  if (cudaEventRecord(c->ev0, c->stream) != cudaSuccess) return FLOW_ERR_CUDA;
  return 0;
}

int enqueue_steps(flow_ctx* c, const flow_params* p, int ts0, int K) {
  if (!c || !c->ok || K < 1) return FLOW_ERR_ARG;
  cudaSetDevice(c->device);
  if (ts0 == 1) {
    int rc = 0;
    for (int i = 0; i < K && !rc; i++) rc |= enqueue_step(c, p, ts0 + i, -1, i == 0);
    return rc;
  }
  return enqueue_chunk(c, p, ts0, K);
}

int post_flags(flow_ctx* c, int slot) {
  int* h = c->h_run + 3 * slot;
  cudaMemcpyAsync(h, c->s.stop, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
  cudaMemcpyAsync(h + 1, c->s.status, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
  cudaMemcpyAsync(h + 2, c->s.steps_done, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
  double* hr = c->h_runr + 2 * slot;
  cudaMemcpyAsync(hr, c->s.scalars + 2, sizeof(double), cudaMemcpyDeviceToHost, c->stream);
  cudaMemcpyAsync(hr + 1, c->s.scalars + 6, sizeof(double), cudaMemcpyDeviceToHost, c->stream);
  if (cudaEventRecord(c->ev_run[slot], c->stream) != cudaSuccess) return FLOW_ERR_CUDA;
  return 0;
}

int flags_ready(flow_ctx* c, int slot, int* stop, int* status, int* steps, double* r_rel) {
  cudaError_t e = cudaEventQuery(c->ev_run[slot]);
  if (e == cudaErrorNotReady) return 0;
  if (e != cudaSuccess) {
    set_error(cudaGetErrorString(e));
    return -1;
  }
  const int* h = c->h_run + 3 * slot;
  *stop = h[0];
  *status = h[1];
  *steps = h[2];
  const double* hr = c->h_runr + 2 * slot;
  *r_rel = hr[1] > 0. ? sqrt(hr[0]) / hr[1] : 1.;
  return 1;
}

double run_ms(flow_ctx* c, int slot) {
  float ms = 0.f;
  cudaEventElapsedTime(&ms, c->ev0, c->ev_run[slot]);
  return ms;
}

int run_norms(flow_ctx* c, double* r_first, double* r_last) {
  double sc[8];
  if (cudaMemcpyAsync(sc, c->s.scalars, sizeof(sc), cudaMemcpyDeviceToHost, c->stream) !=
          cudaSuccess ||
      cudaStreamSynchronize(c->stream) != cudaSuccess)
    return FLOW_ERR_CUDA;
  *r_first = sc[6];
  *r_last = sqrt(sc[2]);
  return 0;
}

int checkpoint_enable(flow_ctx* c) {
  if (!c || !c->ok) return FLOW_ERR_ARG;
  if (c->ckpt[0]) return 0;
  const size_t nq = 4 * (size_t)(c->nn + c->ng + 1);
  double* a = c->buf.alloc<double>(nq);
  double* b = a ? c->buf.alloc<double>(nq) : nullptr;
  if (!a || !b) {
    set_error("checkpoint allocation failed");
    return carve_error(c);
  }
  c->ckpt[0] = a;
  c->ckpt[1] = b;
  return 0;
}

int checkpoint_save(flow_ctx* c, int slot) {
  if (!c->ckpt[slot]) return 0;
  const size_t bytes = sizeof(double) * 4 * (size_t)(c->nn + c->ng + 1);
  return cudaMemcpyAsync(c->ckpt[slot], c->s.Q, bytes, cudaMemcpyDeviceToDevice, c->stream) ==
                 cudaSuccess
             ? 0
             : FLOW_ERR_CUDA;
}

int checkpoint_restore(flow_ctx* c, int slot, int step) {
  if (!c || !c->ok || !c->ckpt[slot] || step < 1) return FLOW_ERR_ARG;
  cudaSetDevice(c->device);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) {
    set_error(cudaGetErrorString(cudaGetLastError()));
    return FLOW_ERR_CUDA;
  }
  const size_t bytes = sizeof(double) * 4 * (size_t)(c->nn + c->ng + 1);
  // the step counters as they stood before `step`: the device-side step
  // index of graph replays continues from citer, and steps_done == 0 makes
  // step 1 the run's first again
  const int before = step - 1;
  bool ok = cudaMemcpyAsync(c->s.Q, c->ckpt[slot], bytes, cudaMemcpyDeviceToDevice,
                            c->stream) == cudaSuccess &&
            cudaMemcpyAsync(c->s.nQ, c->s.Q, bytes, cudaMemcpyDeviceToDevice, c->stream) ==
                cudaSuccess &&
            cudaMemcpyAsync(c->s.citer, &before, sizeof(int), cudaMemcpyHostToDevice,
                            c->stream) == cudaSuccess &&
            cudaMemcpyAsync(c->s.steps_done, &before, sizeof(int), cudaMemcpyHostToDevice,
                            c->stream) == cudaSuccess &&
            cudaMemsetAsync(c->s.status, 0, sizeof(int), c->stream) == cudaSuccess &&
            cudaMemsetAsync(c->s.stop, 0, sizeof(int), c->stream) == cudaSuccess &&
            cudaMemsetAsync(c->s.skip, 0, sizeof(int), c->stream) == cudaSuccess;
  // the first k=2 boundary pass rewrites the curved-wall normals
  if (ok && step == 1)
    ok = cudaMemcpyAsync(c->s.xn_bedges, c->xnb0, sizeof(double) * 3 * (size_t)(c->nbe + 1),
                         cudaMemcpyDeviceToDevice, c->stream) == cudaSuccess;
  if (!ok || cudaStreamSynchronize(c->stream) != cudaSuccess) {
    set_error(cudaGetErrorString(cudaGetLastError()));
    return FLOW_ERR_CUDA;
  }
  return 0;
}

cudaStream_t stream_of(flow_ctx* c) { return c->stream; }
int device_of(flow_ctx* c) { return c->device; }
int jacobian_of(flow_ctx* c) { return c && c->ok && c->precision != 0 ? c->jac_mode : 0; }
int state_of(flow_ctx* c, const double** Q, int* nn, int* ng) {
  if (!c || !c->ok) return FLOW_ERR_ARG;
  *Q = c->s.Q;
  *nn = c->nn;
  *ng = c->ng;
  return 0;
}
void set_last_error(const char* msg) { set_error(msg); }
int step_position(flow_ctx* c, int* citer, double* cfl) {
  if (!c || !c->ok) return FLOW_ERR_ARG;
  cudaSetDevice(c->device);
  if (!download(c, citer, c->s.citer, sizeof(int)) || !download(c, cfl, c->s.scalars + 3, sizeof(double)))
    return FLOW_ERR_CUDA;
  return 0;
}

}  // namespace internal
}  // namespace flow
