// flow_serve.cu - continuous-batching engine for steady solves on one GPU.
//
// A server owns an arena (one device allocation) and a table of slots.  A
// submitted solve becomes a context carved from the arena with its own
// stream; the server keeps up to two chunks of pseudo-time steps in flight
// per running solve (CUDA-graph replays after the first chunk), reads each
// chunk's {stop, status, steps} back through pinned memory without blocking,
// and retires a solve when its density residual dropped by the requested
// factor (the stop flag is raised on the device, so steps queued behind the
// converged one do no work), when it reached its step limit, or on an error.
// Solves of different meshes, orders, flow conditions and precisions run
// side by side; each one's arithmetic is that of a context run alone, so its
// result does not depend on what else is admitted.
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <map>
#include <mutex>
#include <tuple>
#include <string>
#include <thread>
#include <vector>

#include "flow_gpu.h"
#include "flow_internal.h"

namespace {

thread_local std::string g_serve_error;

// Autotuned kernel variants by (device, order, precision, mesh-size bucket),
// kept for the process and shared by every server: the variants give
// bit-identical results and their speed depends only on the device and the
// mesh, so a choice measured once holds for every later admission.
std::mutex g_tuned_mutex;
struct Tuned {
  int node = -1, flux = -1;  // kernel variants (flow_autotune)
  int sweep = 0;             // mode 3 sweep shape (flow_autotune_sweep), 0: not tuned
};
std::map<std::tuple<int, int, int, int>, Tuned> g_tuned;
// one tuning run at a time, so that concurrent admissions do not time their
// variants against each other's kernels
std::mutex g_tuning_run_mutex;

struct Slot {
  flow_ctx* ctx = nullptr;
  flow_params p{};
  double drop = 0.;
  int max_steps = 0;
  long long tag = 0;
  int state = 0;       // 0 free, 1 running, 2 finished (result not yet released), 3 staged,
                       // 4 reserved by a stage call still building its context
  int issued = 0;      // steps enqueued so far
  int inflight = 0;    // chunks whose flags have not been read (0..2)
  int next_flag = 0;   // flag slot of the next chunk
  int oldest_flag = 0; // flag slot of the oldest chunk in flight
  int status = 0, steps = 0;
  double r_first = 0., r_last = 0., ms = 0.;
  double best = 1.;     // best ||R_rho|| relative to the first step, kept by the stall factor
  int best_step = 0;    // step at which it last improved by that factor
  int stall_window = 0; // steps without such an improvement that retire it (0: never)
  int chunk_first[2] = {0, 0};  // first step of the chunk posting each flag slot
  int recoverable = 0;  // approximate face Jacobians with chunk checkpoints kept
  int recovered_at = 0; // step it went back to with the forward-difference Jacobians
};

}  // namespace

struct flow_server {
  flow_arena* arena = nullptr;
  int device = 0;
  int chunk = 32;
  std::vector<Slot> slots;
  int running = 0;
  int autotune_steps = 0;  // 0: no autotuning at admission
  int stall_steps = 0;     // 0: no stall retirement; else the window (its minimum with a rule)
  double stall_drop = 10.;       // the improvement the best residual must make within the window
  double stall_per_sqrt = 0.;    // window steps per square root of the mesh's nodes (0: fixed)
  int sched_sweeps = 0, sched_until = 0;  // sweep schedule of precision-form solves
  long sched_min_nodes = 0;               // ... on meshes of at least this many nodes
  int priority_policy = 0;                // 1: larger meshes get greater stream priority
  int jacobian = 0;                       // face Jacobians of precision-form solves
  int recovery = 1;                       // roll back a failed approximate-Jacobian solve
  // guards the slot table and the counters: stage may run on several host
  // threads at once (each builds its context outside the lock) beside
  // progress / start / result / release
  std::mutex mu;
};

namespace {

void finish(Slot& sl, int status, int steps, int flag_slot) {
  sl.state = 2;
  sl.steps = steps;
  sl.status = status;
  sl.ms = flow::internal::run_ms(sl.ctx, flag_slot);
  flow::internal::run_norms(sl.ctx, &sl.r_first, &sl.r_last);
}

// Queue one more chunk of steps for a running slot.
int issue_chunk(flow_server* sv, Slot& sl) {
  const int K = std::min(sv->chunk, sl.max_steps - sl.issued);
  if (K <= 0) return 0;
  int rc = sl.recoverable ? flow::internal::checkpoint_save(sl.ctx, sl.next_flag) : 0;
  if (rc) return rc;
  sl.chunk_first[sl.next_flag] = 1 + sl.issued;
  rc = flow::internal::enqueue_steps(sl.ctx, &sl.p, 1 + sl.issued, K);
  if (rc) return rc;
  sl.issued += K;
  rc = flow::internal::post_flags(sl.ctx, sl.next_flag);
  if (rc) return rc;
  sl.next_flag ^= 1;
  sl.inflight++;
  return 0;
}

// Error bits of a state that went non-physical (a negative pressure or
// density on the way to a wave speed, dt, the limiter or a far-field state).
constexpr int kNonPhysical = FLOW_ERR_EIGEN | FLOW_ERR_DT | FLOW_ERR_LIMITER | FLOW_ERR_BC;

// A solve on the approximate face Jacobians whose chunk (flag slot fs) ended
// non-physical: the approximation's Newton steps can overshoot where the CFL
// ramp makes them large.  Put back the state of that chunk's first step and
// carry on from there with the forward-difference Jacobians (the reference's
// derivatives of the flux the residual uses), once per solve.  The steps
// after the failure are run once more; they count in the solve's device
// time.
int recover(flow_server* sv, Slot& sl, int fs) {
  const int step = sl.chunk_first[fs];
  int rc = flow::internal::checkpoint_restore(sl.ctx, fs, step);
  if (!rc) rc = flow_set_jacobian(sl.ctx, 0);
  if (rc) return rc;
  sl.recoverable = 0;
  sl.recovered_at = step;
  sl.issued = step - 1;
  sl.inflight = 0;
  sl.next_flag = sl.oldest_flag = 0;
  rc = issue_chunk(sv, sl);
  if (!rc) rc = issue_chunk(sv, sl);
  return rc;
}

}  // namespace

extern "C" {

const char* flow_server_last_error(void) { return g_serve_error.c_str(); }

flow_server* flow_server_create(flow_arena* arena, int chunk, int max_slots, int* status) {
  if (!arena || max_slots < 1) {
    g_serve_error = "flow_server_create: null arena or max_slots < 1";
    if (status) *status = FLOW_ERR_ARG;
    return nullptr;
  }
  flow_server* sv = new flow_server();
  sv->arena = arena;
  sv->chunk = chunk > 0 ? chunk : 32;
  sv->slots.resize(max_slots);
  if (status) *status = 0;
  return sv;
}

void flow_server_destroy(flow_server* sv) {
  if (!sv) return;
  for (auto& sl : sv->slots)
    if (sl.ctx) flow_destroy(sl.ctx);
  delete sv;
}

static int start_slot(flow_server* sv, int idx);

int flow_server_submit(flow_server* sv, const flow_grid_view* g, const flow_params* p,
                       const double* Q0, int precision, double drop, int max_steps,
                       long long tag, int* slot_out) {
  return flow_server_stage(sv, g, p, Q0, precision, drop, max_steps, tag, 0, slot_out);
}

int flow_server_stage(flow_server* sv, const flow_grid_view* g, const flow_params* p,
                      const double* Q0, int precision, double drop, int max_steps,
                      long long tag, int hold, int* slot_out) {
  if (!sv || !g || !p || !Q0 || !(drop > 0.) || max_steps < 1) {
    g_serve_error = "flow_server_submit: bad argument";
    return FLOW_ERR_ARG;
  }
  int idx = -1;
  int autotune_steps = 0, sched_sweeps = 0, sched_until = 0, priority_policy = 0, jacobian = 0;
  int recovery = 0, stall_steps = 0;
  double stall_per_sqrt = 0.;
  long sched_min_nodes = 0;
  {
    std::lock_guard<std::mutex> lock(sv->mu);
    for (int i = 0; i < (int)sv->slots.size(); i++)
      if (sv->slots[i].state == 0) { idx = i; break; }
    if (idx < 0) {
      g_serve_error = "flow_server_submit: every slot is busy";
      return FLOW_ERR_BUDGET;
    }
    sv->slots[idx].state = 4;  // reserved: the context is built outside the lock
    autotune_steps = sv->autotune_steps;
    sched_sweeps = sv->sched_sweeps;
    sched_until = sv->sched_until;
    sched_min_nodes = sv->sched_min_nodes;
    priority_policy = sv->priority_policy;
    jacobian = sv->jacobian;
    recovery = sv->recovery;
    stall_steps = sv->stall_steps;
    stall_per_sqrt = sv->stall_per_sqrt;
  }
  auto unreserve = [&]() {
    std::lock_guard<std::mutex> lock(sv->mu);
    sv->slots[idx] = Slot();
  };
  int st = 0;
  flow_ctx* c = flow_create_in(sv->arena, g, p, &st);
  if (!c) {
    // FLOW_ERR_BUDGET (the arena has no room now: retry after a release) is
    // kept apart from a CUDA error, which retrying does not cure
    g_serve_error = std::string("flow_server_submit: ") + flow_last_error();
    unreserve();
    return st ? st : FLOW_ERR_ARG;
  }
  int rc = flow_set_precision(c, precision);
  // mode 3 needs its chunk windows in shared memory; a mesh whose matrix
  // bandwidth is too large for that is served in mode 1 instead
  if (rc == FLOW_ERR_ARG && precision == 3) rc = flow_set_precision(c, 1);
  if (!rc && precision != 0 && jacobian != 0) rc = flow_set_jacobian(c, jacobian);
  const int recoverable = !rc && recovery && flow::internal::jacobian_of(c) != 0;
  if (recoverable) rc = flow::internal::checkpoint_enable(c);
  if (!rc && precision != 0 && sched_sweeps > 0 && flow_size(c, "dt") - 1 >= sched_min_nodes)
    rc = flow_set_sweep_schedule(c, sched_sweeps, sched_until);
  if (!rc && priority_policy == 1) {
    // greatest priority from 256k nodes, one step down per halving of the mesh
    const long nn = flow_size(c, "dt") - 1;
    int steps_down = 0;
    for (long t = 262144; nn < t && steps_down < 8; t >>= 1) steps_down++;
    int lo = 0, hi = 0;
    cudaDeviceGetStreamPriorityRange(&lo, &hi);
    rc = flow_set_stream_priority(c, std::min(lo, hi + steps_down));
  }
  if (!rc) rc = flow_set_state(c, Q0);
  if (!rc && autotune_steps > 0) {
    // kernel variants: measured once per (device, order, precision, size bucket)
    const long nn = flow_size(c, "dt") - 1;
    const int bucket = (int)std::floor(2.0 * std::log2((double)std::max(nn, 1L)));
    const auto key = std::make_tuple(flow::internal::device_of(c), p->order, precision, bucket);
    auto lookup = [&]() {
      std::lock_guard<std::mutex> lock(g_tuned_mutex);
      auto it = g_tuned.find(key);
      return it != g_tuned.end() ? it->second : Tuned();
    };
    Tuned found = lookup();
    std::unique_lock<std::mutex> run_lock(g_tuning_run_mutex, std::defer_lock);
    if (found.node < 0) {
      run_lock.lock();
      found = lookup();  // another admission may have tuned this bucket meanwhile
    }
    const int mode = flow_precision_of(c);
    if (found.node >= 0) {
      rc = flow_set_variants(c, found.node, found.flux);
      if (!rc && mode == 3 && found.sweep > 0) {
        rc = flow_set_sweep_ring(c, found.sweep % 1000);
        if (!rc && found.sweep >= 1000) rc = flow_set_sweep_dataflow(c, 1);
      }
    } else {
      Tuned t;
      int v[2] = {0, 0};
      int trc = flow_autotune(c, p, 1, autotune_steps, v, nullptr);
      t.node = v[0];
      t.flux = v[1];
      if (!(trc & FLOW_ERR_CUDA) && mode == 3)
        trc |= flow_autotune_sweep(c, p, 1, autotune_steps, 0, &t.sweep, nullptr);
      if (trc & FLOW_ERR_CUDA) {
        rc = trc;  // other bits: the tuning steps' physics, not fatal
      } else {
        std::lock_guard<std::mutex> lock(g_tuned_mutex);
        g_tuned[key] = t;
      }
    }
  }
  if (rc) {
    // the precision tables carved from the arena may not fit (FLOW_ERR_BUDGET);
    // every other failure is returned as it is
    g_serve_error = std::string("flow_server_submit: ") + flow_last_error();
    flow_destroy(c);
    unreserve();
    return rc;
  }
  // the stall window of this solve: the fixed window, or the rule's
  // steps per square root of the mesh's nodes (at least the fixed window),
  // rounded up to whole chunks
  int stall_window = stall_steps;
  if (stall_steps > 0 && stall_per_sqrt > 0.) {
    const double nn = (double)(flow_size(c, "dt") - 1);
    const int chunk = sv->chunk;
    const int w = (int)std::ceil(stall_per_sqrt * std::sqrt(std::max(nn, 1.)) / chunk) * chunk;
    stall_window = std::max(stall_steps, w);
  }
  std::lock_guard<std::mutex> lock(sv->mu);
  Slot& sl = sv->slots[idx];
  sl = Slot();
  sl.ctx = c;
  sl.p = *p;
  sl.drop = drop;
  sl.max_steps = max_steps;
  sl.tag = tag;
  sl.recoverable = recoverable;
  sl.stall_window = stall_window;
  sl.state = 3;  // staged: inputs on the device, nothing launched
  if (slot_out) *slot_out = idx;
  if (hold) return 0;
  return start_slot(sv, idx);
}

static int start_slot(flow_server* sv, int idx) {
  Slot& sl = sv->slots[idx];
  if (sl.state != 3) {
    g_serve_error = "flow_server_start: slot is not staged";
    return FLOW_ERR_ARG;
  }
  // the run's clock starts here
  int rc = flow::internal::begin_run(sl.ctx, &sl.p, sl.drop);
  sl.state = 1;
  sv->running++;
  // two chunks in flight from the start
  if (!rc) rc = issue_chunk(sv, sl);
  if (!rc) rc = issue_chunk(sv, sl);
  if (rc) {
    // nothing of this solve is in flight: the caller learns of the failure
    // here (not through progress) and releases the slot
    if (sl.inflight > 0) cudaStreamSynchronize(flow::internal::stream_of(sl.ctx));
    sl.inflight = 0;
    sl.state = 2;
    sl.status = rc;
    sv->running--;
    g_serve_error = std::string("flow_server_start: ") + flow_last_error();
  }
  return rc;
}

int flow_server_start(flow_server* sv, int slot) {
  if (!sv || slot < 0 || slot >= (int)sv->slots.size()) return FLOW_ERR_ARG;
  std::lock_guard<std::mutex> lock(sv->mu);
  return start_slot(sv, slot);
}

int flow_server_progress(flow_server* sv, int wait_us, flow_completion* out, int max_out,
                         int* nout) {
  if (!sv || (max_out > 0 && !out)) return FLOW_ERR_ARG;
  int n = 0;
  const auto t0 = std::chrono::steady_clock::now();
  for (;;) {
    bool any = false;
    std::unique_lock<std::mutex> lock(sv->mu);
    for (int i = 0; i < (int)sv->slots.size() && n < max_out; i++) {
      Slot& sl = sv->slots[i];
      if (sl.state != 1) continue;
      int stop = 0, status = 0, steps = 0;
      double rr = 1.;
      int r = flow::internal::flags_ready(sl.ctx, sl.oldest_flag, &stop, &status, &steps, &rr);
      if (r == 0) continue;
      any = true;
      if (r < 0) status = FLOW_ERR_CUDA;
      const int fs = sl.oldest_flag;
      sl.oldest_flag ^= 1;
      sl.inflight--;
      if (r > 0 && sl.recoverable && !stop && status && !(status & ~kNonPhysical)) {
        const int rc = recover(sv, sl, fs);
        if (!rc) continue;  // running again from the failed chunk's first step
        status |= rc;
      }
      // stall: the best residual has not dropped by the stall factor within
      // the solve's window
      if (rr < sl.best / sv->stall_drop) {
        sl.best = rr;
        sl.best_step = steps;
      }
      if (!stop && !status && sl.stall_window > 0 && steps - sl.best_step >= sl.stall_window)
        status = FLOW_ERR_STALLED;
      bool done = stop || status || (sl.issued >= sl.max_steps && sl.inflight == 0);
      if (done) {
        // let the chunk still in flight (no-op steps after the stop) drain
        if (sl.inflight > 0) cudaStreamSynchronize(flow::internal::stream_of(sl.ctx));
        sl.inflight = 0;
        finish(sl, status ? status : (stop ? 0 : FLOW_ERR_NOT_CONVERGED), steps, fs);
        sv->running--;
        flow_completion& cpl = out[n++];
        cpl.tag = sl.tag;
        cpl.slot = i;
        cpl.status = sl.status;
        cpl.steps = sl.steps;
        cpl.r_first = sl.r_first;
        cpl.r_last = sl.r_last;
        cpl.device_ms = sl.ms;
        cpl.launches = flow_launch_count(sl.ctx);
        cpl.recovered_at = sl.recovered_at;
        continue;
      }
      if (sl.issued < sl.max_steps) {
        int rc = issue_chunk(sv, sl);
        if (rc) {
          if (sl.inflight > 0) cudaStreamSynchronize(flow::internal::stream_of(sl.ctx));
          sl.inflight = 0;
          finish(sl, rc, steps, fs);
          sv->running--;
          flow_completion& cpl = out[n++];
          cpl.tag = sl.tag;
          cpl.slot = i;
          cpl.status = rc;
          cpl.steps = steps;
          cpl.r_first = sl.r_first;
          cpl.r_last = sl.r_last;
          cpl.device_ms = sl.ms;
          cpl.launches = flow_launch_count(sl.ctx);
        cpl.recovered_at = sl.recovered_at;
        }
      }
    }
    const int running = sv->running;
    lock.unlock();
    if (n > 0 || wait_us <= 0 || running == 0) break;
    const auto dt = std::chrono::duration_cast<std::chrono::microseconds>(
                        std::chrono::steady_clock::now() - t0)
                        .count();
    if (dt >= wait_us) break;
    if (!any) std::this_thread::sleep_for(std::chrono::microseconds(20));
  }
  if (nout) *nout = n;
  return 0;
}

int flow_server_result(flow_server* sv, int slot, double* Q, long nQ, double* forces) {
  if (!sv || slot < 0 || slot >= (int)sv->slots.size()) return FLOW_ERR_ARG;
  std::lock_guard<std::mutex> lock(sv->mu);
  Slot& sl = sv->slots[slot];
  if (sl.state != 2 || !sl.ctx) {
    g_serve_error = "flow_server_result: slot has no finished solve";
    return FLOW_ERR_ARG;
  }
  int rc = 0;
  if (Q) rc |= flow_get(sl.ctx, "Q", Q, nQ);
  if (forces) rc |= flow_body_forces(sl.ctx, &sl.p, forces);
  return rc;
}

int flow_server_release(flow_server* sv, int slot) {
  if (!sv || slot < 0 || slot >= (int)sv->slots.size()) return FLOW_ERR_ARG;
  std::lock_guard<std::mutex> lock(sv->mu);
  Slot& sl = sv->slots[slot];
  if (sl.state == 1 || sl.state == 4) {
    g_serve_error = "flow_server_release: the solve is still running or being staged";
    return FLOW_ERR_ARG;
  }
  if (sl.ctx) flow_destroy(sl.ctx);
  sl = Slot();
  return 0;
}

int flow_server_running(flow_server* sv) {
  if (!sv) return -1;
  std::lock_guard<std::mutex> lock(sv->mu);
  return sv->running;
}

int flow_server_set_sweep_schedule(flow_server* sv, int sweeps, int until_step,
                                   long long min_nodes) {
  if (!sv || sweeps < 0 || until_step < 0 || min_nodes < 0) return FLOW_ERR_ARG;
  std::lock_guard<std::mutex> lock(sv->mu);
  sv->sched_sweeps = sweeps;
  sv->sched_until = until_step;
  sv->sched_min_nodes = (long)min_nodes;
  return 0;
}

int flow_server_set_priority_policy(flow_server* sv, int policy) {
  if (!sv || policy < 0 || policy > 1) return FLOW_ERR_ARG;
  std::lock_guard<std::mutex> lock(sv->mu);
  sv->priority_policy = policy;
  return 0;
}

int flow_server_set_stall_rule(flow_server* sv, double drop, double steps_per_sqrt_node) {
  if (!sv || !(drop > 1.) || !(steps_per_sqrt_node >= 0.)) return FLOW_ERR_ARG;
  std::lock_guard<std::mutex> lock(sv->mu);
  sv->stall_drop = drop;
  sv->stall_per_sqrt = steps_per_sqrt_node;
  return 0;
}

int flow_server_set_stall(flow_server* sv, int steps) {
  if (!sv || steps < 0) return FLOW_ERR_ARG;
  std::lock_guard<std::mutex> lock(sv->mu);
  sv->stall_steps = steps;
  return 0;
}

int flow_server_set_jacobian(flow_server* sv, int mode) {
  if (!sv || mode < 0 || mode > 2) return FLOW_ERR_ARG;
  std::lock_guard<std::mutex> lock(sv->mu);
  sv->jacobian = mode;
  return 0;
}

int flow_server_set_recovery(flow_server* sv, int on) {
  if (!sv) return FLOW_ERR_ARG;
  std::lock_guard<std::mutex> lock(sv->mu);
  sv->recovery = on ? 1 : 0;
  return 0;
}

int flow_server_set_autotune(flow_server* sv, int steps) {
  if (!sv || steps < 0) return FLOW_ERR_ARG;
  std::lock_guard<std::mutex> lock(sv->mu);
  sv->autotune_steps = steps;
  return 0;
}

}  // extern "C"
