// flow_internal.h - hooks of the context implementation (flow_gpu.cu) used by
// the serving engine (flow_serve.cu).  Not part of the C ABI.
#pragma once
#include <cuda_runtime.h>

#include <shared_mutex>

#include "flow_gpu.h"

namespace flow {
namespace internal {

// Process-wide gate between CUDA stream captures and calls that may
// synchronise a whole device.  A device-wide synchronisation (cudaFree,
// cudaFreeHost, cudaDeviceSynchronize, loading a kernel module) issued by one
// thread while another thread captures a chunk of steps into a CUDA graph
// invalidates that capture.  Captures hold the gate shared (several contexts
// may capture at once); the library's device-wide calls hold it exclusive.
std::shared_mutex& device_gate();

// Start a run on the context's stream: clear the stop flag and step count,
// set the target drop of ||R_rho|| and record the run's start event.
int begin_run(flow_ctx* c, const flow_params* p, double drop);
// Enqueue steps ts0 .. ts0+K-1 (ts0 == 1 starts the run); full chunks after
// the first replay the context's CUDA graphs.
int enqueue_steps(flow_ctx* c, const flow_params* p, int ts0, int K);
// Queue a read-back of {stop, status, steps done} into flag slot `slot`
// (0 or 1) of the context's pinned flags, with an event behind it.
int post_flags(flow_ctx* c, int slot);
// 1 when flag slot `slot` has arrived (values in *stop, *status, *steps and
// *r_rel = ||R_rho|| of the last step over that of the run's first),
// 0 while it is in flight, -1 on a CUDA error.
int flags_ready(flow_ctx* c, int slot, int* stop, int* status, int* steps, double* r_rel);
// Device time from the run's start to flag slot `slot` (ms).
double run_ms(flow_ctx* c, int slot);
// ||R_rho|| of the run's first step and of its last step.
int run_norms(flow_ctx* c, double* r_first, double* r_last);
cudaStream_t stream_of(flow_ctx* c);
int device_of(flow_ctx* c);
// The face Jacobians the context's steps build (flow_set_jacobian; 0 when
// the context runs the FP64 drop-in, which always takes the reference's).
int jacobian_of(flow_ctx* c);
// Chunk checkpoints of a served run: checkpoint_enable carves two copies of
// GRID::Q from the context's buffers; checkpoint_save(slot) queues a copy of
// the state into copy `slot` on the context's stream (before the chunk that
// posts flag slot `slot`; nothing when not enabled); checkpoint_restore
// waits for the stream, puts copy `slot` back as the state before step
// `step` and clears the run's error bits and stop flag, so that the next
// enqueue_steps(step, ...) runs from there.
int checkpoint_enable(flow_ctx* c);
int checkpoint_save(flow_ctx* c, int slot);
int checkpoint_restore(flow_ctx* c, int slot, int step);
// The context's resident state GRID::Q ((nn+nn_ghost+1)*4 doubles on the
// device) and its node counts; FLOW_ERR_ARG for a null or failed context.
int state_of(flow_ctx* c, const double** Q, int* nn, int* ng);
// Message returned by flow_last_error() on this thread.
void set_last_error(const char* msg);
// The pseudo-time step the context last ran (GRID::citer) and its CFL
// (GRID::cfl), read from the device after the context's work has finished.
int step_position(flow_ctx* c, int* citer, double* cfl);

}  // namespace internal
}  // namespace flow
