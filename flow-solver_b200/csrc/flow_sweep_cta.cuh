// flow_sweep_cta.cuh - ordered block Gauss-Seidel sweep, one CTA per mesh.
//
// Same arithmetic as k_sweep_ordered (linear_algebra.C:178-344, the reference's
// sequential row order), organised so that no global-memory round trip sits
// on the row-to-row dependency chain:
//   * warp 0 streams the matrix in "stages" (consecutive rows whose blocks
//     fit in one buffer) into a shared-memory ring with cp.async.bulk,
//     completion tracked by one mbarrier per ring slot;
//   * warps 1..31 each run 8 rows at a time, 4 lanes per row (one per
//     matrix row of the 4x4 blocks); row positions are dealt round-robin to
//     the 248 lane groups in the reference's order, and each finished dQ is
//     published in a shared-memory window slot tagged with its row number;
//     a row waits only for the window tags of the neighbours the reference
//     updates before it;
//   * a ring slot is refilled once every row of its previous stage is done.
// Progress: rows only wait for earlier rows, stage t+NS is loaded only after
// stage t finished, and the window is larger than the matrix bandwidth plus
// the rows that can be in flight, so no slot is reused while still needed.
// Every wait is bounded and reports ERR_SWEEP_TIMEOUT instead of hanging.
#pragma once
#include <stdint.h>
#include "flow_kernels.cuh"

namespace flow {

constexpr int kStageBlocks = 192;   // 24 KB of 4x4 FP64 blocks per stage
constexpr int kStageRows = 32;      // at most 32 rows per stage
constexpr int kStages = 6;          // ring depth
constexpr int kWindow = 1024;       // dQ window rows (power of two)
constexpr int kSweepThreads = 1024; // 1 producer warp + 31 row warps

struct SweepTables {
  const int* stage_row0;   // T+1: first row of each stage (rows ascending)
  const int* row_stage;    // nn+1: stage of each row
  const int* ja_pad;       // ja with 16 zero entries of padding at the end
  int nstages;
};

struct __align__(16) StageSlot {
  double lhs[kStageBlocks * 16];
  double lud[kStageRows * 16];
  double rhs[kStageRows * 4];
  int ja[kStageBlocks + 8];
};

struct SweepSmem {
  StageSlot slot[kStages];
  double win[kWindow * 4];
  int tag[kWindow];
  int rows_done[kStages];
  int armed[kStages];      // stage index the slot was last armed for
  unsigned long long full[kStages];
  int abort;
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Global -> shared bulk copy completing on an mbarrier (16-byte aligned
// addresses, size a multiple of 16).
__device__ __forceinline__ void bulk_copy(void* dst, const void* src, uint32_t bytes,
                                          unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

template <bool FWD>
__global__ void __launch_bounds__(kSweepThreads, 1)
    k_sweep_cta(DevMesh m, DevState s, SweepTables tb, long max_spin) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  SweepSmem& sm = *reinterpret_cast<SweepSmem*>(smem_raw);
  const unsigned FULL = 0xffffffffu;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nn = m.nn, T = tb.nstages;
  if (*s.stop || *s.skip) return;

  for (int i = threadIdx.x; i < kWindow; i += blockDim.x) sm.tag[i] = -1;
  if (threadIdx.x < kStages) {
    mbar_init(&sm.full[threadIdx.x], 1);
    sm.rows_done[threadIdx.x] = 0;
    sm.armed[threadIdx.x] = -1;
  }
  if (threadIdx.x == 0) sm.abort = 0;
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  __syncthreads();

  if (warp == 0) {
    // ---------------- producer ----------------
    if (lane == 0) {
      for (int u = 0; u < T; u++) {
        const int slot = u % kStages;
        if (u >= kStages) {
          // wait until every row of the stage that occupied this slot is done
          const int tp = FWD ? (u - kStages) : (T - 1 - (u - kStages));
          const int need = tb.stage_row0[tp + 1] - tb.stage_row0[tp];
          long spins = 0;
          while (*(volatile int*)&sm.rows_done[slot] < need) {
            if (++spins > max_spin || *(volatile int*)&sm.abort) {
              atomicOr(s.status, ERR_SWEEP_TIMEOUT);
              *(volatile int*)&sm.abort = 1;
              break;
            }
          }
          if (*(volatile int*)&sm.abort) break;
          sm.rows_done[slot] = 0;
          __threadfence_block();
        }
        const int t = FWD ? u : (T - 1 - u);
        const int r0 = tb.stage_row0[t], r1 = tb.stage_row0[t + 1];
        const int b0 = m.ia[r0], b1 = m.ia[r1];
        const int j0 = b0 & ~3, j1 = (b1 + 3) & ~3;
        StageSlot& st = sm.slot[slot];
        const uint32_t bl = (uint32_t)(b1 - b0) * 128u, bu = (uint32_t)(r1 - r0) * 128u,
                       br = (uint32_t)(r1 - r0) * 32u, bj = (uint32_t)(j1 - j0) * 4u;
        mbar_expect_tx(&sm.full[slot], bl + bu + br + bj);
        bulk_copy(st.lhs, s.LHS + 16 * (long)b0, bl, &sm.full[slot]);
        bulk_copy(st.lud, s.LUd + 16 * (long)r0, bu, &sm.full[slot]);
        bulk_copy(st.rhs, s.RHS + 4 * (long)r0, br, &sm.full[slot]);
        bulk_copy(st.ja, tb.ja_pad + j0, bj, &sm.full[slot]);
        // publish which stage the slot now holds: a consumer must see this
        // before its parity wait, or it could match the slot's previous phase
        __threadfence_block();
        *(volatile int*)&sm.armed[slot] = u;
      }
    }
    return;
  }

  // ---------------- row groups: 4 lanes per row ----------------
  const int g = lane >> 2, r = lane & 3;
  const unsigned gmask = 0xFu << (4 * g);
  const int ngroups = 31 * 8;
  for (int p = (warp - 1) * 8 + g; p < nn; p += ngroups) {
    const int j = FWD ? (1 + p) : (nn - p);
    const int t = tb.row_stage[j];
    const int u = FWD ? t : (T - 1 - t);
    const int slot = u % kStages;
    const uint32_t parity = (uint32_t)((u / kStages) & 1);
    const int r0 = tb.stage_row0[t];
    const int k0 = m.ia[j], k1 = m.ia[j + 1];
    const int b0 = m.ia[r0];
    const int j0 = b0 & ~3;
    const double old_r = __ldcg(s.dQ + 4 * (long)j + r);
    bool bad = false;
    {
      long spins = 0;
      while (*(volatile int*)&sm.armed[slot] != u) {
        if (++spins > max_spin || *(volatile int*)&sm.abort) {
          atomicOr(s.status, ERR_SWEEP_TIMEOUT);
          sm.abort = 1;
          bad = true;
          break;
        }
      }
    }
    if (__any_sync(gmask, bad)) return;
    {
      long spins = 0;
      while (!mbar_try_wait(&sm.full[slot], parity)) {
        if (++spins > (max_spin >> 4) || *(volatile int*)&sm.abort) {
          atomicOr(s.status, ERR_SWEEP_TIMEOUT);
          sm.abort = 1;
          bad = true;
          break;
        }
      }
    }
    if (__any_sync(gmask, bad)) return;
    const StageSlot& st = sm.slot[slot];
    double acc = st.rhs[4 * (j - r0) + r];
    for (int k = k0; k < k1 && !bad; k++) {
      const int c = st.ja[k - j0];
      if (c == j) continue;
      if (c < 1 || c > nn) {  // a corrupt stage: report, never dereference
        atomicOr(s.status, ERR_SWEEP_TIMEOUT);
        sm.abort = 1;
        bad = true;
        break;
      }
      const double* A = st.lhs + 16 * (k - b0) + 4 * r;
      double d0, d1, d2, d3;
      const bool dep = FWD ? (c < j) : (c > j);
      if (dep) {
        const int w = c & (kWindow - 1);
        long spins = 0;
        while (*(volatile int*)&sm.tag[w] != c) {
          if (++spins > max_spin || *(volatile int*)&sm.abort) {
            atomicOr(s.status, ERR_SWEEP_TIMEOUT);
            sm.abort = 1;
            bad = true;
            break;
          }
        }
        __threadfence_block();
        const volatile double* wv = sm.win + 4 * w;
        d0 = wv[0]; d1 = wv[1]; d2 = wv[2]; d3 = wv[3];
      } else {
        const double2* dq = reinterpret_cast<const double2*>(s.dQ + 4 * (long)c);
        const double2 a = __ldcg(dq), b = __ldcg(dq + 1);
        d0 = a.x; d1 = a.y; d2 = b.x; d3 = b.y;
      }
      acc -= (A[0] * d0 + A[1] * d1 + A[2] * d2 + A[3] * d3);
    }
    if (__any_sync(gmask, bad)) return;
    double b[4], o[4], X[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      b[q] = __shfl_sync(gmask, acc, 4 * g + q);
      o[q] = __shfl_sync(gmask, old_r, 4 * g + q);
    }
    lu_solve4(st.lud + 16 * (j - r0), b, X);
    double xr = X[0], orr = o[0];
#pragma unroll
    for (int q = 1; q < 4; q++)
      if (r == q) { xr = X[q]; orr = o[q]; }
    const double dx = xr - orr;
    const double val = orr + dx;
    const int w = j & (kWindow - 1);
    ((volatile double*)sm.win)[4 * w + r] = val;
    s.dQ[4 * (long)j + r] = val;
    __syncwarp(gmask);
    if (r == 0) {
      __threadfence_block();
      *(volatile int*)&sm.tag[w] = j;
      atomicAdd(&sm.rows_done[slot], 1);
    }
    __syncwarp(gmask);
  }
}

}  // namespace flow
