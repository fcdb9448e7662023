// flow_kernels.cuh - CUDA kernels of one nonlinear iteration (solve.C:44-933).
//
// One pseudo-time step is a fixed sequence of launches on the context's
// stream:
//   k_begin_step      step index and CFL, nQ <- Q, and what the node kernel
//                     will not overwrite of grad/hess <- 0, phi <- 1
//                                                               (init_memory.C:200-224,
//                                                                solve.C:298-348)
//   k_node_prepare    per node: wave-speed sum, dt and V/dt    (build_matrix)
//                     + LSQ gradient or k=2 derivatives + Venkatakrishnan phi
//   k_subedge_flux    per subedge: reconstructed Roe flux and the 8-flux
//                     forward-difference Jacobian               (residual.C, jacobian.C)
//   k_boundary        per boundary edge: ghost state, boundary flux and
//                     approximate Jacobian                      (cvbc.C, residual.C)
//   k_assemble        per node: R, RHS, the node's LHS row, LU of the diagonal
//   k_sweep_ordered   block Gauss-Seidel sweeps in reference row order
//   k_lin_residual    b - Ax RMS after a sweep                  (linear_algebra.C:348-387)
//   k_finish_step     nQ += dQ, pQ <- Q, Q <- nQ, norms, the stop flag
//                                                               (solve.C:883-928)
// (the precision form replaces the sweeps and the RMS by k_sweep_chunk /
// k_sweep_chunk_pair and its face Jacobians may be the approximate ones)
// Face results are written once per face and gathered per node in ascending
// face order, which reproduces the reference's sequential scatter sums
// exactly without atomics.
#pragma once
#include <cuda/atomic>
#include "flow_device.cuh"
#include "flow_state.h"

namespace flow {

enum : int {
  ERR_EIGEN = 4,
  ERR_DT = 8,
  ERR_LIMITER = 16,
  ERR_BC = 32,
  ERR_SWEEP_TIMEOUT = 64,
};

constexpr int kRedBlocks = 296;  // 2 x 148 SMs; fixed so reductions are deterministic
constexpr int kRedThreads = 256;

struct StepArgs {
  double gamma;
  double uinf, vinf, pinf;  // far-field state (cvbc.C:70-74)
  double cos_a, sin_a;      // angle of attack (grid_io.C:1432)
  int do_grad;              // k=1 gradient
  int do_derivs;            // k=2 derivatives
  int do_lim;               // Venkatakrishnan limiter
  int recon;                // interior reconstruction order: 0, 1 or 3
  int gauss;                // k=2 Gauss pass active (curved-boundary side effects)
  int jac;                  // Jacobian update
  int steady_diag;          // V/dt diagonal (steady runs)
  int skip_bnd;             // assembly of the interior faces only (build_interior_residuals)
};

// ---------------------------------------------------------------------------
// Step index and CFL of the step about to run (init_memory.C:200-216).
// citer > 0 sets the index; citer == 0 takes the one after the previous step,
// which lets a captured sequence of steps replay with an advancing ramp.
__device__ __forceinline__ void step_args_body(DevState& s, int citer, int method, int ramp,
                                               double CFL) {
  const int ci = citer > 0 ? citer : *s.citer + 1;
  *s.citer = ci;
  double cfl;
  if (method == 1)
    cfl = ci < ramp ? 1. + (1. * (ci - 1)) / (1. * ramp) * (CFL - 1.) : CFL;
  else if (method == 0)
    cfl = 1.0;
  else
    cfl = CFL;
  s.scalars[3] = cfl;
}
__global__ void k_step_args(DevState s, int citer, int method, int ramp, double CFL) {
  if (*s.stop) return;  // the run has converged
  step_args_body(s, citer, method, ramp, CFL);
}

// flags: kBeginCopyQ nQ <- Q; kBeginResetPhi phi <- 1; kBeginZeroGrad
// grad <- 0; kBeginZeroHess the k=2 derivatives <- 0; kBeginStepArgs the
// step index and CFL (k_step_args, by one thread; nothing else in this
// kernel reads them).  The host leaves out what the step's node kernel
// overwrites for every node anyway.
constexpr int kBeginCopyQ = 1, kBeginResetPhi = 2, kBeginZeroGrad = 4, kBeginZeroHess = 8,
              kBeginStepArgs = 16;
__global__ void k_begin_step(DevMesh m, DevState s, int flags, int citer = 0, int method = 0,
                             int ramp = 0, double CFL = 0.) {
  if (*s.stop) return;  // the run has converged
  if ((flags & kBeginStepArgs) && blockIdx.x == 0 && threadIdx.x == 0)
    step_args_body(s, citer, method, ramp, CFL);
  int total = m.nn + m.ng;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x + 1; i <= total;
       i += gridDim.x * blockDim.x) {
    if (flags & kBeginCopyQ) {
      const double4* q = reinterpret_cast<const double4*>(s.Q) + i;
      reinterpret_cast<double4*>(s.nQ)[i] = *q;
    }
    if (i <= m.nn) {
      double4 z = make_double4(0., 0., 0., 0.);
      if (flags & kBeginZeroGrad) {
        double4* g = reinterpret_cast<double4*>(s.grad) + 2 * i;
        g[0] = z;
        g[1] = z;
      }
      if (m.order == 3 && (flags & kBeginZeroHess)) {
        // 20 doubles a node, 32-byte aligned: five vector stores
        double4* h = reinterpret_cast<double4*>(s.hess5 + 20 * (long)i);
#pragma unroll
        for (int k = 0; k < 5; k++) h[k] = z;
      }
      if (flags & kBeginResetPhi) {
        double4 o = make_double4(1., 1., 1., 1.);
        double4* p = reinterpret_cast<double4*>(s.phi) + 2 * i;
        p[0] = o;
        p[1] = o;
      }
    }
  }
}

// 16-byte asynchronous global -> shared copies (no register staging, many in
// flight per thread) and their completion.
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(
                   static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
               "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// ---------------------------------------------------------------------------
// Per node: cv_calc_eigenvalue_contribution (cv_calc.C:819-953) and the dt /
// V/dt of build_matrix (init_memory.C:200-290); then the LSQ gradient
// (gradient.C:382-403) or the k=2 derivatives (compute_derivatives.C:
// 1438-1521); then the Venkatakrishnan limiter (limiter.C:594-906).
// Four lanes per node, lane v owning conserved variable v: the gradient,
// the k=2 derivatives and point value, and the limiter value of variable v
// only involve variable v, and each lane accumulates its sums in the
// reference's face / stencil order.  The wave-speed sum (all variables) is
// formed by every lane of the quad from node constants computed once.
// MINB: resident blocks per SM the compiler must allow (0: its own choice);
// the autotuner picks the variant that runs fastest on a given mesh.
// LIM: 0 venkat_fold; 1 venkat_fold_nz (no division of or by zero); 2 the
// same, with the wave-speed face terms formed in the limiter's face loop (one
// walk of the node's faces, more registers).  All give the same bits.
template <int ORDER, int MINB, int LIM = 0>
__global__ void __launch_bounds__(128, MINB) k_node_prepare4(DevMesh m, DevState s, StepArgs a) {
  if (*s.stop) return;  // the run has converged
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = (tid >> 2) + 1, v = tid & 3;
  const int qbase = threadIdx.x & ~3 & 31;
  const unsigned qmask = 0xFu << qbase;
  if (n > m.nn) return;  // whole quads leave together
  const double4 q4 = reinterpret_cast<const double4*>(s.nQ)[n];
  const double q0v = v == 0 ? q4.x : v == 1 ? q4.y : v == 2 ? q4.z : q4.w;

  // ---- wave-speed sum (cv_calc.C:819-953): node constants first ----
  double uu, vv, cs;
  auto node_consts = [&](const double4& q) {
    const double rho = q.x;
    uu = q.y / rho;
    vv = q.z / rho;
    const double P = (a.gamma - 1.0) * (q.w - 0.5 * rho * (uu * uu + vv * vv));
    cs = sqrt((a.gamma * P) / rho);
  };
  double ev = 0.;
  int bad = 0;
  const int s0 = m.nsub_ptr[n], s1 = m.nsub_ptr[n + 1];
  auto wave_term = [&](const double4& g) {
    const double theta = uu * g.x + vv * g.y;
    const double tpc = fabs(theta + cs), tmc = fabs(theta - cs);
    const double w = tpc >= tmc ? tpc : tmc;
    if (!isfinite(w)) bad = 1;
    ev += (w * g.z);
  };
  // the boundary edges' terms after the faces', then dt and V/dt
  auto finish_wave = [&]() {
    const int b0 = m.nbed_ptr[n], b1 = m.nbed_ptr[n + 1];
    for (int k = b0; k < b1; k++) {
      const double* xn = s.xn_bedges + 3 * m.nbed[k];
      const double theta = uu * xn[0] + vv * xn[1];
      const double tpc = fabs(theta + cs), tmc = fabs(theta - cs);
      const double w = tpc >= tmc ? tpc : tmc;
      if (!isfinite(w)) bad = 1;
      ev += (w * xn[2]);
    }
    if (v == 0) {
      const double dt = s.scalars[3] * (m.cv_area[n] / ev);  // cfl of the step (step_args_body)
      s.dt[n] = dt;
      if (bad) atomicOr(s.status, ERR_EIGEN);
      if (dt <= 0. || !isfinite(dt)) atomicOr(s.status, ERR_DT);
    }
  };
  // LIM 2 with the limiter on: the face terms are summed inside the
  // limiter's pass over the same faces (the same order), one walk of the
  // node's incidence list instead of two
  const bool merged = LIM == 2 && a.do_lim;
  if (!merged) {
    node_consts(q4);
    #pragma unroll 4
    for (int k = s0; k < s1; k++) wave_term(m.sub_geo[m.nsub[k] >> 1]);
    finish_wave();
  }
  if (!a.do_grad && !a.do_derivs && !a.do_lim) return;

  // ---- 1-ring min/max and the k=1 LSQ gradient of variable v ----
  double qmin = q0v, qmax = q0v, g0 = 0., g1 = 0.;
  const int e0 = m.nedg_ptr[n], e1 = m.nedg_ptr[n + 1];
  #pragma unroll 4
  for (int k = e0; k < e1; k++) {
    // the neighbour straight from the node's incidence list (nedg_nbr), so
    // its state is one dependent load away, not two
    const double qo = s.nQ[4 * (long)m.nedg_nbr[k] + v];
    qmin = qmin <= qo ? qmin : qo;
    qmax = qmax >= qo ? qmax : qo;
    if (ORDER == 1 && a.do_grad) {
      const int ed = m.nedg[k];
      const int e = ed >> 1, side = ed & 1;
      const double4 w = m.edge_w[e];
      const double dq = side ? (q0v - qo) : (qo - q0v);  // nQ[R] - nQ[L]
      if (side == 0) {
        g0 += w.x * dq;
        g1 += w.y * dq;
      } else {
        g0 -= w.z * dq;
        g1 -= w.w * dq;
      }
    }
  }
  if (ORDER == 1 && a.do_grad)
    reinterpret_cast<double2*>(s.grad + 8 * (long)n)[v] = make_double2(g0, g1);

  // ---- k=2: x = V S^-1 U^T b of variable v ----
  double h[5], pv = 0.;
  if (ORDER == 3 && a.do_derivs) {
    const int t0 = m.st_ptr[n], t1 = m.st_ptr[n + 1];
    const int mrows = t1 - t0;
    const double* U = m.svd_U1 + 5 * (long)t0;  // row k: U[k][0..4], contiguous
    double acc[5] = {0., 0., 0., 0., 0.};
#pragma unroll 4
    for (int k = 0; k < mrows; k++) {
      const int nb = m.st_idx[t0 + k];
      const double bv = m.st_w[t0 + k] * (s.nQ[4 * (long)nb + v] - q0v);
#pragma unroll
      for (int c = 0; c < 5; c++) acc[c] += bv * U[5 * k + c];
    }
      const double* VT = m.svd_VT + 25 * (long)n;
    const double* S = m.svd_S + 5 * (long)n;
    double t1v[5];
#pragma unroll
    for (int c = 0; c < 5; c++) t1v[c] = acc[c] / S[c];
#pragma unroll
    for (int j = 0; j < 5; j++) {
      double sum = 0.;
#pragma unroll
      for (int c = 0; c < 5; c++) sum += VT[j * 5 + c] * t1v[c];
      h[j] = sum;
    }
    const double* mo = m.moments + 9 * (long)n;
    pv = q0v - mo[0] * h[0] - mo[1] * h[1] - mo[2] * h[2] * 0.5 - mo[3] * h[3] * 0.5 -
         mo[4] * h[4];
    double* hd = s.hess5 + 20 * (long)n + 5 * v;
#pragma unroll
    for (int c = 0; c < 5; c++) hd[c] = h[c];
    s.pv[4 * (long)n + v] = pv;
  }

  if (!a.do_lim) return;
  // ---- Venkatakrishnan bound of variable v over every face point ----
  double ph = 1.0;
  const double xn0 = m.x[2 * n], xn1 = m.x[2 * n + 1];
  // the node constants formed again here rather than held through the
  // gradient and stencil loops (the same expressions: the same bits)
  if (merged) node_consts(reinterpret_cast<const double4*>(s.nQ)[n]);
  #pragma unroll 4
  for (int k = s0; k < s1; k++) {
    const int sd = m.nsub[k];
    const int sub = sd >> 1, side = sd & 1;
    if (merged) wave_term(m.sub_geo[sub]);
    if (ORDER == 1) {
      const double4 d = m.sub_dx[sub];
      const double dx0 = side ? d.z : d.x, dx1 = side ? d.w : d.y;
      const double qr = q0v + (g0 * dx0 + g1 * dx1);
      ph = venkat_fold_lim<LIM>(ph, qr, q0v, qmin, qmax);
    } else {
      const double* xg = m.sub_xg + 6 * (long)sub;
#pragma unroll
      for (int gpt = 0; gpt < 3; gpt++) {
        const double dx0 = xg[2 * gpt] - xn0, dx1 = xg[2 * gpt + 1] - xn1;
        double qr = pv;
        qr += (h[0] * dx0 + h[1] * dx1 + h[2] * dx0 * dx0 * 0.5 + h[3] * dx1 * dx1 * 0.5 +
               h[4] * dx0 * dx1);
        ph = venkat_fold_lim<LIM>(ph, qr, q0v, qmin, qmax);
      }
    }
  }
  if (merged) finish_wave();
  // min over the variables in order 0..3 (limiter.C:895-906)
  const double p1 = __shfl_sync(qmask, ph, qbase + 1);
  const double p2 = __shfl_sync(qmask, ph, qbase + 2);
  const double p3 = __shfl_sync(qmask, ph, qbase + 3);
  double pmin = ph;
  pmin = pmin <= p1 ? pmin : p1;
  pmin = pmin <= p2 ? pmin : p2;
  pmin = pmin <= p3 ? pmin : p3;
  const double out = v == 0 ? pmin : ph;
  reinterpret_cast<double2*>(s.phi + 8 * (long)n)[v] = make_double2(out, out);
  if (out < 0.0 || out > 1.0) atomicOr(s.status, ERR_LIMITER);
}

// ---------------------------------------------------------------------------
// k_node_prepare4 with each node's serial chains split over 16 lanes (a
// half-warp): lane l = 4 g + v owns variable v in group g.  Nothing is summed
// in another order:
// * the wave-speed sum: lane j forms face j's term, every lane adds the terms
//   in face order from shuffles;
// * the k=1 gradient: its x sum in group 0, its y sum in group 1, each over
//   every edge in order;
// * the k=2 derivatives: the five columns of V S^-1 U^T b are independent
//   sums; group g sums column g (group 0 also column 4) over the stencil rows
//   in order, and every lane then forms h and the point value from the five;
// * the 1-ring min/max and the limiter's MIN over face points are folds of
//   MIN/MAX: over values none of which is NaN (and the limiter bound is
//   never -0) they equal the minimum / maximum whatever the order, so the
//   four groups fold a quarter of the faces each and the results are
//   combined.  Where any value of the node is NaN the fold is order-
//   dependent, and every lane then folds all faces in the reference's order.
__device__ __forceinline__ double hshfl(double x, unsigned mask, int lane) {
  return __shfl_sync(mask, x, lane);
}

// LIM: the limiter's fold, as in k_node_prepare4.
template <int ORDER, int LIM = 0>
__global__ void __launch_bounds__(128) k_node_prepare16(DevMesh m, DevState s, StepArgs a) {
  if (*s.stop) return;  // the run has converged
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = (tid >> 4) + 1, l = tid & 15, v = l & 3, g = l >> 2;
  const int hbase = threadIdx.x & 16;
  const unsigned hmask = 0xFFFFu << hbase;
  if (n > m.nn) return;  // whole half-warps leave together
  const double4 q4 = reinterpret_cast<const double4*>(s.nQ)[n];
  const double q0v = v == 0 ? q4.x : v == 1 ? q4.y : v == 2 ? q4.z : q4.w;

  // ---- wave-speed sum (cv_calc.C:819-953), terms formed in parallel ----
  const double rho = q4.x, uu = q4.y / rho, vv = q4.z / rho;
  const double P = (a.gamma - 1.0) * (q4.w - 0.5 * rho * (uu * uu + vv * vv));
  const double cs = sqrt((a.gamma * P) / rho);
  double ev = 0.;
  int bad = 0;
  const int s0 = m.nsub_ptr[n], s1 = m.nsub_ptr[n + 1];
  for (int base = s0; base < s1; base += 16) {
    double term = 0.;
    if (base + l < s1) {
      const double4 gg = m.sub_geo[m.nsub[base + l] >> 1];
      const double theta = uu * gg.x + vv * gg.y;
      const double tpc = fabs(theta + cs), tmc = fabs(theta - cs);
      const double w = tpc >= tmc ? tpc : tmc;
      if (!isfinite(w)) bad = 1;
      term = (w * gg.z);
    }
    const int cnt = min(16, s1 - base);
    for (int j = 0; j < cnt; j++) ev += hshfl(term, hmask, hbase + j);
  }
  const int b0 = m.nbed_ptr[n], b1 = m.nbed_ptr[n + 1];
  for (int k = b0; k < b1; k++) {
    const double* xn = s.xn_bedges + 3 * m.nbed[k];
    const double theta = uu * xn[0] + vv * xn[1];
    const double tpc = fabs(theta + cs), tmc = fabs(theta - cs);
    const double w = tpc >= tmc ? tpc : tmc;
    if (!isfinite(w)) bad = 1;
    ev += (w * xn[2]);
  }
  bad = __any_sync(hmask, bad);
  if (l == 0) {
    const double dt = s.scalars[3] * (m.cv_area[n] / ev);  // cfl of the step (step_args_body)
    s.dt[n] = dt;
    if (bad) atomicOr(s.status, ERR_EIGEN);
    if (dt <= 0. || !isfinite(dt)) atomicOr(s.status, ERR_DT);
  }
  if (!a.do_grad && !a.do_derivs && !a.do_lim) return;

  // ---- the k=1 gradient (x in group 0, y in group 1) and the 1-ring
  //      min/max (a quarter of the edges per group) ----
  const int e0 = m.nedg_ptr[n], e1 = m.nedg_ptr[n + 1];
  double qmin = q0v, qmax = q0v, gsum = 0.;
  int nan = 0;
  for (int k = e0; k < e1; k++) {
    const int ed = m.nedg[k];
    const int side = ed & 1;
    const bool mine = ((k - e0) & 3) == g;
    const bool grad = ORDER == 1 && a.do_grad && g < 2;
    if (!mine && !grad) continue;
    const double qo = s.nQ[4 * (long)m.nedg_nbr[k] + v];
    if (mine) {
      if (qo != qo) nan = 1;
      qmin = qmin <= qo ? qmin : qo;
      qmax = qmax >= qo ? qmax : qo;
    }
    if (grad) {
      const double4 w = m.edge_w[ed >> 1];
      const double dq = side ? (q0v - qo) : (qo - q0v);  // nQ[R] - nQ[L]
      if (side == 0) gsum += (g == 0 ? w.x : w.y) * dq;
      else gsum -= (g == 0 ? w.z : w.w) * dq;
    }
  }
  double g0 = 0., g1 = 0.;
  if (ORDER == 1 && a.do_grad) {
    g0 = hshfl(gsum, hmask, hbase + v);
    g1 = hshfl(gsum, hmask, hbase + 4 + v);
    if (g == 0) reinterpret_cast<double2*>(s.grad + 8 * (long)n)[v] = make_double2(g0, g1);
  }

  // ---- k=2: column g (and 4) of V S^-1 U^T b of variable v ----
  double h[5] = {0., 0., 0., 0., 0.}, pv = 0.;
  if (ORDER == 3 && a.do_derivs) {
    const int t0 = m.st_ptr[n], t1 = m.st_ptr[n + 1];
    const int mrows = t1 - t0;
    const double* U = m.svd_U1 + 5 * (long)t0;
    double accA = 0., accB = 0.;
#pragma unroll 4
    for (int k = 0; k < mrows; k++) {
      const int nb = m.st_idx[t0 + k];
      const double bv = m.st_w[t0 + k] * (s.nQ[4 * (long)nb + v] - q0v);
      accA += bv * U[5 * k + g];
      if (g == 0) accB += bv * U[5 * k + 4];
    }
    const double* S = m.svd_S + 5 * (long)n;
    const double tA = accA / S[g];
    const double tB = g == 0 ? accB / S[4] : 0.;
    double t1v[5];
    t1v[0] = hshfl(tA, hmask, hbase + v);
    t1v[1] = hshfl(tA, hmask, hbase + 4 + v);
    t1v[2] = hshfl(tA, hmask, hbase + 8 + v);
    t1v[3] = hshfl(tA, hmask, hbase + 12 + v);
    t1v[4] = hshfl(tB, hmask, hbase + v);
    const double* VT = m.svd_VT + 25 * (long)n;
#pragma unroll
    for (int j = 0; j < 5; j++) {
      double sum = 0.;
#pragma unroll
      for (int c = 0; c < 5; c++) sum += VT[j * 5 + c] * t1v[c];
      h[j] = sum;
    }
    const double* mo = m.moments + 9 * (long)n;
    pv = q0v - mo[0] * h[0] - mo[1] * h[1] - mo[2] * h[2] * 0.5 - mo[3] * h[3] * 0.5 -
         mo[4] * h[4];
    if (g == 0) {
      double* hd = s.hess5 + 20 * (long)n + 5 * v;
#pragma unroll
      for (int c = 0; c < 5; c++) hd[c] = h[c];
      s.pv[4 * (long)n + v] = pv;
    }
  }

  if (!a.do_lim) return;
  // ---- Venkatakrishnan bound of variable v over every face point ----
  const double xn0 = m.x[2 * n], xn1 = m.x[2 * n + 1];
  auto fold_faces = [&](double mn, double mx, int first, int stride, int& sawnan) {
    double ph = 1.0;
    for (int k = s0 + first; k < s1; k += stride) {
      const int sd = m.nsub[k];
      const int sub = sd >> 1, side = sd & 1;
      if (ORDER == 1) {
        const double4 d = m.sub_dx[sub];
        const double dx0 = side ? d.z : d.x, dx1 = side ? d.w : d.y;
        const double qr = q0v + (g0 * dx0 + g1 * dx1);
        ph = venkat_fold_lim<LIM>(ph, qr, q0v, mn, mx);
        if (ph != ph) sawnan = 1;
      } else {
        const double* xg = m.sub_xg + 6 * (long)sub;
#pragma unroll
        for (int gpt = 0; gpt < 3; gpt++) {
          const double dx0 = xg[2 * gpt] - xn0, dx1 = xg[2 * gpt + 1] - xn1;
          double qr = pv;
          qr += (h[0] * dx0 + h[1] * dx1 + h[2] * dx0 * dx0 * 0.5 + h[3] * dx1 * dx1 * 0.5 +
                 h[4] * dx0 * dx1);
          ph = venkat_fold_lim<LIM>(ph, qr, q0v, mn, mx);
          if (ph != ph) sawnan = 1;
        }
      }
    }
    return ph;
  };
  // this variable's 1-ring min/max from the four groups
  double mn = qmin, mx = qmax;
#pragma unroll
  for (int gg = 1; gg < 4; gg++) {
    const double omn = hshfl(qmin, hmask, hbase + ((g + gg) & 3) * 4 + v);
    const double omx = hshfl(qmax, hmask, hbase + ((g + gg) & 3) * 4 + v);
    mn = mn <= omn ? mn : omn;
    mx = mx >= omx ? mx : omx;
  }
  int sawnan = 0;
  double ph = fold_faces(mn, mx, g, 4, sawnan);
  double pg = ph;
#pragma unroll
  for (int gg = 1; gg < 4; gg++) {
    const double o = hshfl(ph, hmask, hbase + ((g + gg) & 3) * 4 + v);
    pg = pg <= o ? pg : o;
  }
  if (__any_sync(hmask, nan | sawnan)) {
    // a NaN makes the folds order-dependent: the reference's order throughout
    mn = q0v;
    mx = q0v;
    for (int k = e0; k < e1; k++) {
      const double qo = s.nQ[4 * (long)m.nedg_nbr[k] + v];
      mn = mn <= qo ? mn : qo;
      mx = mx >= qo ? mx : qo;
    }
    int unused = 0;
    pg = fold_faces(mn, mx, 0, 1, unused);
  }
  // min over the variables in order 0..3 (limiter.C:895-906)
  const double p1 = hshfl(pg, hmask, hbase + 1);
  const double p2 = hshfl(pg, hmask, hbase + 2);
  const double p3 = hshfl(pg, hmask, hbase + 3);
  double pmin = hshfl(pg, hmask, hbase);
  pmin = pmin <= p1 ? pmin : p1;
  pmin = pmin <= p2 ? pmin : p2;
  pmin = pmin <= p3 ? pmin : p3;
  if (g == 0) {
    const double out = v == 0 ? pmin : pg;
    reinterpret_cast<double2*>(s.phi + 8 * (long)n)[v] = make_double2(out, out);
    if (out < 0.0 || out > 1.0) atomicOr(s.status, ERR_LIMITER);
  }
}

// ---------------------------------------------------------------------------
// k_node_prepare4 with its gathers staged in shared memory: the same per-lane
// arithmetic in the same order (so the same bits), but a CTA of kStageNodes
// consecutive nodes first copies its slices of the incidence lists and the
// stencil (contiguous, coalesced), then issues every face-record and
// neighbour-state gather at once as 16-byte cp.async copies, so the chains
// incidence -> face record -> neighbour state cost one round trip each for
// the whole tile instead of one per loop iteration.  StageCaps holds the
// largest slice any tile has (host-computed), which sizes the shared memory.
constexpr int kStageNodes = 32;

struct StageCaps {
  int sub;   // subedge incidences of a tile
  int edg;   // edge incidences of a tile
  int sten;  // k=2 stencil rows of a tile
};

__host__ __device__ inline size_t stage_smem_bytes(int order, StageCaps c) {
  const size_t face = order == 3 ? 32 + 48 : 32 + 32;  // geometry + Gauss points or offsets
  const size_t edge = order == 1 ? 64 : 32;            // neighbour state (+ LSQ weights)
  return face * c.sub + edge * c.edg + 32 * (size_t)c.sten +
         4 * ((size_t)c.sub + 2 * (size_t)c.edg + (size_t)c.sten);
}

template <int ORDER>
__global__ void __launch_bounds__(128) k_node_stage(DevMesh m, DevState s, StepArgs a,
                                                    StageCaps cap) {
  if (*s.stop) return;  // the run has converged
  extern __shared__ __align__(16) unsigned char sm[];
  double4* s_geo = reinterpret_cast<double4*>(sm);
  char* p = reinterpret_cast<char*>(s_geo + cap.sub);
  double2* s_xg = reinterpret_cast<double2*>(p);  // k=2: 3 Gauss points per incidence
  double4* s_dx = reinterpret_cast<double4*>(p);  // k=1: face-point offsets
  p += (size_t)cap.sub * (ORDER == 3 ? 48 : 32);
  double4* s_nqe = reinterpret_cast<double4*>(p);  // edge neighbours' states
  double4* s_ew = s_nqe + cap.edg;                 // k=1: LSQ weights
  p += (size_t)cap.edg * (ORDER == 1 ? 64 : 32);
  double4* s_nqs = reinterpret_cast<double4*>(p);  // k=2: stencil neighbours' states
  int* s_sub = reinterpret_cast<int*>(s_nqs + cap.sten);
  int* s_edg = s_sub + cap.sub;
  int* s_nbr = s_edg + cap.edg;
  int* s_st = s_nbr + cap.edg;

  const int n0 = blockIdx.x * kStageNodes + 1;
  const int nlast = min(n0 + kStageNodes - 1, m.nn);
  const int K0 = m.nsub_ptr[n0], K1 = m.nsub_ptr[nlast + 1];
  const bool rest = a.do_grad || a.do_derivs || a.do_lim;
  const int E0 = m.nedg_ptr[n0], E1 = rest ? m.nedg_ptr[nlast + 1] : E0;
  const bool derivs = ORDER == 3 && a.do_derivs;
  const int R0 = derivs ? m.st_ptr[n0] : 0, R1 = derivs ? m.st_ptr[nlast + 1] : 0;
  const int tid = threadIdx.x, nt = blockDim.x;
  // the tile's slices of the lists (contiguous)
  for (int k = tid; k < K1 - K0; k += nt) s_sub[k] = m.nsub[K0 + k];
  for (int k = tid; k < E1 - E0; k += nt) {
    s_edg[k] = m.nedg[E0 + k];
    s_nbr[k] = m.nedg_nbr[E0 + k];
  }
  for (int k = tid; k < R1 - R0; k += nt) s_st[k] = m.st_idx[R0 + k];
  __syncthreads();
  // every gather of the tile in flight at once
  const double4* nq4 = reinterpret_cast<const double4*>(s.nQ);
  for (int k = tid; k < K1 - K0; k += nt) {
    const int sub = s_sub[k] >> 1;
    const char* g = reinterpret_cast<const char*>(m.sub_geo + sub);
    cp_async16(&s_geo[k], g);
    cp_async16(reinterpret_cast<char*>(&s_geo[k]) + 16, g + 16);
    if (a.do_lim) {
      if (ORDER == 1) {
        const char* d = reinterpret_cast<const char*>(m.sub_dx + sub);
        cp_async16(&s_dx[k], d);
        cp_async16(reinterpret_cast<char*>(&s_dx[k]) + 16, d + 16);
      } else {
        const double2* x = reinterpret_cast<const double2*>(m.sub_xg + 6 * (long)sub);
        cp_async16(&s_xg[3 * k], x);
        cp_async16(&s_xg[3 * k + 1], x + 1);
        cp_async16(&s_xg[3 * k + 2], x + 2);
      }
    }
  }
  for (int k = tid; k < E1 - E0; k += nt) {
    const char* q = reinterpret_cast<const char*>(nq4 + s_nbr[k]);
    cp_async16(&s_nqe[k], q);
    cp_async16(reinterpret_cast<char*>(&s_nqe[k]) + 16, q + 16);
    if (ORDER == 1 && a.do_grad) {
      const char* w = reinterpret_cast<const char*>(m.edge_w + (s_edg[k] >> 1));
      cp_async16(&s_ew[k], w);
      cp_async16(reinterpret_cast<char*>(&s_ew[k]) + 16, w + 16);
    }
  }
  for (int k = tid; k < R1 - R0; k += nt) {
    const char* q = reinterpret_cast<const char*>(nq4 + s_st[k]);
    cp_async16(&s_nqs[k], q);
    cp_async16(reinterpret_cast<char*>(&s_nqs[k]) + 16, q + 16);
  }
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();

  // ---- per node and variable, as k_node_prepare4 ----
  const int n = n0 + (tid >> 2), v = tid & 3;
  const int qbase = tid & ~3 & 31;
  const unsigned qmask = 0xFu << qbase;
  if (n > nlast) return;  // whole quads leave together; no barrier follows
  const double4 q4 = nq4[n];
  const double q0v = v == 0 ? q4.x : v == 1 ? q4.y : v == 2 ? q4.z : q4.w;
  const double rho = q4.x, uu = q4.y / rho, vv = q4.z / rho;
  const double P = (a.gamma - 1.0) * (q4.w - 0.5 * rho * (uu * uu + vv * vv));
  const double cs = sqrt((a.gamma * P) / rho);
  double ev = 0.;
  int bad = 0;
  const int s0 = m.nsub_ptr[n], s1 = m.nsub_ptr[n + 1];
  #pragma unroll 4
  for (int k = s0; k < s1; k++) {
    const double4 g = s_geo[k - K0];
    const double theta = uu * g.x + vv * g.y;
    const double tpc = fabs(theta + cs), tmc = fabs(theta - cs);
    const double w = tpc >= tmc ? tpc : tmc;
    if (!isfinite(w)) bad = 1;
    ev += (w * g.z);
  }
  const int b0 = m.nbed_ptr[n], b1 = m.nbed_ptr[n + 1];
  for (int k = b0; k < b1; k++) {
    const double* xn = s.xn_bedges + 3 * m.nbed[k];
    const double theta = uu * xn[0] + vv * xn[1];
    const double tpc = fabs(theta + cs), tmc = fabs(theta - cs);
    const double w = tpc >= tmc ? tpc : tmc;
    if (!isfinite(w)) bad = 1;
    ev += (w * xn[2]);
  }
  if (v == 0) {
    const double dt = s.scalars[3] * (m.cv_area[n] / ev);
    s.dt[n] = dt;
    if (bad) atomicOr(s.status, ERR_EIGEN);
    if (dt <= 0. || !isfinite(dt)) atomicOr(s.status, ERR_DT);
  }
  if (!rest) return;

  double qmin = q0v, qmax = q0v, g0 = 0., g1 = 0.;
  const int e0 = m.nedg_ptr[n], e1 = m.nedg_ptr[n + 1];
  #pragma unroll 4
  for (int k = e0; k < e1; k++) {
    const int side = s_edg[k - E0] & 1;
    const double qo = reinterpret_cast<const double*>(&s_nqe[k - E0])[v];
    qmin = qmin <= qo ? qmin : qo;
    qmax = qmax >= qo ? qmax : qo;
    if (ORDER == 1 && a.do_grad) {
      const double4 w = s_ew[k - E0];
      const double dq = side ? (q0v - qo) : (qo - q0v);
      if (side == 0) {
        g0 += w.x * dq;
        g1 += w.y * dq;
      } else {
        g0 -= w.z * dq;
        g1 -= w.w * dq;
      }
    }
  }
  if (ORDER == 1 && a.do_grad)
    reinterpret_cast<double2*>(s.grad + 8 * (long)n)[v] = make_double2(g0, g1);

  double h[5], pv = 0.;
  if (derivs) {
    const int t0 = m.st_ptr[n], t1 = m.st_ptr[n + 1];
    const int mrows = t1 - t0;
    const double* U = m.svd_U1 + 5 * (long)t0;
    double acc[5] = {0., 0., 0., 0., 0.};
#pragma unroll 4
    for (int k = 0; k < mrows; k++) {
      const double qn = reinterpret_cast<const double*>(&s_nqs[t0 - R0 + k])[v];
      const double bv = m.st_w[t0 + k] * (qn - q0v);
#pragma unroll
      for (int c = 0; c < 5; c++) acc[c] += bv * U[5 * k + c];
    }
    const double* VT = m.svd_VT + 25 * (long)n;
    const double* S = m.svd_S + 5 * (long)n;
    double t1v[5];
#pragma unroll
    for (int c = 0; c < 5; c++) t1v[c] = acc[c] / S[c];
#pragma unroll
    for (int j = 0; j < 5; j++) {
      double sum = 0.;
#pragma unroll
      for (int c = 0; c < 5; c++) sum += VT[j * 5 + c] * t1v[c];
      h[j] = sum;
    }
    const double* mo = m.moments + 9 * (long)n;
    pv = q0v - mo[0] * h[0] - mo[1] * h[1] - mo[2] * h[2] * 0.5 - mo[3] * h[3] * 0.5 -
         mo[4] * h[4];
    double* hd = s.hess5 + 20 * (long)n + 5 * v;
#pragma unroll
    for (int c = 0; c < 5; c++) hd[c] = h[c];
    s.pv[4 * (long)n + v] = pv;
  }

  if (!a.do_lim) return;
  double ph = 1.0;
  const double xn0 = m.x[2 * n], xn1 = m.x[2 * n + 1];
  #pragma unroll 4
  for (int k = s0; k < s1; k++) {
    const int side = s_sub[k - K0] & 1;
    if (ORDER == 1) {
      const double4 d = s_dx[k - K0];
      const double dx0 = side ? d.z : d.x, dx1 = side ? d.w : d.y;
      const double qr = q0v + (g0 * dx0 + g1 * dx1);
      ph = venkat_fold(ph, qr, q0v, qmin, qmax);
    } else {
#pragma unroll
      for (int gpt = 0; gpt < 3; gpt++) {
        const double2 xg = s_xg[3 * (k - K0) + gpt];
        const double dx0 = xg.x - xn0, dx1 = xg.y - xn1;
        double qr = pv;
        qr += (h[0] * dx0 + h[1] * dx1 + h[2] * dx0 * dx0 * 0.5 + h[3] * dx1 * dx1 * 0.5 +
               h[4] * dx0 * dx1);
        ph = venkat_fold(ph, qr, q0v, qmin, qmax);
      }
    }
  }
  const double p1 = __shfl_sync(qmask, ph, qbase + 1);
  const double p2 = __shfl_sync(qmask, ph, qbase + 2);
  const double p3 = __shfl_sync(qmask, ph, qbase + 3);
  double pmin = ph;
  pmin = pmin <= p1 ? pmin : p1;
  pmin = pmin <= p2 ? pmin : p2;
  pmin = pmin <= p3 ? pmin : p3;
  const double out = v == 0 ? pmin : ph;
  reinterpret_cast<double2*>(s.phi + 8 * (long)n)[v] = make_double2(out, out);
  if (out < 0.0 || out > 1.0) atomicOr(s.status, ERR_LIMITER);
}

// ---------------------------------------------------------------------------
// The two face states of subedge sub: the node states, reconstructed to the
// face point (reconstruct.C:181-203) when RECON is 1.
template <int RECON>
__device__ __forceinline__ void face_states(const DevMesh& m, const DevState& s, int sub,
                                            int2 lr, double* qL, double* qR) {
  const double4 qa = reinterpret_cast<const double4*>(s.nQ)[lr.x];
  const double4 qb = reinterpret_cast<const double4*>(s.nQ)[lr.y];
  qL[0] = qa.x; qL[1] = qa.y; qL[2] = qa.z; qL[3] = qa.w;
  qR[0] = qb.x; qR[1] = qb.y; qR[2] = qb.z; qR[3] = qb.w;
  if (RECON == 1) {
    const double4 d = m.sub_dx[sub];
    const double* gL = s.grad + 8 * (long)lr.x;
    const double* gR = s.grad + 8 * (long)lr.y;
    const double phL = s.phi[8 * (long)lr.x], phR = s.phi[8 * (long)lr.y];
#pragma unroll
    for (int j = 0; j < 4; j++) {
      qL[j] += (phL * gL[2 * j] * d.x + phL * gL[2 * j + 1] * d.y);
      qR[j] += (phR * gR[2 * j] * d.z + phR * gR[2 * j + 1] * d.w);
    }
  }
}

// The Roe flux of a face and its approximate Jacobians (JL, JR row-major):
// dF/dqL = (A(qL) + |A~|) len / 2, dF/dqR = (A(qR) - |A~|) len / 2.
__device__ __forceinline__ void face_flux_approx(double4 g, double gamma, const double* qL,
                                                 const double* qR, double* flux, double* JL,
                                                 double* JR) {
  const double ogm1 = 1.0 / (gamma - 1.0);
  RoeSide SL, SR;
  roe_side(qL, g.x, g.y, g.z, gamma, SL);
  roe_side(qR, g.x, g.y, g.z, gamma, SR);
  const double bg = roe_weight(SL.rho, SR.rho);
  double Rm[16], dL[16], dR[16];
  roe_core(g.x, g.y, g.z, gamma, ogm1, qL, qR, SL, SR, bg, flux, Rm);
  euler_jacobian(qL, g.x, g.y, gamma, dL);
  euler_jacobian(qR, g.x, g.y, gamma, dR);
  // each entry rounded to FP32: the blocks these feed are FP32, and the
  // face-to-assembly round trip carries half the bytes
#pragma unroll
  for (int k = 0; k < 16; k++) {
    JL[k] = (double)__double2float_rn(0.5 * (dL[k] + Rm[k]) * g.z);
    JR[k] = (double)__double2float_rn(0.5 * (dR[k] - Rm[k]) * g.z);
  }
}

// ---------------------------------------------------------------------------
// Per node: R and RHS = -R, the diagonal block (V/dt plus the face Jacobians
// in face order), the off-diagonal blocks of the node's LHS row, and the LU
// factors of the diagonal block for the sweeps (linear_algebra.C:226-246).
// Four lanes per node, lane q owning row q of every 4x4 block and component
// q of R; each lane sums its row in the reference's face order.  MIXED (the
// precision form) writes FP32 off-diagonal blocks and FP32 LU factors with
// reciprocal pivots instead of the FP64 row: into the mode 1/2 tables
// (MIXED 1) or into the row's forward and backward sweep records (MIXED 2).

// Row q of face `sub`'s Jacobian block J (JL or JR): FP64, or FP32 entries
// (JF) widened exactly.
template <bool JF>
__device__ __forceinline__ double4 face_jac_row(const double* J, int sub, int q) {
  if (JF) {
    const float4 f = reinterpret_cast<const float4*>(J)[4 * (long)sub + q];
    return make_double4(f.x, f.y, f.z, f.w);
  }
  return reinterpret_cast<const double4*>(J + 16 * (long)sub)[q];
}

// The V/dt diagonal row q of node n's block (build_matrix).
__device__ __forceinline__ void diag_row(const DevMesh& m, const DevState& s, const StepArgs& a,
                                         int n, int q, double& D0, double& D1, double& D2,
                                         double& D3) {
  D0 = D1 = D2 = D3 = 0.;
  const double diag = m.cv_area[n] / (s.dt[n]);
  if (a.steady_diag) {
    if (q == 0) D0 = diag;
    if (q == 1) D1 = diag;
    if (q == 2) D2 = diag;
    if (q == 3) D3 = diag;
  }
}

// Row q of node n after the interior faces were summed into r and D: the
// boundary edges' terms, R and RHS, the row's blocks (offb(k, B) gives
// off-diagonal block k's row q) and the LU factors of the diagonal block.
template <int MIXED, class OffBlock>
__device__ __forceinline__ void assemble_row(const DevMesh& m, const DevState& s,
                                             const StepArgs& a, const MixedTables& mt,
                                             const ChunkTables& ct, int n, int q, int qbase,
                                             unsigned qmask, bool jac, double r, double D0,
                                             double D1, double D2, double D3, OffBlock&& offb) {
  const int b0 = a.skip_bnd ? 0 : m.nbed_ptr[n], b1 = a.skip_bnd ? 0 : m.nbed_ptr[n + 1];
  for (int k = b0; k < b1; k++) {
    const int b = m.nbed[k];
    r += s.Fb[4 * (long)b + q];
    if (jac) {
      const double4 J = reinterpret_cast<const double4*>(s.Jb + 16 * (long)b)[q];
      D0 += J.x; D1 += J.y; D2 += J.z; D3 += J.w;
    }
  }
  s.R[4 * (long)n + q] = r;
  s.RHS[4 * (long)n + q] = -(r);
  const int k0 = m.ia[n], k1 = m.ia[n + 1];
  // precision form: this row's off-diagonal blocks in colour order (the
  // diagonal block is the row's last, so block k is off-diagonal k - k0)
  const int mpos = MIXED == 1 ? mt.pos[n] : 0;
  const int moff = MIXED == 1 ? mt.offd_ptr[mpos] : 0;
  SweepRec* rf = MIXED == 2 ? ct.rec[0] + ct.pos[0][n] : nullptr;
  SweepRec* rb = MIXED == 2 ? ct.rec[1] + ct.pos[1][n] : nullptr;
  if (MIXED == 2) {
    const float rh = __double2float_rn(-(r));
    reinterpret_cast<float*>(&rf->rhs)[q] = rh;
    reinterpret_cast<float*>(&rb->rhs)[q] = rh;
  }
  for (int k = k0; k < k1; k++) {
    double4* out = reinterpret_cast<double4*>(s.LHS + 16 * (long)k) + q;
    if (m.ja[k] == n) {
      if (!MIXED) *out = make_double4(D0, D1, D2, D3);
      continue;
    }
    double B0 = 0., B1 = 0., B2 = 0., B3 = 0.;
    offb(k, B0, B1, B2, B3);
    const float4 b32 = make_float4(__double2float_rn(B0), __double2float_rn(B1),
                                   __double2float_rn(B2), __double2float_rn(B3));
    if (MIXED == 1) {
      reinterpret_cast<float4*>(mt.lhs32 + 16 * (long)(moff + (k - k0)))[q] = b32;
    } else if (MIXED == 2) {
      rf->a[4 * (k - k0) + q] = b32;
      rb->a[4 * (k - k0) + q] = b32;
    } else {
      *out = make_double4(B0, B1, B2, B3);
    }
  }
  // LU of the diagonal block: every lane factors the whole block
  double M[16];
#pragma unroll
  for (int row = 0; row < 4; row++) {
    M[4 * row + 0] = __shfl_sync(qmask, D0, qbase + row);
    M[4 * row + 1] = __shfl_sync(qmask, D1, qbase + row);
    M[4 * row + 2] = __shfl_sync(qmask, D2, qbase + row);
    M[4 * row + 3] = __shfl_sync(qmask, D3, qbase + row);
  }
  lu4(M);
  double o0 = M[0], o1 = M[1], o2 = M[2], o3 = M[3];
#pragma unroll
  for (int row = 1; row < 4; row++)
    if (q == row) {
      o0 = M[4 * row]; o1 = M[4 * row + 1]; o2 = M[4 * row + 2]; o3 = M[4 * row + 3];
    }
  if (MIXED) {
    // FP32 factors with reciprocal pivots (1/u_qq in FP64, then rounded)
    float f[4] = {__double2float_rn(o0), __double2float_rn(o1), __double2float_rn(o2),
                  __double2float_rn(o3)};
    const double piv = q == 0 ? o0 : q == 1 ? o1 : q == 2 ? o2 : o3;
    const float rp = __double2float_rn(1.0 / piv);
    if (q == 0) f[0] = rp;
    if (q == 1) f[1] = rp;
    if (q == 2) f[2] = rp;
    if (q == 3) f[3] = rp;
    const float4 lu = make_float4(f[0], f[1], f[2], f[3]);
    if (MIXED == 1) {
      reinterpret_cast<float4*>(mt.lu32 + 16 * (long)mpos)[q] = lu;
    } else {
      rf->lu[q] = lu;
      rb->lu[q] = lu;
    }
  } else {
    reinterpret_cast<double4*>(s.LUd + 16 * (long)n)[q] = make_double4(o0, o1, o2, o3);
  }
}

// JF: the face Jacobians are the approximate ones, stored as FP32
// (k_subedge_flux<., true, ., 1>).
template <bool JAC, int MIXED, bool JF = false>
__global__ void __launch_bounds__(128) k_assemble4(DevMesh m, DevState s, StepArgs a,
                                                   MixedTables mt, ChunkTables ct) {
  if (*s.stop) return;  // the run has converged
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = (tid >> 2) + 1, q = tid & 3;
  const int qbase = threadIdx.x & ~3 & 31;
  const unsigned qmask = 0xFu << qbase;
  if (n > m.nn) return;
  double r = 0.;
  double D0, D1, D2, D3;
  diag_row(m, s, a, n, q, D0, D1, D2, D3);
  const int s0 = m.nsub_ptr[n], s1 = m.nsub_ptr[n + 1];
  for (int k = s0; k < s1; k++) {
    const int sd = m.nsub[k];
    const int sub = sd >> 1, side = sd & 1;
    const double f = s.F[4 * (long)sub + q];
    if (side == 0) r += f;
    else r -= f;
    if (JAC) {
      const double4 J = face_jac_row<JF>(side ? s.JR : s.JL, sub, q);
      if (side == 0) {
        D0 += J.x; D1 += J.y; D2 += J.z; D3 += J.w;
      } else {
        D0 -= J.x; D1 -= J.y; D2 -= J.z; D3 -= J.w;
      }
    }
  }
  assemble_row<MIXED>(m, s, a, mt, ct, n, q, qbase, qmask, JAC, r, D0, D1, D2, D3,
                      [&](int k, double& B0, double& B1, double& B2, double& B3) {
    if (!JAC) return;
    const int4 cs = m.csr_sub[k];
    const double* src = cs.z == 0 ? s.JR : s.JL;
    for (int t = 0; t < 2; t++) {
      const int sub = t == 0 ? cs.x : cs.y;
      if (sub < 0) break;
      const double4 J = face_jac_row<JF>(src, sub, q);
      if (cs.z == 0) {
        B0 += J.x; B1 += J.y; B2 += J.z; B3 += J.w;
      } else {
        B0 -= J.x; B1 -= J.y; B2 -= J.z; B3 -= J.w;
      }
    }
  });
}

// ---------------------------------------------------------------------------
// Precision form with the approximate Jacobian (flow_set_jacobian 1): the
// interior faces' fluxes and Jacobians formed by the nodes that gather them,
// instead of written per face and read back (k_subedge_flux + k_assemble4:
// 288 bytes a face through HBM).  The four lanes of a node take its faces
// four at a time (face_states / face_flux_approx, the arithmetic of
// k_subedge_flux<., true, ., 1>), leave F, JL, JR in shared memory, and then
// each lane sums its row in face order as k_assemble4 does; an off-diagonal
// block gathers the faces of its edge in a shared-memory accumulator, in the
// same order (its first subedge, then its second).  So R, every block and the
// factors are the bits of the two-kernel path; each face is formed twice (once
// per end), which costs less than the round trip.  k_boundary runs first.
// Rows with more than kRecBlocks off-diagonal blocks take the two-kernel path
// (host-checked).
constexpr int kFusedNodes = 32;
// per node 4 face buffers of 36 doubles (+1: consecutive nodes start on
// different banks); per lane kRecBlocks block rows of 4 doubles (+1, same)
constexpr int kFusedFace = 4 * 36 + 1, kFusedOff = kRecBlocks * 4 + 1;
constexpr size_t kFusedSmem = (size_t)kFusedNodes * kFusedFace * 8 +
                              (size_t)kFusedNodes * 4 * kFusedOff * 8;

template <int RECON, int MIXED>
__global__ void __launch_bounds__(128) k_faces_assemble(DevMesh m, DevState s, StepArgs a,
                                                        MixedTables mt, ChunkTables ct) {
  if (*s.stop) return;  // the run has converged
  extern __shared__ __align__(16) double fsm[];
  const int tid = threadIdx.x, nl = tid >> 2, q = tid & 3;
  const int n = blockIdx.x * kFusedNodes + nl + 1;
  const int qbase = tid & ~3 & 31;
  const unsigned qmask = 0xFu << qbase;
  if (n > m.nn) return;  // whole quads leave together; only quad-wide syncs follow
  double* face = fsm + (size_t)nl * kFusedFace;  // F (4), JL (16), JR (16) of 4 faces
  double* off = fsm + (size_t)kFusedNodes * kFusedFace + ((size_t)nl * 4 + q) * kFusedOff;
#pragma unroll
  for (int t = 0; t < kRecBlocks * 4; t++) off[t] = 0.;
  double r = 0.;
  double D0, D1, D2, D3;
  diag_row(m, s, a, n, q, D0, D1, D2, D3);
  const int s0 = m.nsub_ptr[n], s1 = m.nsub_ptr[n + 1];
  for (int base = s0; base < s1; base += 4) {
    if (base + q < s1) {
      const int sub = m.nsub[base + q] >> 1;
      double qL[4], qR[4];
      face_states<RECON>(m, s, sub, m.sub_lr[sub], qL, qR);
      double* fb = face + q * 36;
      face_flux_approx(m.sub_geo[sub], a.gamma, qL, qR, fb, fb + 4, fb + 20);
    }
    __syncwarp(qmask);
    const int cnt = min(4, s1 - base);
    for (int f = 0; f < cnt; f++) {
      const int side = m.nsub[base + f] & 1;
      const double* fb = face + f * 36;
      const double fl = fb[q];
      if (side == 0) r += fl;
      else r -= fl;
      const double* JL = fb + 4 + 4 * q;
      const double* JR = fb + 20 + 4 * q;
      double* o = off + 4 * m.nsub_slot[base + f];
      if (side == 0) {
        D0 += JL[0]; D1 += JL[1]; D2 += JL[2]; D3 += JL[3];
        o[0] += JR[0]; o[1] += JR[1]; o[2] += JR[2]; o[3] += JR[3];
      } else {
        D0 -= JR[0]; D1 -= JR[1]; D2 -= JR[2]; D3 -= JR[3];
        o[0] -= JL[0]; o[1] -= JL[1]; o[2] -= JL[2]; o[3] -= JL[3];
      }
    }
    __syncwarp(qmask);
  }
  const int k0 = m.ia[n];
  assemble_row<MIXED>(m, s, a, mt, ct, n, q, qbase, qmask, true, r, D0, D1, D2, D3,
                      [&](int k, double& B0, double& B1, double& B2, double& B3) {
    const double* o = off + 4 * (k - k0);
    B0 = o[0]; B1 = o[1]; B2 = o[2]; B3 = o[3];
  });
}

// ---------------------------------------------------------------------------
// build_boundary_residuals after an interior-only assembly (a.skip_bnd): the
// boundary fluxes and approximate Jacobians of each node's boundary edges,
// in ascending order, added to the node's R and diagonal block as the full
// assembly adds them after the interior faces (residual.C:1147-1167), so
// interior + boundary gives the bits of the one-pass assembly.  The LU
// factors of the changed diagonal blocks are formed again.  FP64 only.
template <bool JAC>
__global__ void __launch_bounds__(128) k_boundary_add4(DevMesh m, DevState s) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = (tid >> 2) + 1, q = tid & 3;
  const int qbase = threadIdx.x & ~3 & 31;
  const unsigned qmask = 0xFu << qbase;
  if (n > m.nn) return;
  const int b0 = m.nbed_ptr[n], b1 = m.nbed_ptr[n + 1];
  if (b0 == b1) return;  // whole quads leave together
  double r = s.R[4 * (long)n + q];
  double4* drow = reinterpret_cast<double4*>(s.LHS + 16 * (long)m.iau[n]) + q;
  double4 d = *drow;
  for (int k = b0; k < b1; k++) {
    const int b = m.nbed[k];
    r += s.Fb[4 * (long)b + q];
    if (JAC) {
      const double4 J = reinterpret_cast<const double4*>(s.Jb + 16 * (long)b)[q];
      d.x += J.x; d.y += J.y; d.z += J.z; d.w += J.w;
    }
  }
  s.R[4 * (long)n + q] = r;
  s.RHS[4 * (long)n + q] = -(r);
  *drow = d;
  double M[16];
#pragma unroll
  for (int row = 0; row < 4; row++) {
    M[4 * row + 0] = __shfl_sync(qmask, d.x, qbase + row);
    M[4 * row + 1] = __shfl_sync(qmask, d.y, qbase + row);
    M[4 * row + 2] = __shfl_sync(qmask, d.z, qbase + row);
    M[4 * row + 3] = __shfl_sync(qmask, d.w, qbase + row);
  }
  lu4(M);
  reinterpret_cast<double4*>(s.LUd + 16 * (long)n)[q] =
      make_double4(M[4 * q], M[4 * q + 1], M[4 * q + 2], M[4 * q + 3]);
}

// LU factors of every diagonal block (linear_algebra.C:226-246), from an LHS
// the caller supplied (flow_set "LHS"): what the assembly would have formed.
__global__ void __launch_bounds__(128) k_diag_lu(DevMesh m, DevState s) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (n > m.nn) return;
  const double4* src = reinterpret_cast<const double4*>(s.LHS + 16 * (long)m.iau[n]);
  double M[16];
#pragma unroll
  for (int row = 0; row < 4; row++) {
    const double4 v = src[row];
    M[4 * row] = v.x; M[4 * row + 1] = v.y; M[4 * row + 2] = v.z; M[4 * row + 3] = v.w;
  }
  lu4(M);
  double4* dst = reinterpret_cast<double4*>(s.LUd + 16 * (long)n);
#pragma unroll
  for (int row = 0; row < 4; row++)
    dst[row] = make_double4(M[4 * row], M[4 * row + 1], M[4 * row + 2], M[4 * row + 3]);
}

// ---------------------------------------------------------------------------
// Per subedge: face states, Roe flux, forward-difference Jacobian
// (residual.C:112-333, reconstruct.C:181-203, jacobian.C:45-110).
// JMODE 0: the reference's forward differences.  JMODE 1 (precision form
// only): the approximate Roe Jacobian dF/dqL = (A(qL) + |A~|) len / 2,
// dF/dqR = (A(qR) - |A~|) len / 2 (|A~| frozen: the form jacobian.C:681-962
// gives the boundary faces), from the |A~| the flux formed anyway.
template <int RECON, bool JAC, int MINB, int JMODE = 0>
__global__ void __launch_bounds__(128, MINB) k_subedge_flux(DevMesh m, DevState s, StepArgs a) {
  if (*s.stop) return;  // the run has converged
  int sub = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (sub > m.ns) return;
  const int2 lr = m.sub_lr[sub];
  const double4 g = m.sub_geo[sub];
  double qL[4], qR[4];
  face_states<RECON>(m, s, sub, lr, qL, qR);
  double flux[4];
  if (JAC && JMODE == 1) {
    // face_flux_approx's arithmetic with the physical Jacobians formed and
    // stored a row at a time (fewer values live at once; the same bits)
    const double ogm1 = 1.0 / (a.gamma - 1.0);
    RoeSide SL, SR;
    roe_side(qL, g.x, g.y, g.z, a.gamma, SL);
    roe_side(qR, g.x, g.y, g.z, a.gamma, SR);
    const double bg = roe_weight(SL.rho, SR.rho);
    double Rm[16];
    roe_core(g.x, g.y, g.z, a.gamma, ogm1, qL, qR, SL, SR, bg, flux, Rm);
    reinterpret_cast<double4*>(s.F)[sub] = make_double4(flux[0], flux[1], flux[2], flux[3]);
    const EulerJacSide EL = euler_jacobian_side(qL, g.x, g.y, a.gamma);
    const EulerJacSide ER = euler_jacobian_side(qR, g.x, g.y, a.gamma);
    // FP32-valued entries stored as FP32 (16 floats a face and side)
    float4* JLo = reinterpret_cast<float4*>(s.JL) + 4 * (long)sub;
    float4* JRo = reinterpret_cast<float4*>(s.JR) + 4 * (long)sub;
#pragma unroll
    for (int r = 0; r < 4; r++) {
      double dl[4], dr[4];
      euler_jacobian_row(EL, g.x, g.y, a.gamma, r, dl);
      euler_jacobian_row(ER, g.x, g.y, a.gamma, r, dr);
      float jl[4], jr[4];
#pragma unroll
      for (int k = 0; k < 4; k++) {
        jl[k] = __double2float_rn(0.5 * (dl[k] + Rm[4 * r + k]) * g.z);
        jr[k] = __double2float_rn(0.5 * (dr[k] - Rm[4 * r + k]) * g.z);
      }
      JLo[r] = make_float4(jl[0], jl[1], jl[2], jl[3]);
      JRo[r] = make_float4(jr[0], jr[1], jr[2], jr[3]);
    }
    return;
  }
  // Roe_flux_centered and its 8 forward differences (jacobian.C:45-185): the
  // unperturbed side's quantities and, unless the density is perturbed, the
  // Roe density weight are reused from the base evaluation
  const double ogm1 = 1.0 / (a.gamma - 1.0);
  RoeSide SL, SR;
  roe_side(qL, g.x, g.y, g.z, a.gamma, SL);
  roe_side(qR, g.x, g.y, g.z, a.gamma, SR);
  const double bg = roe_weight(SL.rho, SR.rho);
  roe_core(g.x, g.y, g.z, a.gamma, ogm1, qL, qR, SL, SR, bg, flux);
  reinterpret_cast<double4*>(s.F)[sub] = make_double4(flux[0], flux[1], flux[2], flux[3]);
  if (!JAC) return;
  const double eps = 1.0e-08;
  double* JLo = s.JL + 16 * (long)sub;
  double* JRo = s.JR + 16 * (long)sub;
#pragma unroll 1
  for (int side = 0; side < 2; side++) {
    double* Jo = side ? JRo : JLo;
#pragma unroll 1
    for (int i = 0; i < 4; i++) {
      double qp[4], fp[4];
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const double bj = side ? qR[j] : qL[j];
        qp[j] = j == i ? bj + eps : bj;
      }
      RoeSide SP;
      roe_side(qp, g.x, g.y, g.z, a.gamma, SP);
      double bgp = bg;
      if (i == 0) bgp = side ? roe_weight(SL.rho, SP.rho) : roe_weight(SP.rho, SR.rho);
      if (side == 0)
        roe_core(g.x, g.y, g.z, a.gamma, ogm1, qp, qR, SP, SR, bgp, fp);
      else
        roe_core(g.x, g.y, g.z, a.gamma, ogm1, qL, qp, SL, SP, bgp, fp);
#pragma unroll
      for (int j = 0; j < 4; j++) Jo[j * 4 + i] = (fp[j] - flux[j]) / eps;
    }
  }
}

// ---------------------------------------------------------------------------
// Per boundary edge: Set_Boundary_Values (cvbc.C:78-471) for its ghost, the
// low-order boundary flux (residual.C:1147-1167) and the approximate
// Jacobian (jacobian.C:681-962).  On the k=2 Gauss pass a curved bedge uses
// the node normal and the arc length and writes the normal back into
// xn_bedges (residual.C:1103-1143), as the reference does.
template <bool JAC>
__global__ void __launch_bounds__(128) k_boundary(DevMesh m, DevState s, StepArgs a) {
  if (*s.stop) return;  // the run has converged
  int b = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (b > m.nbe) return;
  int4 info = m.bed_info[b];
  const int rn = info.x, gn = info.y, bc = info.z;
  double* xnb = s.xn_bedges + 3 * (long)b;
  double nx = xnb[0], ny = xnb[1];
  const double gamma = a.gamma;
  double4 qi4 = reinterpret_cast<const double4*>(s.nQ)[rn];
  double4 qg4 = reinterpret_cast<const double4*>(s.nQ)[gn];
  double rhoi = qi4.x, ui = qi4.y / rhoi, vi = qi4.z / rhoi;
  double pi = (gamma - 1.) * (qi4.w - 0.5 * rhoi * (ui * ui + vi * vi));
  double ci = sqrt((gamma * pi) / rhoi);
  double rhob = qg4.x, ub = qg4.y / rhob, vb = qg4.z / rhob;
  double pb = (gamma - 1.) * (qg4.w - 0.5 * rhob * (ub * ub + vb * vb));
  double cb = sqrt((gamma * pb) / rhob);
  double rho0 = 0.5 * (rhoi + rhob);
  double c0 = 0.5 * (ci + cb);
  double theta = ui * nx + vi * ny;
  double ev1 = theta, ev3 = theta + ci, ev4 = theta - ci;
  bool ok = true;
  if (bc == 0 || (bc % 2 == 0)) {
    if (ev1 <= 0.0 && ev4 <= 0.0) {
      if (ev3 >= 0.0) {
        pb = 0.5 * (a.pinf + pi - rho0 * c0 * ((a.uinf - ui) * nx + (a.vinf - vi) * ny));
        rhob = 1.0 + (pb - a.pinf) / (c0 * c0);
        ub = a.uinf + (pb - a.pinf) / (rho0 * c0) * nx;
        vb = a.vinf + (pb - a.pinf) / (rho0 * c0) * ny;
      } else if (ev3 < 0.0) {
        rhob = 1.0; ub = a.uinf; vb = a.vinf; pb = a.pinf;
      } else {
        ok = false;
      }
    } else if (ev1 >= 0.0 && ev3 >= 0.0) {
      if (ev4 <= 0.0) {
        pb = a.pinf;
        rhob = rhoi + (pb - pi) / (c0 * c0);
        ub = ui - (pb - pi) / (rho0 * c0) * nx;
        vb = vi - (pb - pi) / (rho0 * c0) * ny;
      } else if (ev4 > 0.0) {
        rhob = rhoi; ub = ui; vb = vi; pb = pi;
      } else {
        ok = false;
      }
    } else {
      ok = false;
    }
  } else {
    pb = pi + rho0 * c0 * theta;
    rhob = rhoi + (pb - pi) / (c0 * c0);
    ub = ui - (pb - pi) / (rho0 * c0) * nx;
    vb = vi - (pb - pi) / (rho0 * c0) * ny;
  }
  if (!ok) {
    atomicOr(s.status, ERR_BC);
    return;
  }
  double qg[4];
  qg[0] = rhob;
  qg[1] = rhob * ub;
  qg[2] = rhob * vb;
  qg[3] = pb / (gamma - 1.0) + 0.5 * rhob * (ub * ub + vb * vb);
  if (rhob < 0.0) {  // cvbc.C:447-470
    rhob = rhoi;
    ub = (1. - 2. * nx * nx) * ui - 2. * nx * ny * vi;
    vb = (1. - 2. * ny * ny) * vi - 2. * nx * ny * ui;
    pb = pi;
    qg[0] = rhob;
    qg[1] = rhob * ub;
    qg[2] = rhob * vb;
    qg[3] = pb / (gamma - 1.0) + 0.5 * rhob * (ub * ub + vb * vb);
  }
  reinterpret_cast<double4*>(s.nQ)[gn] = make_double4(qg[0], qg[1], qg[2], qg[3]);

  double len = xnb[2];
  if (a.gauss && bc > 10) {
    double2 cn = m.bed_cnrm[b];
    nx = cn.x;
    ny = cn.y;
    len = m.xgn_bedges[9 * (long)b + 2];
    xnb[0] = nx;
    xnb[1] = ny;
  }
  double qL[4] = {qi4.x, qi4.y, qi4.z, qi4.w};
  double flux[4];
  roe_flux(nx, ny, len, gamma, qL, qg, flux);
  reinterpret_cast<double4*>(s.Fb)[b] = make_double4(flux[0], flux[1], flux[2], flux[3]);
  if (!JAC) return;
  double Rm[16];
  roe_matrix(nx, ny, gamma, qL, qg, Rm);
  double d[16];
  euler_jacobian(qL, nx, ny, gamma, d);
  double* Jo = s.Jb + 16 * (long)b;
#pragma unroll
  for (int k = 0; k < 16; k++) Jo[k] = 0.5 * (d[k] + Rm[k]) * len;
}

// LHS = 0 with V/dt on the diagonal blocks (init_memory.C:189-290).
__global__ void __launch_bounds__(128) k_diag_only(DevMesh m, DevState s) {
  int n = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (n > m.nn) return;
  double d = m.cv_area[n] / (s.dt[n]);
  for (int k = m.ia[n]; k < m.ia[n + 1]; k++) {
    double4* out = reinterpret_cast<double4*>(s.LHS + 16 * (long)k);
    bool dg = m.ja[k] == n;
    out[0] = make_double4(dg ? d : 0., 0., 0., 0.);
    out[1] = make_double4(0., dg ? d : 0., 0., 0.);
    out[2] = make_double4(0., 0., dg ? d : 0., 0.);
    out[3] = make_double4(0., 0., 0., dg ? d : 0.);
  }
}

// ---------------------------------------------------------------------------
// Ordered block Gauss-Seidel sweep (linear_algebra.C:178-344).  Rows are
// handed out in the reference's order (ascending forward, descending
// backward) by an atomic dispenser; one warp per row.  The sweep writes its
// results into dq_new, which is filled with an all-ones bit pattern (a NaN
// no arithmetic produces) before the sweep: a row that needs a neighbour the
// reference updates earlier in the same sweep polls that neighbour's four
// values until none is the pattern any more (each 8-byte store is
// single-copy atomic), so the value itself is the ready signal.  Other
// neighbours and the row's own previous value come from dq_old.  Rows are
// only claimed by running warps and every dependency was claimed earlier,
// so the earliest unfinished row always proceeds; every wait is nevertheless
// bounded and reports ERR_SWEEP_TIMEOUT instead of spinning forever.
// Lanes: 8 block slots x 4 matrix rows.
constexpr unsigned long long kNotReady = 0xFFFFFFFFFFFFFFFFull;

__device__ __forceinline__ unsigned long long ld_relaxed_u64(const double* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_relaxed_f64(double* p, double v) {
  asm volatile("st.relaxed.gpu.global.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}

template <bool FWD>
__global__ void __launch_bounds__(128) k_sweep_ordered(DevMesh m, DevState s,
                                                       const double* __restrict__ dq_old,
                                                       double* dq_new, long max_spin) {
  if (*s.stop) return;  // the run has converged
  if (*s.skip) return;
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int slot = lane >> 2, r = lane & 3;
  const int nn = m.nn;
  for (;;) {
    unsigned t = 0;
    if (lane == 0) t = atomicAdd(s.counter, 1u);
    t = __shfl_sync(FULL, t, 0);
    if (t >= (unsigned)nn) break;
    const int j = FWD ? (int)(1 + t) : (int)(nn - t);
    const int k0 = m.ia[j], k1 = m.ia[j + 1];
    // everything that does not depend on this sweep's results first
    double acc = s.RHS[4 * (long)j + r];
    const double lu_v = (lane < 16) ? s.LUd[16 * (long)j + lane] : 0.;
    const double old_v = (lane < 4) ? dq_old[4 * (long)j + lane] : 0.;
    bool timeout = false;
    for (int base = k0; base < k1; base += 8) {
      const int k = base + slot;
      int c = 0;
      bool use = false;
      double a0 = 0., a1 = 0., a2 = 0., a3 = 0.;
      if (k < k1) {
        c = m.ja[k];
        use = c != j;
        if (use) {
          const double4 av = reinterpret_cast<const double4*>(s.LHS + 16 * (long)k)[r];
          a0 = av.x; a1 = av.y; a2 = av.z; a3 = av.w;
        }
      }
      double term = 0.;
      if (use) {
        const bool dep = FWD ? (c < j) : (c > j);
        double d0, d1, d2, d3;
        if (dep) {
          const double* src = dq_new + 4 * (long)c;
          unsigned long long u0, u1, u2, u3;
          long spins = 0;
          for (;;) {
            u0 = ld_relaxed_u64(src);
            u1 = ld_relaxed_u64(src + 1);
            u2 = ld_relaxed_u64(src + 2);
            u3 = ld_relaxed_u64(src + 3);
            if (u0 != kNotReady && u1 != kNotReady && u2 != kNotReady && u3 != kNotReady) break;
            if (++spins > max_spin) {
              atomicOr(s.status, ERR_SWEEP_TIMEOUT);
              timeout = true;
              break;
            }
            // once any wait has timed out, every other wait gives up too
            if ((spins & 1023) == 0 && (*(volatile int*)s.status & ERR_SWEEP_TIMEOUT)) {
              timeout = true;
              break;
            }
            if (spins > 256) __nanosleep(32);
          }
          d0 = __longlong_as_double((long long)u0);
          d1 = __longlong_as_double((long long)u1);
          d2 = __longlong_as_double((long long)u2);
          d3 = __longlong_as_double((long long)u3);
        } else {
          const double2* dq = reinterpret_cast<const double2*>(dq_old + 4 * (long)c);
          const double2 x01 = __ldcg(dq), x23 = __ldcg(dq + 1);
          d0 = x01.x; d1 = x01.y; d2 = x23.x; d3 = x23.y;
        }
        term = (a0 * d0 + a1 * d1 + a2 * d2 + a3 * d3);
      }
      const unsigned used = __ballot_sync(FULL, use);
#pragma unroll
      for (int sl = 0; sl < 8; sl++) {
        double tv = __shfl_sync(FULL, term, sl * 4 + r);
        if (used & (1u << (sl * 4))) acc -= tv;
      }
    }
    double b[4], M[16], o[4];
#pragma unroll
    for (int q = 0; q < 4; q++) b[q] = __shfl_sync(FULL, acc, q);
#pragma unroll
    for (int q = 0; q < 16; q++) M[q] = __shfl_sync(FULL, lu_v, q);
#pragma unroll
    for (int q = 0; q < 4; q++) o[q] = __shfl_sync(FULL, old_v, q);
    double X[4];
    lu_solve4(M, b, X);
    double mine = X[0], own = o[0];
#pragma unroll
    for (int q = 1; q < 4; q++)
      if (lane == q) { mine = X[q]; own = o[q]; }
    if (__any_sync(FULL, timeout)) {
      // a timed-out row publishes something so that nothing waits on it
      mine = 0.;
      own = 0.;
    }
    if (lane < 4) {
      const double dx = mine - own;
      st_relaxed_f64(dq_new + 4 * (long)j + lane, own + dx);
    }
    __syncwarp();
  }
}

// Precision form: one colour of a multicolour block Gauss-Seidel sweep in
// FP32.  Four lanes per row (lane q owns matrix row q): each lane forms
// b_q - sum_k A_k[q,:] . dQ[col_k] over the row's off-diagonal blocks in
// block order, with one multiply and three fused multiply-adds per block;
// lane 0 then solves with the FP32 LU factors (reciprocal pivots).  Rows of
// one colour share no block, so they run in parallel and in any order.  All
// loads that do not depend on the iterate (row record, blocks, columns, LU
// factors) are issued before the neighbour gathers.  The last sweep also
// writes the FP64 dQ the update reads.
constexpr int kMixedMaxB = 12;  // off-diagonal blocks held in registers per row

template <bool LAST>
__global__ void __launch_bounds__(128) k_sweep_color32(DevState s, MixedTables mt, int p0,
                                                       int p1) {
  if (*s.stop) return;  // the run has converged
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int pp = p0 + (tid >> 2), q = tid & 3;
  const int qbase = threadIdx.x & ~3 & 31;
  const unsigned qmask = 0xFu << qbase;
  if (pp >= p1) return;  // whole quads leave together
  const int4 rw = mt.rowinfo[pp];  // row, first block, end block
  const int n = rw.x, b0 = rw.y, nb = rw.z - rw.y;
  const float4* A = reinterpret_cast<const float4*>(mt.lhs32);
  const float4* X = reinterpret_cast<const float4*>(mt.dq32);
  float4 M0 = make_float4(0.f, 0.f, 0.f, 0.f), M1 = M0, M2 = M0, M3 = M0;
  if (q == 0) {
    const float4* L = reinterpret_cast<const float4*>(mt.lu32) + 4 * (long)pp;
    M0 = L[0]; M1 = L[1]; M2 = L[2]; M3 = L[3];
  }
  int cols[kMixedMaxB];
  float4 a[kMixedMaxB];
#pragma unroll
  for (int i = 0; i < kMixedMaxB; i++) {
    if (i < nb) {
      cols[i] = mt.offd_col[b0 + i];
      a[i] = A[4 * (long)(b0 + i) + q];
    }
  }
  float acc = __double2float_rn(s.RHS[4 * (long)n + q]);
#pragma unroll
  for (int i = 0; i < kMixedMaxB; i += 2) {
    if (i + 1 < nb) {
      const float4 d0 = X[cols[i]], d1 = X[cols[i + 1]];
      float t0 = __fmul_rn(a[i].x, d0.x);
      t0 = __fmaf_rn(a[i].y, d0.y, t0);
      t0 = __fmaf_rn(a[i].z, d0.z, t0);
      t0 = __fmaf_rn(a[i].w, d0.w, t0);
      float t1 = __fmul_rn(a[i + 1].x, d1.x);
      t1 = __fmaf_rn(a[i + 1].y, d1.y, t1);
      t1 = __fmaf_rn(a[i + 1].z, d1.z, t1);
      t1 = __fmaf_rn(a[i + 1].w, d1.w, t1);
      acc = __fsub_rn(acc, t0);
      acc = __fsub_rn(acc, t1);
    } else if (i < nb) {
      const float4 d0 = X[cols[i]];
      float t0 = __fmul_rn(a[i].x, d0.x);
      t0 = __fmaf_rn(a[i].y, d0.y, t0);
      t0 = __fmaf_rn(a[i].z, d0.z, t0);
      t0 = __fmaf_rn(a[i].w, d0.w, t0);
      acc = __fsub_rn(acc, t0);
    }
  }
  for (int i = kMixedMaxB; i < nb; i++) {  // rows with more blocks than the window
    const float4 ai = A[4 * (long)(b0 + i) + q];
    const float4 d0 = X[mt.offd_col[b0 + i]];
    float t0 = __fmul_rn(ai.x, d0.x);
    t0 = __fmaf_rn(ai.y, d0.y, t0);
    t0 = __fmaf_rn(ai.z, d0.z, t0);
    t0 = __fmaf_rn(ai.w, d0.w, t0);
    acc = __fsub_rn(acc, t0);
  }
  const float r0 = __shfl_sync(qmask, acc, qbase);
  const float r1 = __shfl_sync(qmask, acc, qbase + 1);
  const float r2 = __shfl_sync(qmask, acc, qbase + 2);
  const float r3 = __shfl_sync(qmask, acc, qbase + 3);
  if (q != 0) return;
  const float y0 = r0;
  const float y1 = __fmaf_rn(-M1.x, y0, r1);
  const float y2 = __fmaf_rn(-M2.y, y1, __fmaf_rn(-M2.x, y0, r2));
  const float y3 = __fmaf_rn(-M3.z, y2, __fmaf_rn(-M3.y, y1, __fmaf_rn(-M3.x, y0, r3)));
  const float x3 = __fmul_rn(y3, M3.w);
  const float x2 = __fmul_rn(__fmaf_rn(-M2.w, x3, y2), M2.z);
  const float x1 = __fmul_rn(__fmaf_rn(-M1.w, x3, __fmaf_rn(-M1.z, x2, y1)), M1.y);
  const float x0 =
      __fmul_rn(__fmaf_rn(-M0.w, x3, __fmaf_rn(-M0.z, x2, __fmaf_rn(-M0.y, x1, y0))), M0.x);
  reinterpret_cast<float4*>(mt.dq32)[n] = make_float4(x0, x1, x2, x3);
  if (LAST)
    reinterpret_cast<double4*>(s.dQ)[n] = make_double4(x0, x1, x2, x3);
}

// Precision form with the reference's row order: the ordered sweep of
// k_sweep_ordered (row dispenser, a warp per row, 8 blocks x 4 rows per
// pass, dependencies polled on this sweep's results) on FP32 blocks in row
// order (MixedTables built with the identity ordering).  Per row the
// arithmetic is that of k_sweep_color32: one multiply and three fused
// multiply-adds per block and row, subtracted in block order, then the FP32
// LU solve with reciprocal pivots.  A float's not-ready pattern is
// 0xFFFFFFFF (computed NaNs are 0x7FFFFFFF).
constexpr unsigned kNotReady32 = 0xFFFFFFFFu;

__device__ __forceinline__ unsigned ld_relaxed_u32(const float* p) {
  unsigned v;
  asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_relaxed_f32(float* p, float v) {
  asm volatile("st.relaxed.gpu.global.f32 [%0], %1;" ::"l"(p), "f"(v) : "memory");
}

template <bool FWD>
__global__ void __launch_bounds__(128) k_sweep_ordered32(DevState s, MixedTables mt, int nn,
                                                         const float* __restrict__ dq_old,
                                                         float* dq_new, int last,
                                                         long max_spin) {
  if (*s.stop) return;  // the run has converged
  if (*s.skip) return;
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int slot = lane >> 2, r = lane & 3;
  const float4* A = reinterpret_cast<const float4*>(mt.lhs32);
  for (;;) {
    unsigned t = 0;
    if (lane == 0) t = atomicAdd(s.counter, 1u);
    t = __shfl_sync(FULL, t, 0);
    if (t >= (unsigned)nn) break;
    const int j = FWD ? (int)(1 + t) : (int)(nn - t);
    const int4 rw = mt.rowinfo[j - 1];  // identity ordering: position j-1
    const int b0 = rw.y, b1 = rw.z;
    float acc = __double2float_rn(s.RHS[4 * (long)j + r]);
    const float lu_v = (lane < 16) ? mt.lu32[16 * (long)(j - 1) + lane] : 0.f;
    bool timeout = false;
    for (int base = b0; base < b1; base += 8) {
      const int k = base + slot;
      const bool use = k < b1;
      int c = 0;
      float4 a = make_float4(0.f, 0.f, 0.f, 0.f);
      if (use) {
        c = mt.offd_col[k];
        a = A[4 * (long)k + r];
      }
      float term = 0.f;
      if (use) {
        const bool dep = FWD ? (c < j) : (c > j);
        float d0, d1, d2, d3;
        if (dep) {
          const float* src = dq_new + 4 * (long)c;
          unsigned u0, u1, u2, u3;
          long spins = 0;
          for (;;) {
            u0 = ld_relaxed_u32(src);
            u1 = ld_relaxed_u32(src + 1);
            u2 = ld_relaxed_u32(src + 2);
            u3 = ld_relaxed_u32(src + 3);
            if (u0 != kNotReady32 && u1 != kNotReady32 && u2 != kNotReady32 &&
                u3 != kNotReady32)
              break;
            if (++spins > max_spin) {
              atomicOr(s.status, ERR_SWEEP_TIMEOUT);
              timeout = true;
              break;
            }
            // once any wait has timed out, every other wait gives up too
            if ((spins & 1023) == 0 && (*(volatile int*)s.status & ERR_SWEEP_TIMEOUT)) {
              timeout = true;
              break;
            }
            if (spins > 256) __nanosleep(32);
          }
          d0 = __uint_as_float(u0);
          d1 = __uint_as_float(u1);
          d2 = __uint_as_float(u2);
          d3 = __uint_as_float(u3);
        } else {
          const float4 x = __ldcg(reinterpret_cast<const float4*>(dq_old) + c);
          d0 = x.x; d1 = x.y; d2 = x.z; d3 = x.w;
        }
        term = __fmul_rn(a.x, d0);
        term = __fmaf_rn(a.y, d1, term);
        term = __fmaf_rn(a.z, d2, term);
        term = __fmaf_rn(a.w, d3, term);
      }
      const unsigned used = __ballot_sync(FULL, use);
#pragma unroll
      for (int sl = 0; sl < 8; sl++) {
        const float tv = __shfl_sync(FULL, term, sl * 4 + r);
        if (used & (1u << (sl * 4))) acc = __fsub_rn(acc, tv);
      }
    }
    const float r0 = __shfl_sync(FULL, acc, 0), r1 = __shfl_sync(FULL, acc, 1);
    const float r2 = __shfl_sync(FULL, acc, 2), r3 = __shfl_sync(FULL, acc, 3);
    float M[16];
#pragma unroll
    for (int q = 0; q < 16; q++) M[q] = __shfl_sync(FULL, lu_v, q);
    const float y0 = r0;
    const float y1 = __fmaf_rn(-M[4], y0, r1);
    const float y2 = __fmaf_rn(-M[9], y1, __fmaf_rn(-M[8], y0, r2));
    const float y3 = __fmaf_rn(-M[14], y2, __fmaf_rn(-M[13], y1, __fmaf_rn(-M[12], y0, r3)));
    const float x3 = __fmul_rn(y3, M[15]);
    const float x2 = __fmul_rn(__fmaf_rn(-M[11], x3, y2), M[10]);
    const float x1 = __fmul_rn(__fmaf_rn(-M[7], x3, __fmaf_rn(-M[6], x2, y1)), M[5]);
    const float x0 =
        __fmul_rn(__fmaf_rn(-M[3], x3, __fmaf_rn(-M[2], x2, __fmaf_rn(-M[1], x1, y0))), M[0]);
    float mine = lane == 0 ? x0 : lane == 1 ? x1 : lane == 2 ? x2 : x3;
    // a timed-out row publishes something so that nothing waits on it
    if (__any_sync(FULL, timeout)) mine = 0.f;
    if (lane < 4) {
      st_relaxed_f32(dq_new + 4 * (long)j + lane, mine);
      if (last) s.dQ[4 * (long)j + lane] = (double)mine;
    }
    __syncwarp();
  }
}

// Before an FP32 ordered sweep: its result buffer gets the not-ready pattern
// (or the current iterate when the sweep will not run).
__global__ void k_prepare_sweep32(DevState s, const float* cur, float* next, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < 4 || i >= n) return;  // row 0 is unused
  if (*s.stop || *s.skip)
    next[i] = cur[i];
  else
    next[i] = __uint_as_float(kNotReady32);
}

// Precision form, chunked order (mode 3): one colour of chunks, a CTA per
// chunk, 64 rows (one per quad of 4 lanes, lane r owning block row r) per
// pass.  The CTA first copies its window of the FP32 iterate (every row its
// chunk touches) into shared memory, then walks the chunk's sub-levels in
// order: the records of sub-level u+S-1 are copied into an S-slot ring with
// cp.async while sub-level u is computed, so the dependency chain only ever
// reads shared memory.  The ring holds kRingRecords records in one of three
// shapes (ROWS rows a sub-level x S slots: 64 x 3, 32 x 6, 16 x 12): smaller
// sub-levels prefetch further ahead for the same shared memory, at the
// price of more barriers on levels wider than ROWS rows.  Rows of one sub-level are independent; a barrier
// separates sub-levels.  Rows of other chunks in the window are not written
// by any CTA of this launch (chunks of one colour share no block).  Per row
// the arithmetic is that of k_sweep_color32.
constexpr int kRecRows = 64;        // rows of a sub-level in the largest ring shape
constexpr int kRingRecords = 192;   // records the ring holds, whatever its shape
constexpr int kRingShapes = 3;      // sub-levels of 64, 32 or 16 rows
__host__ __device__ constexpr int ring_rows(int shape) { return 64 >> shape; }
constexpr int kRecInts = (int)(sizeof(SweepRec) / 16);  // 16-byte words per record
// records sit 704 bytes apart in shared memory (640 + 64 of padding), so the
// two quads of a half-warp read disjoint bank ranges
constexpr int kRecStride = kRecInts + 4;
constexpr int kChunkSubMax = 256;   // sub-levels per chunk (host-checked)
// shared memory the chunk sweep declares statically (room left for the rest)
constexpr int kChunkStaticSmem = 2048;


// Static part of mode 3's sweep records: record i holds row order[i]'s
// header (row, off-diagonal block count; the diagonal block is the row's
// last) and its off-diagonal column indices, every other word zero until
// assembly writes the values.  One thread per 16-byte word: word 0 the
// header, 1 the right-hand side, 2-5 the LU factors, 6-7 the columns, 8-39
// the blocks.
static_assert(offsetof(SweepRec, cols) == 6 * 16 && offsetof(SweepRec, a) == 8 * 16 &&
                  sizeof(SweepRec) == 40 * 16,
              "k_fill_sweep_records assumes the SweepRec word layout");
__global__ void k_fill_sweep_records(SweepRec* __restrict__ rec, const int* __restrict__ order,
                                     int nrec, const int* __restrict__ ia,
                                     const int* __restrict__ ja) {
  const long w = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (w >= (long)nrec * kRecInts) return;
  const int i = (int)(w / kRecInts), k = (int)(w - (long)i * kRecInts);
  int4 v = make_int4(0, 0, 0, 0);
  if (k == 0 || k == 6 || k == 7) {
    const int j = order[i];
    const int k0 = ia[j], nb = ia[j + 1] - k0 - 1;
    if (k == 0) {
      v = make_int4(j, nb, 0, 0);
    } else {
      const int t0 = 4 * (k - 6);
      v.x = t0 + 0 < nb ? ja[k0 + t0 + 0] : 0;
      v.y = t0 + 1 < nb ? ja[k0 + t0 + 1] : 0;
      v.z = t0 + 2 < nb ? ja[k0 + t0 + 2] : 0;
      v.w = t0 + 3 < nb ? ja[k0 + t0 + 3] : 0;
    }
  }
  reinterpret_cast<int4*>(rec)[w] = v;
}

// One chunk q of a mode 3 sweep, run by the whole CTA (256 threads).  The
// colour-synchronous kernel (DF false) queues the chunk's window of the
// iterate first and its first sub-levels' records after it; the dataflow
// kernel (DF true) queues the records first, calls wait_deps() (which
// returns once the chunk's earlier-colour neighbours have finished this
// sweep, every thread past a barrier) and only then reads the window.
// reuse_window: the chunk's window is already in shared memory, current (the
// CTA's previous pass over the same chunk left it there).
template <int DIR, int ROWS, bool DF, class Wait>
__device__ __forceinline__ void sweep_chunk_body(const DevState& s, const ChunkTables& ct,
                                                 float* dq32, int q, int last, int* ss,
                                                 Wait&& wait_deps, bool reuse_window = false) {
  constexpr int SLOTS = kRingRecords / ROWS;
  static_assert(SLOTS * ROWS == kRingRecords && SLOTS >= 3 && 4 * ROWS <= 256,
                "ring shape");
  extern __shared__ __align__(16) unsigned char sweep_smem[];
  int4* slots = reinterpret_cast<int4*>(sweep_smem);
  float4* win = reinterpret_cast<float4*>(sweep_smem + 16 * kRecStride * kRingRecords);
  const int tid = threadIdx.x;
  const int2 w = ct.window[q];
  const int nwin = w.y - w.x + 1;
  float4* X = reinterpret_cast<float4*>(dq32);
  auto load_window = [&]() {
    if (!reuse_window)
      for (int i = tid; i < nwin; i += blockDim.x) cp_async16(win + i, X + w.x + i);
    cp_async_commit();
  };
  if (!DF) load_window();
  const int S0 = ct.chunk_sub[DIR][q], nsub = ct.chunk_sub[DIR][q + 1] - S0;
  // the chunk's sub-level starts, read once into shared memory ss (the
  // caller's kChunkSubMax + 1 ints; they sit on the loop's critical path); a
  // chunk has at most kChunkSubMax sub-levels
  for (int i = tid; i <= nsub && i <= kChunkSubMax; i += blockDim.x)
    ss[i] = ct.sub_start[DIR][S0 + i];
  __syncthreads();
  const int4* recs = reinterpret_cast<const int4*>(ct.rec[DIR]);
  auto issue = [&](int u) {
    if (u < nsub) {
      const int r0 = ss[u], words = (ss[u + 1] - r0) * kRecInts;
      const int4* src = recs + (long)r0 * kRecInts;
      int4* dst = slots + (u % SLOTS) * ROWS * kRecStride;
      for (int i = tid; i < words; i += blockDim.x) {
        const int rr = i / kRecInts, ww = i - rr * kRecInts;
        cp_async16(dst + rr * kRecStride + ww, src + i);
      }
    }
    cp_async_commit();  // one group per sub-level, empty past the end
  };
  for (int k = 0; k < SLOTS - 1; k++) issue(k);
  const int quad = tid >> 2, r = tid & 3;
  const int qbase = tid & 31 & ~3;
  const unsigned qmask = 0xFu << qbase;
  if (DF) {
    wait_deps();
    load_window();
    cp_async_wait<0>();  // the window and the first sub-levels have landed
  } else {
    cp_async_wait<SLOTS - 2>();  // the window and sub-level 0 have landed
  }
  __syncthreads();
  for (int u = 0; u < nsub; u++) {
    issue(u + SLOTS - 1);  // into the slot sub-level u-1 left
    if (quad < ss[u + 1] - ss[u]) {
      const SweepRec& R = *reinterpret_cast<const SweepRec*>(
          slots + ((u % SLOTS) * ROWS + quad) * kRecStride);
      const int j = R.hdr.x, nb = R.hdr.y;
      const int* cols = reinterpret_cast<const int*>(R.cols);
      float acc = reinterpret_cast<const float*>(&R.rhs)[r];
#pragma unroll
      for (int t = 0; t < kRecBlocks; t++) {
        if (t < nb) {
          const float4 a = R.a[4 * t + r];
          const float4 d = win[cols[t] - w.x];
          float tt = __fmul_rn(a.x, d.x);
          tt = __fmaf_rn(a.y, d.y, tt);
          tt = __fmaf_rn(a.z, d.z, tt);
          tt = __fmaf_rn(a.w, d.w, tt);
          acc = __fsub_rn(acc, tt);
        }
      }
      const float b0 = __shfl_sync(qmask, acc, qbase);
      const float b1 = __shfl_sync(qmask, acc, qbase + 1);
      const float b2 = __shfl_sync(qmask, acc, qbase + 2);
      const float b3 = __shfl_sync(qmask, acc, qbase + 3);
      if (r == 0) {
        const float4 M0 = R.lu[0], M1 = R.lu[1], M2 = R.lu[2], M3 = R.lu[3];
        const float y0 = b0;
        const float y1 = __fmaf_rn(-M1.x, y0, b1);
        const float y2 = __fmaf_rn(-M2.y, y1, __fmaf_rn(-M2.x, y0, b2));
        const float y3 = __fmaf_rn(-M3.z, y2, __fmaf_rn(-M3.y, y1, __fmaf_rn(-M3.x, y0, b3)));
        const float x3 = __fmul_rn(y3, M3.w);
        const float x2 = __fmul_rn(__fmaf_rn(-M2.w, x3, y2), M2.z);
        const float x1 = __fmul_rn(__fmaf_rn(-M1.w, x3, __fmaf_rn(-M1.z, x2, y1)), M1.y);
        const float x0 = __fmul_rn(
            __fmaf_rn(-M0.w, x3, __fmaf_rn(-M0.z, x2, __fmaf_rn(-M0.y, x1, y0))), M0.x);
        const float4 x = make_float4(x0, x1, x2, x3);
        win[j - w.x] = x;
        X[j] = x;
        if (last) reinterpret_cast<double4*>(s.dQ)[j] = make_double4(x0, x1, x2, x3);
      }
    }
    // one barrier per sub-level: this level's results are visible to the
    // next, and the next level's records (all but the newest SLOTS-2 copy
    // groups) have landed
    cp_async_wait<SLOTS - 2>();
    __syncthreads();
  }
  cp_async_wait<0>();
}

template <int DIR, int ROWS>
__global__ void __launch_bounds__(256) k_sweep_chunk(DevState s, ChunkTables ct, float* dq32,
                                                     int colour, int last) {
  if (*s.stop) return;  // the run has converged
  const int q = ct.col_chunks[ct.col_ptr[colour] + blockIdx.x];
  __shared__ int ss[kChunkSubMax + 1];
  sweep_chunk_body<DIR, ROWS, false>(s, ct, dq32, q, last, ss, [] {});
}

// Two passes of one colour back to back: the DIR pass of a sweep (it ends
// with this colour) and the opposite pass of the next sweep (it starts with
// it).  Chunks of one colour read only rows of other colours and their own,
// and no other colour runs between the two passes, so each chunk sweeps
// itself twice with its window kept in shared memory: what two launches
// compute, with one launch, one window load and no barrier between them.
template <int DIR, int ROWS>
__global__ void __launch_bounds__(256) k_sweep_chunk_pair(DevState s, ChunkTables ct,
                                                          float* dq32, int colour, int last) {
  if (*s.stop) return;  // the run has converged
  const int q = ct.col_chunks[ct.col_ptr[colour] + blockIdx.x];
  __shared__ int ss[kChunkSubMax + 1];
  sweep_chunk_body<DIR, ROWS, false>(s, ct, dq32, q, 0, ss, [] {});
  __syncthreads();  // the first pass's window is complete before the second reads it
  sweep_chunk_body<1 - DIR, ROWS, false>(s, ct, dq32, q, last, ss, [] {}, true);
}

// A whole mode 3 sweep in one launch (one CTA per chunk): CTAs take chunks
// from a dispenser in the sweep's colour order, and a chunk waits only for
// the chunks of earlier colours its window overlaps (finished this sweep),
// not for every chunk of the colour before it.  A chunk reads exactly what
// it reads in the colour-synchronous sweep: its earlier-colour neighbours
// after their update, its later-colour neighbours before theirs (they take
// their chunks later and wait for this one), so the results are the same.
// A chunk only waits for chunks dispensed before it, held by CTAs that are
// running or done, so the waits end whatever the residency.  ct.sync: [0]
// the dispenser, [1] chunks finished, [2] the sweep generation; the last
// chunk to finish resets [0] and [1] and advances [2], and a finished chunk
// stores generation + 1 in ct.done.  A wait gives up after max_spin polls,
// sets FLOW_ERR_SWEEP_TIMEOUT and goes on (the chunk still finishes, so the
// counters stay consistent).
template <int DIR>
__global__ void __launch_bounds__(256) k_sweep_chunk_df(DevState s, ChunkTables ct,
                                                        float* dq32, int last, long max_spin) {
  if (*s.stop) return;  // the run has converged (every CTA of the launch sees it)
  __shared__ int task_q, task_gen;
  if (threadIdx.x == 0) {
    const unsigned t = atomicAdd(&ct.sync[0], 1u);
    task_gen = cuda::atomic_ref<unsigned, cuda::thread_scope_device>(ct.sync[2])
                   .load(cuda::memory_order_relaxed);
    task_q = t < (unsigned)ct.nchunks ? ct.task_chunk[DIR][t] : -1;
  }
  __syncthreads();
  const int q = task_q;
  const int gen = task_gen;
  if (q < 0) {  // more CTAs than chunks: only a broken launch gets here
    if (threadIdx.x == 0) atomicOr(s.status, ERR_SWEEP_TIMEOUT);
    return;
  }
  auto wait_deps = [&]() {
    if (threadIdx.x == 0) {
      const int mine = DIR == 0 ? ct.colour[q] : ct.ncol - 1 - ct.colour[q];
      const int2 nr = ct.nbr[q];
      for (int o = nr.x; o <= nr.y; o++) {
        const int rank = DIR == 0 ? ct.colour[o] : ct.ncol - 1 - ct.colour[o];
        if (o == q || rank >= mine) continue;
        cuda::atomic_ref<int, cuda::thread_scope_device> flag(ct.done[o]);
        long spin = 0;
        while (flag.load(cuda::memory_order_acquire) != gen + 1) {
          if (++spin > max_spin) {
            atomicOr(s.status, ERR_SWEEP_TIMEOUT);
            break;
          }
        }
      }
    }
    __syncthreads();
  };
  __shared__ int ss[kChunkSubMax + 1];
  sweep_chunk_body<DIR, 64, true>(s, ct, dq32, q, last, ss, wait_deps);
  // publish: every thread's iterate writes before the chunk's flag
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    cuda::atomic_ref<int, cuda::thread_scope_device>(ct.done[q])
        .store(gen + 1, cuda::memory_order_release);
    if (atomicAdd(&ct.sync[1], 1u) == (unsigned)ct.nchunks - 1) {
      // every chunk of this sweep has finished (and read the generation)
      atomicExch(&ct.sync[0], 0u);
      atomicExch(&ct.sync[1], 0u);
      __threadfence();
      atomicAdd(&ct.sync[2], 1u);
    }
  }
}

// Before an ordered sweep: fill its result buffer with the not-ready
// pattern.  When the sweep will not run (the run converged, or the linear
// residual already dropped below 1e-15, linear_algebra.C:389) carry the
// current dQ over instead, so that the buffer swap after the sweep keeps it.
__global__ void k_prepare_sweep(DevState s, const double* cur, double* next, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < 4 || i >= n) return;  // row 0 is unused (and stays zero)
  if (*s.stop || *s.skip)
    next[i] = cur[i];
  else
    next[i] = __longlong_as_double((long long)0xFFFFFFFFFFFFFFFFull);
}

// ---------------------------------------------------------------------------
// Deterministic block reduction helper: fixed tree over kRedThreads lanes.
__device__ __forceinline__ double block_sum(double v, double* sh) {
  const int tid = threadIdx.x;
  sh[tid] = v;
  __syncthreads();
#pragma unroll
  for (int w = kRedThreads / 2; w > 0; w >>= 1) {
    if (tid < w) sh[tid] += sh[tid + w];
    __syncthreads();
  }
  double out = sh[0];
  __syncthreads();
  return out;
}

// b - Ax of every row (linear_algebra.C:348-387), squared, partial sums.
__global__ void __launch_bounds__(kRedThreads) k_lin_residual(DevMesh m, DevState s) {
  if (*s.stop) return;  // the run has converged
  __shared__ double sh[kRedThreads];
  double acc = 0.;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x + 1; j <= m.nn;
       j += gridDim.x * blockDim.x) {
    double r[4];
    const double4 rh = reinterpret_cast<const double4*>(s.RHS)[j];
    r[0] = rh.x; r[1] = rh.y; r[2] = rh.z; r[3] = rh.w;
    for (int k = m.ia[j]; k < m.ia[j + 1]; k++) {
      const double4 d4 = reinterpret_cast<const double4*>(s.dQ)[m.ja[k]];
      const double d[4] = {d4.x, d4.y, d4.z, d4.w};
      const double* A = s.LHS + 16 * (long)k;
#pragma unroll
      for (int q = 0; q < 4; q++) r[q] -= row_dot(A, q, d);
    }
    acc += (r[0] * r[0] + r[1] * r[1] + r[2] * r[2] + r[3] * r[3]);
  }
  double tot = block_sum(acc, sh);
  if (threadIdx.x == 0) s.partial[blockIdx.x] = tot;
}

// Sum the partials in a fixed order; slot 0 = RMS (sets skip below 1e-15).
// The tree sum differs from the reference's row-order sum by at most
// (nn-1) u of the sum (u = 2^-53, every term is positive), so the RMS by at
// most about half that: when the RMS lies that close to the 1e-15 test of
// linear_algebra.C:387, k_exact_rms settles the test in the reference's order.
__global__ void k_finalize_rms(DevState s, int nparts, int nn, int always_exact) {
  if (*s.stop) return;  // the run has converged
  __shared__ double sh[kRedThreads];
  double v = 0.;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) v += s.partial[i];
  double tot = block_sum(v, sh);
  if (threadIdx.x == 0) {
    double rms = tot / (1. * nn);
    rms = sqrt(rms);
    s.scalars[0] = rms;
    if (rms < 1.0E-15) *s.skip = 1;
    if (always_exact || fabs(rms - 1.0E-15) <= 1.0E-15 * ((nn + 16.) * 2.3e-16)) *s.exact = 1;
  }
}

// The b - Ax RMS in the reference's order (linear_algebra.C:348-387), run only
// when k_finalize_rms found the tree RMS within its error bound of 1e-15: the
// CTA forms 256 rows' squared residuals at a time, thread 0 adds them in row
// order.  It sets the RMS and the skip flag as the reference's test decides.
__global__ void __launch_bounds__(256) k_exact_rms(DevMesh m, DevState s) {
  if (*s.stop || !*s.exact) return;
  __shared__ double term[256];
  double acc = 0.;
  for (int j0 = 1; j0 <= m.nn; j0 += 256) {
    const int j = j0 + threadIdx.x;
    if (j <= m.nn) {
      double r[4];
      const double4 rh = reinterpret_cast<const double4*>(s.RHS)[j];
      r[0] = rh.x; r[1] = rh.y; r[2] = rh.z; r[3] = rh.w;
      for (int k = m.ia[j]; k < m.ia[j + 1]; k++) {
        const double4 d4 = reinterpret_cast<const double4*>(s.dQ)[m.ja[k]];
        const double d[4] = {d4.x, d4.y, d4.z, d4.w};
        const double* A = s.LHS + 16 * (long)k;
#pragma unroll
        for (int q = 0; q < 4; q++) r[q] -= row_dot(A, q, d);
      }
      term[threadIdx.x] = (r[0] * r[0] + r[1] * r[1] + r[2] * r[2] + r[3] * r[3]);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      const int cnt = min(256, m.nn - j0 + 1);
      for (int t = 0; t < cnt; t++) acc += term[t];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    double rms = acc;
    rms /= (1. * m.nn);
    rms = sqrt(rms);
    s.scalars[0] = rms;
    *s.skip = rms < 1.0E-15 ? 1 : 0;
    *s.exact = 0;
  }
}

// The step's norms from the per-block partial sums (summed in block order,
// the same bits whatever block forms them), the history, the run's first
// residual, the step count and the stop flag.
__device__ __forceinline__ void finalize_step_body(DevState& s, double* sh, double* hist_dq,
                                                   double* hist_r, int slot, int first) {
  double a = 0., b = 0.;
  for (int i = threadIdx.x; i < kRedBlocks; i += blockDim.x) {
    a += __ldcg(s.partial + i);
    b += __ldcg(s.partial + kRedBlocks + i);
  }
  double ta = block_sum(a, sh);
  double tb = block_sum(b, sh);
  if (threadIdx.x == 0) {
    s.scalars[1] = ta;
    s.scalars[2] = tb;
    double r = sqrt(tb);
    if (hist_dq) hist_dq[slot] = sqrt(ta);
    if (hist_r) hist_r[slot] = r;
    // first < 0: the first step of the run is the one with no step done yet
    if (first > 0 || (first < 0 && *s.steps_done == 0)) s.scalars[6] = r;
    *s.steps_done += 1;
    // stop once ||R_rho|| < drop * ||R_rho|| of the first step
    if (s.scalars[7] > 0. && r < s.scalars[7] * s.scalars[6]) *s.stop = 1;
  }
}

// nQ += dQ, pQ <- Q, Q <- nQ (solve.C:901-928) and partial sums of |dQ|^2
// and |R_rho|^2; the last block to finish sums the partials
// (finalize_step_body), so the step needs no separate one-block launch.
// The blocks count themselves in the word after the partials, which the
// last block sets back to zero.
__global__ void __launch_bounds__(kRedThreads) k_finish_step(DevMesh m, DevState s, int last,
                                                            double* hist_dq, double* hist_r,
                                                            int slot, int first) {
  if (*s.stop) return;  // the run has converged (every block sees the same flag)
  __shared__ double sh[kRedThreads];
  __shared__ int is_last;
  double dq2 = 0., r2 = 0.;
  const int total = m.nn + m.ng;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x + 1; i <= total;
       i += gridDim.x * blockDim.x) {
    double4 nq = reinterpret_cast<const double4*>(s.nQ)[i];
    if (i <= m.nn) {
      double4 d = reinterpret_cast<const double4*>(s.dQ)[i];
      dq2 += (d.x * d.x + d.y * d.y + d.z * d.z + d.w * d.w);
      double rr = s.R[4 * (long)i];
      r2 += rr * rr;
      nq.x += d.x; nq.y += d.y; nq.z += d.z; nq.w += d.w;
      reinterpret_cast<double4*>(s.nQ)[i] = nq;
    }
    if (last) {
      reinterpret_cast<double4*>(s.pQ)[i] = reinterpret_cast<const double4*>(s.Q)[i];
      reinterpret_cast<double4*>(s.Q)[i] = nq;
    }
  }
  double a = block_sum(dq2, sh);
  double b = block_sum(r2, sh);
  unsigned* done = reinterpret_cast<unsigned*>(s.partial + 2 * kRedBlocks);
  if (threadIdx.x == 0) {
    s.partial[blockIdx.x] = a;
    s.partial[kRedBlocks + blockIdx.x] = b;
    __threadfence();  // the partials are visible before the count says so
    is_last = atomicAdd(done, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!is_last) return;
  __threadfence();
  finalize_step_body(s, sh, hist_dq, hist_r, slot, first);
  if (threadIdx.x == 0) *done = 0u;
}

// ---------------------------------------------------------------------------
// Compute_Body_Forces (grid_io.C:1430-1694): per wall bedge the 3-point
// pressure integral, then the reference's sequential sum over bedges.
__device__ __forceinline__ void recon_boundary_point(const DevMesh& m, const DevState& s, int n,
                                                     int order, const double* gp, double* q) {
  double4 q4 = reinterpret_cast<const double4*>(s.nQ)[n];
  q[0] = q4.x; q[1] = q4.y; q[2] = q4.z; q[3] = q4.w;
  if (order == 0) return;
  double phi = s.phi[8 * (long)n], sig = s.phi[8 * (long)n + 1];
  double dx0 = gp[0] - m.x[2 * n], dx1 = gp[1] - m.x[2 * n + 1];
  if (order == 1) {
    const double* g = s.grad + 8 * (long)n;
#pragma unroll
    for (int j = 0; j < 4; j++) q[j] += (phi * g[2 * j] * dx0 + phi * g[2 * j + 1] * dx1);
  } else {
    const double* h = s.hess5 + 20 * (long)n;
#pragma unroll
    for (int j = 0; j < 4; j++) q[j] = s.pv[4 * (long)n + j];
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const double* hh = h + 5 * j;
      q[j] += (phi * hh[0] * dx0 + phi * hh[1] * dx1 + sig * hh[2] * dx0 * dx0 * 0.5 +
               sig * hh[3] * dx1 * dx1 * 0.5 + sig * hh[4] * dx0 * dx1);
    }
  }
}

__global__ void k_body_forces(DevMesh m, DevState s, StepArgs a, int recon_order) {
  int b = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (b > m.nbe) return;
  int4 info = m.bed_info[b];
  double* out = s.bforce + 4 * (long)b;
  if (!info.w) {
    out[0] = 0.;
    out[1] = 0.;
    out[2] = 0.;
    return;
  }
  const int rn = info.x, bc = info.z;
  double t1 = 0., t2 = 0., len, q[4];
  if (bc <= 10) {
    const double* xnb = s.xn_bedges + 3 * (long)b;
    double nx = -xnb[0], ny = -xnb[1];
    len = xnb[2];
    const double w[3] = {5. / 9., 8. / 9., 5. / 9.};
    for (int k = 0; k < 3; k++) {
      recon_boundary_point(m, s, rn, recon_order, m.xg_bedges + 6 * (long)b + 2 * k, q);
      double rr = q[0], u = q[1] / rr, v = q[2] / rr, e = q[3];
      double P = (a.gamma - 1.) * (e - 0.5 * rr * (u * u + v * v));
      t1 += (w[k] * (P * ny * a.cos_a - P * nx * a.sin_a));
      t2 += (w[k] * (P * nx * a.cos_a + P * ny * a.sin_a));
    }
  } else {
    len = m.xgn_bedges[9 * (long)b + 2];
    const double w[3] = {8. / 9., 5. / 9., 5. / 9.};
    for (int k = 0; k < 3; k++) {
      double nx = -m.xgn_bedges[9 * (long)b + 3 * k], ny = -m.xgn_bedges[9 * (long)b + 3 * k + 1];
      recon_boundary_point(m, s, rn, recon_order, m.xg_bedges + 6 * (long)b + 2 * k, q);
      double rr = q[0], u = q[1] / rr, v = q[2] / rr, e = q[3];
      double P = (a.gamma - 1.) * (e - 0.5 * rr * (u * u + v * v));
      t1 += (w[k] * (P * ny * a.cos_a - P * nx * a.sin_a));
      t2 += (w[k] * (P * nx * a.cos_a + P * ny * a.sin_a));
    }
  }
  out[0] = t1 * len * 0.5;
  out[1] = t2 * len * 0.5;
  out[2] = 1.;
}

__global__ void k_body_forces_sum(DevMesh m, DevState s) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double f0 = 0., f1 = 0.;
  for (int b = 1; b <= m.nbe; b++) {
    const double* o = s.bforce + 4 * (long)b;
    if (o[2] != 0.) {
      f0 += o[0];
      f1 += o[1];
    }
  }
  s.scalars[4] = f0;
  s.scalars[5] = f1;
}

}  // namespace flow
