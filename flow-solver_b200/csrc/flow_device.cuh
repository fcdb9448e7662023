// flow_device.cuh - per-face / per-node device math of the nonlinear iteration.
//
// Every expression keeps the operand order of the reference line it cites and
// the translation unit is compiled with --fmad=false, so each function returns
// the same bits as the reference's host code (IEEE double +,-,*,/ and sqrt are
// correctly rounded on both sides).
#pragma once
#include <cuda_runtime.h>

namespace flow {

// flux.C:37-68 Incompressible_Euler_Flux (the physical Euler flux).
__device__ __forceinline__ void euler_flux(const double* Q, double* F, double nx, double ny,
                                           double len, double gamma) {
  double rho = Q[0];
  double u = Q[1] / Q[0];
  double v = Q[2] / Q[0];
  double E = Q[3];
  double P = (gamma - 1.0) * (E - 0.5 * rho * (u * u + v * v));
  double theta = u * nx + v * ny;
  F[0] = rho * theta * len;
  F[1] = rho * u * theta * len + P * nx * len;
  F[2] = rho * v * theta * len + P * ny * len;
  F[3] = theta * (E + P) * len;
}

// Roe-averaged dissipation matrix |A| = T |Lambda| T^-1, row-major
// (flux.C:355-524; the same block is repeated in jacobian.C:764-866).
__device__ __forceinline__ void roe_matrix(double nx, double ny, double gamma, const double* ql,
                                           const double* qr, double* Rm) {
  double rhoL = ql[0], uL = ql[1] / ql[0], vL = ql[2] / ql[0], EL = ql[3];
  double pL = (gamma - 1.) * (EL - 0.5 * rhoL * (uL * uL + vL * vL));
  double HL = EL + pL, hL = HL / rhoL;
  double rhoR = qr[0], uR = qr[1] / qr[0], vR = qr[2] / qr[0], ER = qr[3];
  double pR = (gamma - 1.) * (ER - 0.5 * rhoR * (uR * uR + vR * vR));
  double HR = ER + pR, hR = HR / rhoR;
  double rhobar = sqrt(rhoL * rhoR);
  double bg = rhobar / (rhoL + rhobar);
  double ubar = uL + bg * (uR - uL);
  double vbar = vL + bg * (vR - vL);
  double hbar = hL + bg * (hR - hL);
  double thetabar = ubar * nx + vbar * ny;
  double V2bar = (ubar * ubar + vbar * vbar);
  double cbar = sqrt((gamma - 1.0) * (hbar - 0.5 * V2bar));
  double lam[4], T[16], Ti[16];
  lam[0] = fabs(thetabar);
  lam[1] = fabs(thetabar);
  lam[2] = fabs(thetabar + cbar);
  lam[3] = fabs(thetabar - cbar);
  double c2 = cbar * cbar;
  T[0] = 1.0;
  T[1] = 0.0;
  T[2] = 1.0 / c2;
  T[3] = 1.0 / c2;
  T[4] = ubar;
  T[5] = -ny;
  T[6] = ubar / c2 + nx / cbar;
  T[7] = ubar / c2 - nx / cbar;
  T[8] = vbar;
  T[9] = nx;
  T[10] = vbar / c2 + ny / cbar;
  T[11] = vbar / c2 - ny / cbar;
  T[12] = 0.5 * V2bar;
  T[13] = ubar * (-ny) + vbar * nx;
  double ogm1 = 1.0 / (gamma - 1.0), tc = thetabar / cbar, hv = (0.5 * V2bar) / c2;
  T[14] = ogm1 + tc + hv;
  T[15] = ogm1 - tc + hv;
  Ti[0] = 1.0 - (gamma - 1.0) * (0.5 * V2bar) / c2;
  Ti[1] = (gamma - 1.0) * ubar / c2;
  Ti[2] = (gamma - 1.0) * vbar / c2;
  Ti[3] = -1.0 * (gamma - 1.0) / c2;
  Ti[4] = -1.0 * (ubar * (-ny) + vbar * nx);
  Ti[5] = -ny;
  Ti[6] = nx;
  Ti[7] = 0.;
  Ti[8] = 0.5 * (-cbar * thetabar + (gamma - 1.0) * 0.5 * V2bar);
  Ti[9] = 0.5 * (cbar * nx - (gamma - 1.0) * ubar);
  Ti[10] = 0.5 * (cbar * ny - (gamma - 1.0) * vbar);
  Ti[11] = 0.5 * (gamma - 1.0);
  Ti[12] = 0.5 * (cbar * thetabar + (gamma - 1.0) * 0.5 * V2bar);
  Ti[13] = -0.5 * (cbar * nx + (gamma - 1.0) * ubar);
  Ti[14] = -0.5 * (cbar * ny + (gamma - 1.0) * vbar);
  Ti[15] = 0.5 * (gamma - 1.0);
  // linear_algebra.C:657-736: MMMult_DtG (Lambda * Tinv) then MMMult_GtG.
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) {
      double s = 0.;
#pragma unroll
      for (int k = 0; k < 4; k++) s += T[i * 4 + k] * (lam[k] * Ti[k * 4 + j]);
      Rm[i * 4 + j] = s;
    }
}

// flux.C:299-541 Roe_flux_centered.
__device__ __forceinline__ void roe_flux(double nx, double ny, double len, double gamma,
                                         const double* ql, const double* qr, double* flux) {
  double Rm[16], FL[4], FR[4];
  roe_matrix(nx, ny, gamma, ql, qr, Rm);
  double dq[4];
#pragma unroll
  for (int i = 0; i < 4; i++) dq[i] = qr[i] - ql[i];
  double diss[4];
#pragma unroll
  for (int i = 0; i < 4; i++) {
    double s = 0.;
#pragma unroll
    for (int j = 0; j < 4; j++) s += Rm[i * 4 + j] * dq[j];
    diss[i] = s * len;
  }
  euler_flux(ql, FL, nx, ny, len, gamma);
  euler_flux(qr, FR, nx, ny, len, gamma);
#pragma unroll
  for (int i = 0; i < 4; i++) flux[i] = 0.5 * (FL[i] + FR[i] - diss[i]);
}

// roe_flux split for the forward-difference Jacobian: the quantities of one
// face state (primitive variables, h = (E+p)/rho, its physical flux) and of
// the Roe average's density weight are formed once and reused by the
// evaluations that do not perturb them.  Each piece is the same expression
// on the same operands as in euler_flux / roe_matrix / roe_flux, so
// roe_core(...) returns the bits roe_flux(...) returns.
struct RoeSide {
  double rho, u, v, E, p, h;
  double F[4];
};

__device__ __forceinline__ void roe_side(const double* q, double nx, double ny, double len,
                                         double gamma, RoeSide& S) {
  S.rho = q[0];
  S.u = q[1] / q[0];
  S.v = q[2] / q[0];
  S.E = q[3];
  S.p = (gamma - 1.0) * (S.E - 0.5 * S.rho * (S.u * S.u + S.v * S.v));
  const double H = S.E + S.p;
  S.h = H / S.rho;
  const double theta = S.u * nx + S.v * ny;
  S.F[0] = S.rho * theta * len;
  S.F[1] = S.rho * S.u * theta * len + S.p * nx * len;
  S.F[2] = S.rho * S.v * theta * len + S.p * ny * len;
  S.F[3] = theta * (S.E + S.p) * len;
}

// bg = rhobar / (rhoL + rhobar), rhobar = sqrt(rhoL * rhoR)  (flux.C:371-372)
__device__ __forceinline__ double roe_weight(double rhoL, double rhoR) {
  const double rhobar = sqrt(rhoL * rhoR);
  return rhobar / (rhoL + rhobar);
}

// ogm1 = 1 / (gamma - 1), a per-run constant of the eigenvector matrix.
// Rm (may be null): the dissipation matrix |A~| = T |Lambda| T^-1 the flux
// formed on the way, row-major, the bits roe_matrix gives for ql, qr.
__device__ __forceinline__ void roe_core(double nx, double ny, double len, double gamma,
                                         double ogm1, const double* ql, const double* qr,
                                         const RoeSide& L, const RoeSide& R, double bg,
                                         double* flux, double* Rm = nullptr) {
  const double ubar = L.u + bg * (R.u - L.u);
  const double vbar = L.v + bg * (R.v - L.v);
  const double hbar = L.h + bg * (R.h - L.h);
  const double thetabar = ubar * nx + vbar * ny;
  const double V2bar = (ubar * ubar + vbar * vbar);
  const double cbar = sqrt((gamma - 1.0) * (hbar - 0.5 * V2bar));
  double lam[4], T[16], Ti[16];
  lam[0] = fabs(thetabar);
  lam[1] = fabs(thetabar);
  lam[2] = fabs(thetabar + cbar);
  lam[3] = fabs(thetabar - cbar);
  const double c2 = cbar * cbar;
  T[0] = 1.0;
  T[1] = 0.0;
  T[2] = 1.0 / c2;
  T[3] = 1.0 / c2;
  T[4] = ubar;
  T[5] = -ny;
  T[6] = ubar / c2 + nx / cbar;
  T[7] = ubar / c2 - nx / cbar;
  T[8] = vbar;
  T[9] = nx;
  T[10] = vbar / c2 + ny / cbar;
  T[11] = vbar / c2 - ny / cbar;
  T[12] = 0.5 * V2bar;
  T[13] = ubar * (-ny) + vbar * nx;
  const double tc = thetabar / cbar, hv = (0.5 * V2bar) / c2;
  T[14] = ogm1 + tc + hv;
  T[15] = ogm1 - tc + hv;
  Ti[0] = 1.0 - (gamma - 1.0) * (0.5 * V2bar) / c2;
  Ti[1] = (gamma - 1.0) * ubar / c2;
  Ti[2] = (gamma - 1.0) * vbar / c2;
  Ti[3] = -1.0 * (gamma - 1.0) / c2;
  Ti[4] = -1.0 * (ubar * (-ny) + vbar * nx);
  Ti[5] = -ny;
  Ti[6] = nx;
  Ti[7] = 0.;
  Ti[8] = 0.5 * (-cbar * thetabar + (gamma - 1.0) * 0.5 * V2bar);
  Ti[9] = 0.5 * (cbar * nx - (gamma - 1.0) * ubar);
  Ti[10] = 0.5 * (cbar * ny - (gamma - 1.0) * vbar);
  Ti[11] = 0.5 * (gamma - 1.0);
  Ti[12] = 0.5 * (cbar * thetabar + (gamma - 1.0) * 0.5 * V2bar);
  Ti[13] = -0.5 * (cbar * nx + (gamma - 1.0) * ubar);
  Ti[14] = -0.5 * (cbar * ny + (gamma - 1.0) * vbar);
  Ti[15] = 0.5 * (gamma - 1.0);
  double dq[4];
#pragma unroll
  for (int i = 0; i < 4; i++) dq[i] = qr[i] - ql[i];
#pragma unroll
  for (int i = 0; i < 4; i++) {
    double sd = 0.;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      double rm = 0.;
#pragma unroll
      for (int k = 0; k < 4; k++) rm += T[i * 4 + k] * (lam[k] * Ti[k * 4 + j]);
      if (Rm) Rm[i * 4 + j] = rm;
      sd += rm * dq[j];
    }
    const double diss = sd * len;
    flux[i] = 0.5 * (L.F[i] + R.F[i] - diss);
  }
}

// jacobian.C:764-866: the physical flux's Jacobian A(q) = dF/dq of one
// state for a unit normal (no length), row-major (row = flux component).
__device__ __forceinline__ void euler_jacobian(const double* q, double nx, double ny,
                                               double gamma, double* d) {
  const double rhoL = q[0], uL = q[1] / q[0], vL = q[2] / q[0], EL = q[3];
  const double th = uL * nx + vL * ny;
  const double ph = 0.5 * (gamma - 1.) * (uL * uL + vL * vL);
  d[0] = 0.;
  d[1] = nx;
  d[2] = ny;
  d[3] = 0.;
  d[4] = ph * nx - uL * th;
  d[5] = (2. - gamma) * uL * nx + th;
  d[6] = uL * ny - (gamma - 1.) * vL * nx;
  d[7] = (gamma - 1.) * nx;
  d[8] = ph * ny - vL * th;
  d[9] = vL * nx - (gamma - 1.) * uL * ny;
  d[10] = th + (2. - gamma) * vL * ny;
  d[11] = (gamma - 1.) * ny;
  const double ger = gamma * EL / rhoL;
  d[12] = (2. * ph - ger) * th;
  d[13] = (1. - gamma) * uL * th + nx * (ger - ph);
  d[14] = (1. - gamma) * vL * th + ny * (ger - ph);
  d[15] = gamma * th;
}

// euler_jacobian one row at a time: the state's scalars once, then row r's
// four entries by the same expressions (the same bits as d[4r .. 4r+3]).
struct EulerJacSide {
  double u, v, th, ph, ger;
};
__device__ __forceinline__ EulerJacSide euler_jacobian_side(const double* q, double nx,
                                                            double ny, double gamma) {
  EulerJacSide S;
  const double rho = q[0];
  S.u = q[1] / q[0];
  S.v = q[2] / q[0];
  S.th = S.u * nx + S.v * ny;
  S.ph = 0.5 * (gamma - 1.) * (S.u * S.u + S.v * S.v);
  S.ger = gamma * q[3] / rho;
  return S;
}
__device__ __forceinline__ void euler_jacobian_row(const EulerJacSide& S, double nx, double ny,
                                                   double gamma, int r, double* d) {
  if (r == 0) {
    d[0] = 0.; d[1] = nx; d[2] = ny; d[3] = 0.;
  } else if (r == 1) {
    d[0] = S.ph * nx - S.u * S.th;
    d[1] = (2. - gamma) * S.u * nx + S.th;
    d[2] = S.u * ny - (gamma - 1.) * S.v * nx;
    d[3] = (gamma - 1.) * nx;
  } else if (r == 2) {
    d[0] = S.ph * ny - S.v * S.th;
    d[1] = S.v * nx - (gamma - 1.) * S.u * ny;
    d[2] = S.th + (2. - gamma) * S.v * ny;
    d[3] = (gamma - 1.) * ny;
  } else {
    d[0] = (2. * S.ph - S.ger) * S.th;
    d[1] = (1. - gamma) * S.u * S.th + nx * (S.ger - S.ph);
    d[2] = (1. - gamma) * S.v * S.th + ny * (S.ger - S.ph);
    d[3] = gamma * S.th;
  }
}

// cv_calc.C:840-866: max(|theta+c|, |theta-c|) for one node state.
__device__ __forceinline__ double max_wave(const double* q, double nx, double ny, double gamma) {
  double rho = q[0];
  double u = q[1] / rho;
  double v = q[2] / rho;
  double P = (gamma - 1.0) * (q[3] - 0.5 * rho * (u * u + v * v));
  double c = sqrt((gamma * P) / rho);
  double theta = u * nx + v * ny;
  double tpc = fabs(theta + c), tmc = fabs(theta - c);
  return tpc >= tmc ? tpc : tmc;
}

// limiter.C:672-700: one reconstructed value's Venkatakrishnan bound
// (phi(y) = (y^2+2y)/(y^2+y+2), no epsilon), folded into phi with MIN().
// Written without branches: the reference's two branches differ only in the
// numerator (qmax - q0 above, qmin - q0 below), so the numerator is selected
// and the quotients formed for every point; where the difference is zero or
// NaN (the reference's third branch) the quotients are discarded and the
// fold takes MIN(phi, 1).  The same expressions on the same operands give the
// same bits, and the divisions of a lane's face points no longer wait on one
// another's branches.
__device__ __forceinline__ double venkat_fold(double ph, double qrec, double q0, double qmin,
                                              double qmax) {
  const double d = qrec - q0;
  const bool up = d > 0., down = d < 0.;
  double t = (up ? qmax - q0 : qmin - q0) / (qrec - q0);
  t = (t * t + 2. * t) / (t * t + t + 2.);
  const double b = (up || down) ? t : 1.0;
  return ph <= b ? ph : b;
}

// venkat_fold without a division of a zero or by a zero: a point the fold
// discards (qrec == q0, or a NaN difference) and a point whose bound is the
// node's own value (qmax == q0 going up, qmin == q0 going down: a zero
// dividend) divide 1 by 1 instead.  The first folds in 1 as before; the
// second folds in +0, the bits the reference's quotients give there
// (0/d = +-0, then (+0 + +-0) / (+0 +- 0 + 2) = +0).  Every other point
// divides the same operands, so phi has the same bits.  Where the state is
// uniform (the free stream of the first steps) most points are of the two
// kinds, and a division of or by zero leaves the fast path of the division.
__device__ __forceinline__ double venkat_fold_nz(double ph, double qrec, double q0, double qmin,
                                                 double qmax) {
  const double d = qrec - q0;
  const bool up = d > 0., down = d < 0.;
  const bool used = up || down;
  const double num = up ? qmax - q0 : qmin - q0;
  const bool flat = num == 0.;
  const bool div = used && !flat;
  double t = (div ? num : 1.0) / (div ? d : 1.0);
  t = (t * t + 2. * t) / (t * t + t + 2.);
  const double b = used ? (flat ? 0.0 : t) : 1.0;
  return ph <= b ? ph : b;
}

// The limiter fold of a node kernel: 0 venkat_fold, 1 or 2 venkat_fold_nz.
template <int LIM>
__device__ __forceinline__ double venkat_fold_lim(double ph, double qrec, double q0, double qmin,
                                                  double qmax) {
  if (LIM >= 1) return venkat_fold_nz(ph, qrec, q0, qmin, qmax);
  return venkat_fold(ph, qrec, q0, qmin, qmax);
}

// linear_algebra.C:571-596 lu() on a 4x4 row-major block, in place.
__device__ __forceinline__ void lu4(double* A) {
#pragma unroll
  for (int k = 0; k < 4; k++) {
#pragma unroll
    for (int i = k + 1; i < 4; i++) A[i * 4 + k] = A[i * 4 + k] / A[k * 4 + k];
#pragma unroll
    for (int j = k + 1; j < 4; j++)
#pragma unroll
      for (int i = k + 1; i < 4; i++) A[i * 4 + j] = A[i * 4 + j] - A[i * 4 + k] * A[k * 4 + j];
  }
}

// linear_algebra.C:611-638 forwardstab() then backstab().
__device__ __forceinline__ void lu_solve4(const double* M, const double* b, double* x) {
  double y0 = b[0];
  double y1 = b[1] - M[4] * y0;
  double y2 = b[2] - M[8] * y0 - M[9] * y1;
  double y3 = b[3] - M[12] * y0 - M[13] * y1 - M[14] * y2;
  x[3] = y3 / M[15];
  x[2] = (y2 - M[11] * x[3]) / M[10];
  x[1] = (y1 - M[6] * x[2] - M[7] * x[3]) / M[5];
  x[0] = (y0 - M[1] * x[1] - M[2] * x[2] - M[3] * x[3]) / M[0];
}

// A[r,:] . d in the reference's grouping (linear_algebra.C:200-221).
__device__ __forceinline__ double row_dot(const double* A, int r, const double* d) {
  return (A[r * 4] * d[0] + A[r * 4 + 1] * d[1] + A[r * 4 + 2] * d[2] + A[r * 4 + 3] * d[3]);
}

}  // namespace flow
