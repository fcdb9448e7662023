/*
 * flow_oracle.c - CPU restatement of the reference's nonlinear iteration.
 *
 * TEST INFRASTRUCTURE: the checker for the CUDA path, never part of it.
 * Every expression keeps the operand order of the reference line it cites,
 * because the parity bar is bit-for-bit equality with the compiled reference
 * (built by oracle/build_ref.sh).  Compile without FMA contraction
 * (-ffp-contract=off), as the reference's -ansi build is.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "flow_oracle.h"

#define NV 4
#define MINV(a, b) ((a) <= (b) ? (a) : (b))
#define MAXV(a, b) ((a) >= (b) ? (a) : (b))

/* ------------------------------------------------------------------ */
/* flux.C:37-68 Incompressible_Euler_Flux (the physical Euler flux)     */
/* ------------------------------------------------------------------ */
static void euler_flux(const double *Q, double *F, double nx, double ny, double len,
                       double gamma)
{
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

/* Roe average and |A| = T |Lambda| T^-1 (flux.C:355-524; the same block is
 * repeated in jacobian.C:764-866).  Writes the 4x4 row-major Roe matrix. */
static void roe_matrix(double nx, double ny, double gamma, const double *ql,
                       const double *qr, double *Roemat)
{
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
  double lam[4], T[16], Ti[16], tmp[16];
  lam[0] = fabs(thetabar);
  lam[1] = fabs(thetabar);
  lam[2] = fabs(thetabar + cbar);
  lam[3] = fabs(thetabar - cbar);
  T[0] = 1.0;
  T[1] = 0.0;
  T[2] = 1.0 / (cbar * cbar);
  T[3] = 1.0 / (cbar * cbar);
  T[4] = ubar;
  T[5] = -ny;
  T[6] = ubar / (cbar * cbar) + nx / cbar;
  T[7] = ubar / (cbar * cbar) - nx / cbar;
  T[8] = vbar;
  T[9] = nx;
  T[10] = vbar / (cbar * cbar) + ny / cbar;
  T[11] = vbar / (cbar * cbar) - ny / cbar;
  T[12] = 0.5 * V2bar;
  T[13] = ubar * (-ny) + vbar * nx;
  T[14] = 1.0 / (gamma - 1.0) + thetabar / cbar + (0.5 * V2bar) / (cbar * cbar);
  T[15] = 1.0 / (gamma - 1.0) - thetabar / cbar + (0.5 * V2bar) / (cbar * cbar);
  Ti[0] = 1.0 - (gamma - 1.0) * (0.5 * V2bar) / (cbar * cbar);
  Ti[1] = (gamma - 1.0) * ubar / (cbar * cbar);
  Ti[2] = (gamma - 1.0) * vbar / (cbar * cbar);
  Ti[3] = -1.0 * (gamma - 1.0) / (cbar * cbar);
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
  /* linear_algebra.C:657-736 MMMult_DtG then MMMult_GtG */
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) tmp[i * 4 + j] = lam[i] * Ti[i * 4 + j];
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) {
      double s = 0.;
      for (int k = 0; k < 4; k++) s += T[i * 4 + k] * tmp[k * 4 + j];
      Roemat[i * 4 + j] = s;
    }
}

/* flux.C:299-541 Roe_flux_centered */
int orc_roe_flux(double nx, double ny, double len, double gamma, const double *ql,
                 const double *qr, double *flux)
{
  double Rm[16], dq[4], diss[4], FL[4], FR[4];
  roe_matrix(nx, ny, gamma, ql, qr, Rm);
  for (int i = 0; i < 4; i++) dq[i] = qr[i] - ql[i];
  for (int i = 0; i < 4; i++) {
    double s = 0.;
    for (int j = 0; j < 4; j++) s += Rm[i * 4 + j] * dq[j];
    diss[i] = s;
  }
  for (int i = 0; i < 4; i++) diss[i] = diss[i] * len;
  euler_flux(ql, FL, nx, ny, len, gamma);
  euler_flux(qr, FR, nx, ny, len, gamma);
  for (int i = 0; i < 4; i++) flux[i] = 0.5 * (FL[i] + FR[i] - diss[i]);
  return 1;
}

/* ------------------------------------------------------------------ */
/* cv_calc.C:790-965 + init_memory.C:159-310                           */
/* ------------------------------------------------------------------ */
static double max_wave(const double *q, double nx, double ny, double gamma)
{
  double rho = q[0];
  double u = q[1] / rho;
  double v = q[2] / rho;
  double P = (gamma - 1.0) * (q[3] - 0.5 * rho * (u * u + v * v));
  double c = sqrt((gamma * P) / rho);
  double theta = u * nx + v * ny;
  double tpc = fabs(theta + c), tmc = fabs(theta - c);
  return MAXV(tpc, tmc);
}

int orc_build_matrix(orc_grid *g, const orc_params *p)
{
  int nn = g->nn;
  long mdim = (long)g->ia[nn + 1] * 16;
  for (long i = 0; i < mdim; i++) g->LHS[i] = 0.;
  for (int n = 1; n <= nn; n++) g->ev_con[n] = 0.;
  for (int s = 1; s <= g->nsubedges; s++) {
    int e = g->subedges[s * 2];
    double nx = g->xn_subedges[s * 3], ny = g->xn_subedges[s * 3 + 1],
           len = g->xn_subedges[s * 3 + 2];
    int L = g->edges[e * 2], R = g->edges[e * 2 + 1];
    double m = max_wave(&g->nQ[L * NV], nx, ny, p->gamma);
    if (!isfinite(m)) return 1;
    g->ev_con[L] += (m * len);
    m = max_wave(&g->nQ[R * NV], nx, ny, p->gamma);
    if (!isfinite(m)) return 1;
    g->ev_con[R] += (m * len);
  }
  for (int b = 1; b <= g->nbedges; b++) {
    int L = g->bedges[b * 5];
    double m = max_wave(&g->nQ[L * NV], g->xn_bedges[b * 3], g->xn_bedges[b * 3 + 1], p->gamma);
    if (!isfinite(m)) return 1;
    g->ev_con[L] += (m * g->xn_bedges[b * 3 + 2]);
  }
  double cfl;
  if (p->method == 1) {
    if (g->citer < p->ramp)
      cfl = 1. + (1. * (g->citer - 1)) / (1. * p->ramp) * (p->CFL - 1.);
    else
      cfl = p->CFL;
  } else if (p->method == 0) {
    cfl = 1.0;
  } else {
    cfl = p->CFL;
  }
  g->cfl = cfl;
  for (int j = 1; j <= nn; j++) {
    int i = g->iau[j];
    double V = g->cv_area[j];
    g->dt[j] = cfl * (V / g->ev_con[j]);
    if (g->dt[j] <= 0.) return 2;
    if (!isfinite(g->dt[j])) return 3;
    for (int k = 0; k < NV; k++) {
      double d;
      if (p->tacc == 2 && g->citer > 1) /* rfiter = 0: no restart */
        d = 1.5 * V / p->mintime;
      else if (p->unsteady > 0)
        d = V / p->mintime;
      else
        d = V / (g->dt[j]);
      g->LHS[(long)i * 16 + k * NV + k] = d;
    }
  }
  return 0;
}

/* ------------------------------------------------------------------ */
/* gradient.C:370-403 (edge-based LSQ gradient, weights precomputed)    */
/* ------------------------------------------------------------------ */
void orc_gradient_lsq(orc_grid *g)
{
  for (int n = 1; n <= g->nn; n++)
    for (int k = 0; k < 8; k++) g->grad[n * 8 + k] = 0.;
  for (int j = 0; j < NV; j++)
    for (int i = 1; i <= g->nedges; i++) {
      int L = g->edges[2 * i], R = g->edges[2 * i + 1];
      const double *wl = &g->edge_weight[i * 4], *wr = &g->edge_weight[i * 4 + 2];
      double dq = g->nQ[R * NV + j] - g->nQ[L * NV + j];
      for (int k = 0; k < 2; k++) {
        g->grad[L * 8 + 2 * j + k] += wl[k] * dq;
        g->grad[R * 8 + 2 * j + k] -= wr[k] * dq;
      }
    }
}

/* ------------------------------------------------------------------ */
/* compute_derivatives.C:1438-1534 (order 3 apply of V S^-1 U^T)        */
/* ------------------------------------------------------------------ */
void orc_derivatives_k2(orc_grid *g)
{
  double b[64], t2[64], t1[64], sol[5];
  for (int i = 1; i <= g->nn; i++) {
    if (g->node_order[i] < 3) continue;
    int m = g->svd_m[i];
    const double *U = g->svd_U + g->svd_off[i];
    const double *VT = g->svd_VT + (long)i * 25;
    const double *S = g->svd_S + (long)i * 5;
    int s0 = g->gnnsn[g->gnnsn1[i] + 1], s1 = g->gnnsn[g->gnnsn1[i + 1]];
    for (int var = 0; var < NV; var++) {
      for (int j = s0; j < s1; j++) {
        int node = g->gnsn[j];
        double dx0 = g->x[node * 2] - g->x[i * 2];
        double dx1 = g->x[node * 2 + 1] - g->x[i * 2 + 1];
        double dist = sqrt(dx0 * dx0 + dx1 * dx1);
        double w = 1.0 / pow(dist, 1.0);
        b[j - s0] = w * (g->nQ[node * NV + var] - g->nQ[i * NV + var]);
      }
      /* linear_algebra.C dotProductGeneral: sequential sum from 0.  The
       * reference forms all m entries of U^T b but reads only the first 5
       * (compute_derivatives.C:1479-1491). */
      for (int j = 0; j < 5; j++) {
        double s = 0.;
        for (int k = 0; k < m; k++) s += b[k] * U[j * m + k];
        t2[j] = s;
      }
      for (int j = 0; j < 5; j++) t1[j] = t2[j] / S[j];
      for (int j = 0; j < 5; j++) {
        double s = 0.;
        for (int k = 0; k < 5; k++) s += VT[j * 5 + k] * t1[k];
        sol[j] = s;
      }
      for (int k = 0; k < 5; k++) g->hess[i * 36 + var * 9 + k] = sol[k];
      const double *mo = &g->moments[i * 9];
      g->point_value[i * NV + var] = g->nQ[i * NV + var] - mo[0] * sol[0] - mo[1] * sol[1] -
                                     mo[2] * sol[2] * 0.5 - mo[3] * sol[3] * 0.5 -
                                     mo[4] * sol[4];
    }
  }
}

/* ------------------------------------------------------------------ */
/* reconstruction (reconstruct.C)                                       */
/* ------------------------------------------------------------------ */
static int recon_order(const orc_grid *g, const orc_params *p, int node, int ts)
{
  /* reconstruct.C:72-167 for orders 1 and 3 */
  if (p->order == 1) return ts <= p->foits ? 0 : 1;
  if (p->order == 3) {
    if (ts <= p->foits) return 0;
    if (ts <= p->foits + p->soits) return 1;
    return g->node_order[node];
  }
  return 0;
}

/* linear: q + phi*g.dx (reconstruct.C:181-203) */
static void recon_linear(const orc_grid *g, int n, double phi, const double *dx, double *q)
{
  for (int j = 0; j < NV; j++)
    q[j] += (phi * g->grad[n * 8 + j * 2] * dx[0] + phi * g->grad[n * 8 + j * 2 + 1] * dx[1]);
}

/* quadratic from the point value (reconstruct.C:226-257) */
static void recon_quad(const orc_grid *g, int n, double phi, double sigma, const double *dx,
                       double *q)
{
  for (int j = 0; j < NV; j++) q[j] = g->point_value[n * NV + j];
  for (int j = 0; j < NV; j++) {
    const double *h = &g->hess[n * 36 + j * 9];
    q[j] += (phi * h[0] * dx[0] + phi * h[1] * dx[1] + sigma * h[2] * dx[0] * dx[0] * 0.5 +
             sigma * h[3] * dx[1] * dx[1] * 0.5 + sigma * h[4] * dx[0] * dx[1]);
  }
}

/* Reconstruct (reconstruct.C:38-446) to the subedge's face point */
static void reconstruct_face(const orc_grid *g, const orc_params *p, int s, int L, int R,
                             int ts, double *qL, double *qR, int limited)
{
  for (int j = 0; j < NV; j++) { qL[j] = g->nQ[L * NV + j]; qR[j] = g->nQ[R * NV + j]; }
  double phiL = limited ? g->phi[L * 8] : 1.0, phiR = limited ? g->phi[R * 8] : 1.0;
  double sigL = limited ? g->phi[L * 8 + 1] : 1.0, sigR = limited ? g->phi[R * 8 + 1] : 1.0;
  int ro[2] = {recon_order(g, p, L, ts), recon_order(g, p, R, ts)};
  int gel = g->subedges[s * 2 + 1];
  double fc[2], dx[2];
  fc[0] = (g->el_cent[gel * 2] + g->xm_subedges[s * 2]) * 0.5;
  fc[1] = (g->el_cent[gel * 2 + 1] + g->xm_subedges[s * 2 + 1]) * 0.5;
  for (int side = 0; side < 2; side++) {
    int n = side ? R : L;
    double *q = side ? qR : qL;
    double phi = side ? phiR : phiL, sig = side ? sigR : sigL;
    if (ro[side] == 0) continue;
    dx[0] = fc[0] - g->x[n * 2];
    dx[1] = fc[1] - g->x[n * 2 + 1];
    if (ro[side] == 1) {
      if (limited)
        recon_linear(g, n, phi, dx, q);
      else
        for (int j = 0; j < NV; j++)
          q[j] += (g->grad[n * 8 + j * 2] * dx[0] + g->grad[n * 8 + j * 2 + 1] * dx[1]);
    } else {
      recon_quad(g, n, phi, sig, dx, q);
    }
  }
}

/* Reconstruct_Gauss_UL (reconstruct.C:1420-) to a Gauss point, unlimited */
static void reconstruct_gauss_ul(const orc_grid *g, const orc_params *p, int L, int R,
                                 const double *gp, double *qL, double *qR)
{
  for (int j = 0; j < NV; j++) { qL[j] = g->nQ[L * NV + j]; qR[j] = g->nQ[R * NV + j]; }
  int ro[2] = {recon_order(g, p, L, g->citer), recon_order(g, p, R, g->citer)};
  double dx[2];
  for (int side = 0; side < 2; side++) {
    int n = side ? R : L;
    double *q = side ? qR : qL;
    if (ro[side] == 0) continue;
    dx[0] = gp[0] - g->x[n * 2];
    dx[1] = gp[1] - g->x[n * 2 + 1];
    if (ro[side] == 1) {
      for (int j = 0; j < NV; j++)
        q[j] += (g->grad[n * 8 + j * 2] * dx[0] + g->grad[n * 8 + j * 2 + 1] * dx[1]);
    } else {
      for (int j = 0; j < NV; j++) q[j] = g->point_value[n * NV + j];
      for (int j = 0; j < NV; j++) {
        const double *h = &g->hess[n * 36 + j * 9];
        q[j] += (h[0] * dx[0] + h[1] * dx[1] + h[2] * dx[0] * dx[0] * 0.5 +
                 h[3] * dx[1] * dx[1] * 0.5 + h[4] * dx[0] * dx[1]);
      }
    }
  }
}

/* Reconstruct_Gauss_Boundary (reconstruct.C:1708-1890), limited */
static void reconstruct_gauss_boundary(const orc_grid *g, const orc_params *p, int n,
                                       const double *gp, double *q)
{
  for (int j = 0; j < NV; j++) q[j] = g->nQ[n * NV + j];
  int ro = recon_order(g, p, n, g->citer);
  double phi = g->phi[n * 8], sig = g->phi[n * 8 + 1], dx[2];
  if (ro == 0) return;
  dx[0] = gp[0] - g->x[n * 2];
  dx[1] = gp[1] - g->x[n * 2 + 1];
  if (ro == 1)
    recon_linear(g, n, phi, dx, q);
  else
    recon_quad(g, n, phi, sig, dx, q);
}

/* ------------------------------------------------------------------ */
/* limiter.C:511-983 compute_limiter_venkatakrishnan                    */
/* ------------------------------------------------------------------ */
static void venkat_side(orc_grid *g, int n, const double *q, const double *qmin,
                        const double *qmax)
{
  for (int j = 0; j < NV; j++) {
    double d = q[j] - g->nQ[n * NV + j], t;
    double *ph = &g->phi[n * 8 + j * 2];
    if (d > 0.) {
      t = (qmax[n * NV + j] - g->nQ[n * NV + j]) / (q[j] - g->nQ[n * NV + j]);
      t = (t * t + 2. * t) / (t * t + t + 2.);
      *ph = MINV(*ph, t);
    } else if (d < 0.) {
      t = (qmin[n * NV + j] - g->nQ[n * NV + j]) / (q[j] - g->nQ[n * NV + j]);
      t = (t * t + 2. * t) / (t * t + t + 2.);
      *ph = MINV(*ph, t);
    } else {
      *ph = MINV(*ph, 1.0);
    }
  }
}

int orc_limiter_venkat(orc_grid *g, const orc_params *p)
{
  int nn = g->nn;
  double *qmin = (double *)malloc(sizeof(double) * (nn + 1) * NV);
  double *qmax = (double *)malloc(sizeof(double) * (nn + 1) * NV);
  for (int i = 1; i <= nn; i++) {
    for (int j = 0; j < 8; j++) g->phi[i * 8 + j] = 0.0;
    for (int j = 0; j < NV; j++) qmin[i * NV + j] = qmax[i * NV + j] = g->nQ[i * NV + j];
    for (int j = 0; j < NV; j++) g->phi[i * 8 + j * 2] = 1.0;
  }
  for (int i = 1; i <= g->nedges; i++) {
    int L = g->edges[i * 2], R = g->edges[i * 2 + 1];
    for (int j = 0; j < NV; j++) {
      qmin[L * NV + j] = MINV(qmin[L * NV + j], g->nQ[R * NV + j]);
      qmax[L * NV + j] = MAXV(qmax[L * NV + j], g->nQ[R * NV + j]);
      qmin[R * NV + j] = MINV(qmin[R * NV + j], g->nQ[L * NV + j]);
      qmax[R * NV + j] = MAXV(qmax[R * NV + j], g->nQ[L * NV + j]);
    }
  }
  int gauss = (p->order == 3 && g->citer > (p->foits + p->soits));
  double qL[4], qR[4];
  for (int s = 1; s <= g->nsubedges; s++) {
    int e = g->subedges[s * 2];
    int L = g->edges[e * 2], R = g->edges[e * 2 + 1];
    if (gauss) {
      for (int k = 0; k < 3; k++) {
        reconstruct_gauss_ul(g, p, L, R, &g->xg_subedges[s * 6 + 2 * k], qL, qR);
        venkat_side(g, L, qL, qmin, qmax);
        venkat_side(g, R, qR, qmin, qmax);
      }
    } else {
      reconstruct_face(g, p, s, L, R, g->citer, qL, qR, 0);
      venkat_side(g, L, qL, qmin, qmax);
      venkat_side(g, R, qR, qmin, qmax);
    }
  }
  int bad = 0;
  for (int i = 1; i <= nn; i++)
    for (int j = 0; j < NV; j++) g->phi[i * 8 + j * 2 + 1] = g->phi[i * 8 + j * 2];
  for (int i = 1; i <= nn; i++) {
    double t = g->phi[i * 8];
    for (int j = 1; j < NV; j++) t = MINV(t, g->phi[i * 8 + j * 2]);
    g->phi[i * 8] = t;
    g->phi[i * 8 + 1] = t;
  }
  for (int i = 1; i <= nn; i++)
    for (int j = 0; j < NV; j++)
      if (g->phi[i * 8 + j * 2] < 0.0 || g->phi[i * 8 + j * 2] > 1.0) bad = 1;
  free(qmin);
  free(qmax);
  return bad;
}

/* ------------------------------------------------------------------ */
/* residual.C:40-342 + jacobian.C:45-185                                */
/* ------------------------------------------------------------------ */
static void add_block(double *blk, double (*d)[4], double sgn)
{
  for (int i = 0; i < 4; i++)
    for (int k = 0; k < 4; k++) {
      if (sgn > 0) blk[i * 4 + k] += d[i][k];
      else blk[i * 4 + k] -= d[i][k];
    }
}

static void numerical_jacobian(orc_grid *g, const orc_params *p, int L, int R,
                               const double *QL, const double *QR, const double *flux,
                               double nx, double ny, double len)
{
  double Qp[4], fp[4], dL[4][4], dR[4][4];
  const double eps = 1.0e-08;
  for (int i = 0; i < NV; i++) {
    for (int j = 0; j < NV; j++) Qp[j] = QL[j];
    Qp[i] += eps;
    orc_roe_flux(nx, ny, len, p->gamma, Qp, QR, fp);
    for (int j = 0; j < NV; j++) dL[j][i] = (fp[j] - flux[j]) / eps;
  }
  for (int i = 0; i < NV; i++) {
    for (int j = 0; j < NV; j++) Qp[j] = QR[j];
    Qp[i] += eps;
    orc_roe_flux(nx, ny, len, p->gamma, QL, Qp, fp);
    for (int j = 0; j < NV; j++) dR[j][i] = (fp[j] - flux[j]) / eps;
  }
  add_block(&g->LHS[(long)g->iau[L] * 16], dL, 1.0);
  add_block(&g->LHS[(long)g->iau[R] * 16], dR, -1.0);
  for (int i = g->ia[L]; i < g->ia[L + 1]; i++)
    if (g->ja[i] == R) add_block(&g->LHS[(long)i * 16], dR, 1.0);
  for (int i = g->ia[R]; i < g->ia[R + 1]; i++)
    if (g->ja[i] == L) add_block(&g->LHS[(long)i * 16], dL, -1.0);
}

/* The flux Jacobian A(q) of one state for a unit normal (jacobian.C:764-866,
 * the terms boundary_jacobian uses), row-major. */
static void euler_jacobian(const double *Q, double nx, double ny, double gamma, double (*d)[4])
{
  double rhoL = Q[0], uL = Q[1] / Q[0], vL = Q[2] / Q[0], EL = Q[3];
  double theta = uL * nx + vL * ny;
  double phi = 0.5 * (gamma - 1.) * (uL * uL + vL * vL);
  d[0][0] = 0.;
  d[0][1] = nx;
  d[0][2] = ny;
  d[0][3] = 0.;
  d[1][0] = phi * nx - uL * theta;
  d[1][1] = (2. - gamma) * uL * nx + theta;
  d[1][2] = uL * ny - (gamma - 1.) * vL * nx;
  d[1][3] = (gamma - 1.) * nx;
  d[2][0] = phi * ny - vL * theta;
  d[2][1] = vL * nx - (gamma - 1.) * uL * ny;
  d[2][2] = theta + (2. - gamma) * vL * ny;
  d[2][3] = (gamma - 1.) * ny;
  d[3][0] = (2. * phi - gamma * EL / rhoL) * theta;
  d[3][1] = (1. - gamma) * uL * theta + nx * (gamma * EL / rhoL - phi);
  d[3][2] = (1. - gamma) * vL * theta + ny * (gamma * EL / rhoL - phi);
  d[3][3] = gamma * theta;
}

/* Precision form, jac_approx: dF/dqL = (A(qL) + |A~|) len/2 and
 * dF/dqR = (A(qR) - |A~|) len/2, |A~| the Roe dissipation matrix of the face
 * (no reference counterpart; the reference's boundary faces use this form,
 * jacobian.C:681-962), each entry rounded to FP32 (the blocks it feeds are
 * FP32) and accumulated in double like numerical_jacobian's blocks. */
static void approximate_jacobian(orc_grid *g, const orc_params *p, int L, int R,
                                 const double *QL, const double *QR, double nx, double ny,
                                 double len)
{
  double Rm[16], dL[4][4], dR[4][4];
  roe_matrix(nx, ny, p->gamma, QL, QR, Rm);
  euler_jacobian(QL, nx, ny, p->gamma, dL);
  euler_jacobian(QR, nx, ny, p->gamma, dR);
  for (int i = 0; i < 4; i++)
    for (int k = 0; k < 4; k++) {
      dL[i][k] = (double)(float)(0.5 * (dL[i][k] + Rm[i * 4 + k]) * len);
      dR[i][k] = (double)(float)(0.5 * (dR[i][k] - Rm[i * 4 + k]) * len);
    }
  add_block(&g->LHS[(long)g->iau[L] * 16], dL, 1.0);
  add_block(&g->LHS[(long)g->iau[R] * 16], dR, -1.0);
  for (int i = g->ia[L]; i < g->ia[L + 1]; i++)
    if (g->ja[i] == R) add_block(&g->LHS[(long)i * 16], dR, 1.0);
  for (int i = g->ia[R]; i < g->ia[R + 1]; i++)
    if (g->ja[i] == L) add_block(&g->LHS[(long)i * 16], dL, -1.0);
}

void orc_interior_residuals(orc_grid *g, const orc_params *p, int jupdate, int ts)
{
  int nn = g->nn;
  for (int i = 1; i <= nn; i++)
    for (int j = 0; j < NV; j++) { g->RHS[i * NV + j] = 0.; g->R[i * NV + j] = 0.; }
  int gauss = (p->order == 3 && ts > (p->foits + p->soits));
  double qL[4], qR[4], flux[4];
  for (int s = 1; s <= g->nsubedges; s++) {
    int e = g->subedges[s * 2];
    double nx = g->xn_subedges[s * 3], ny = g->xn_subedges[s * 3 + 1],
           len = g->xn_subedges[s * 3 + 2];
    int L = g->edges[e * 2], R = g->edges[e * 2 + 1];
    if (gauss) {
      /* residual.C:205-290: the three Gauss-point fluxes are computed and
       * then overwritten by the unreconstructed flux; only that survives. */
      for (int j = 0; j < NV; j++) { qL[j] = g->nQ[L * NV + j]; qR[j] = g->nQ[R * NV + j]; }
      orc_roe_flux(nx, ny, len, p->gamma, qL, qR, flux);
    } else {
      reconstruct_face(g, p, s, L, R, ts, qL, qR, 1);
      orc_roe_flux(nx, ny, len, p->gamma, qL, qR, flux);
    }
    if (jupdate && p->jac_approx) approximate_jacobian(g, p, L, R, qL, qR, nx, ny, len);
    else if (jupdate) numerical_jacobian(g, p, L, R, qL, qR, flux, nx, ny, len);
    for (int k = 0; k < NV; k++) {
      g->R[L * NV + k] += flux[k];
      g->R[R * NV + k] -= flux[k];
    }
  }
}

/* ------------------------------------------------------------------ */
/* cvbc.C:37-481 Set_Boundary_Values (conserved variables, no MMS)      */
/* ------------------------------------------------------------------ */
int orc_set_boundary_values(orc_grid *g, const orc_params *p)
{
  double gamma = p->gamma;
  double angle = p->alpha * M_PI / 180.;
  double rhoinf = 1.0, uinf = p->mach * cos(angle), vinf = p->mach * sin(angle);
  double pinf = 1. / gamma;
  for (int i = 1; i <= g->nbedges; i++) {
    int rn = g->bedges[i * 5], gn = g->bedges[i * 5 + 1] + g->nn;
    int bc = g->bbc[g->bedges[i * 5 + 3]];
    double nx = g->xn_bedges[i * 3], ny = g->xn_bedges[i * 3 + 1];
    const double *qi = &g->nQ[rn * NV];
    double *qb = &g->nQ[gn * NV];
    double rhoi = qi[0], ui = qi[1] / rhoi, vi = qi[2] / rhoi;
    double pi = (gamma - 1.) * (qi[3] - 0.5 * rhoi * (ui * ui + vi * vi));
    double ci = sqrt((gamma * pi) / rhoi);
    double rhob = qb[0], ub = qb[1] / rhob, vb = qb[2] / rhob;
    double pb = (gamma - 1.) * (qb[3] - 0.5 * rhob * (ub * ub + vb * vb));
    double cb = sqrt((gamma * pb) / rhob);
    double rho0 = 0.5 * (rhoi + rhob);
    double p0 = 0.5 * (pi + pb);
    double c0 = 0.5 * (ci + cb);
    (void)p0;
    double theta = ui * nx + vi * ny;
    double ev1 = theta, ev3 = theta + ci, ev4 = theta - ci;
    if (bc == 0 || (bc % 2 == 0)) {
      if (ev1 <= 0.0 && ev4 <= 0.0) {
        if (ev3 >= 0.0) {
          pb = 0.5 * (pinf + pi - rho0 * c0 * ((uinf - ui) * nx + (vinf - vi) * ny));
          rhob = rhoinf + (pb - pinf) / (c0 * c0);
          ub = uinf + (pb - pinf) / (rho0 * c0) * nx;
          vb = vinf + (pb - pinf) / (rho0 * c0) * ny;
        } else if (ev3 < 0.0) {
          rhob = rhoinf; ub = uinf; vb = vinf; pb = pinf;
        } else {
          return 1;
        }
      } else if (ev1 >= 0.0 && ev3 >= 0.0) {
        if (ev4 <= 0.0) {
          pb = pinf;
          rhob = rhoi + (pb - pi) / (c0 * c0);
          ub = ui - (pb - pi) / (rho0 * c0) * nx;
          vb = vi - (pb - pi) / (rho0 * c0) * ny;
        } else if (ev4 > 0.0) {
          rhob = rhoi; ub = ui; vb = vi; pb = pi;
        } else {
          return 1;
        }
      } else {
        return 1;
      }
    } else if (bc == 1 || (bc % 2 == 1)) {
      pb = pi + rho0 * c0 * theta;
      rhob = rhoi + (pb - pi) / (c0 * c0);
      ub = ui - (pb - pi) / (rho0 * c0) * nx;
      vb = vi - (pb - pi) / (rho0 * c0) * ny;
    } else {
      return 1;
    }
    qb[0] = rhob;
    qb[1] = rhob * ub;
    qb[2] = rhob * vb;
    qb[3] = pb / (gamma - 1.0) + 0.5 * rhob * (ub * ub + vb * vb);
    if (rhob < 0.0) {
      /* cvbc.C:447-470: reflect the interior state */
      rhob = rhoi;
      ub = (1. - 2. * nx * nx) * ui - 2. * nx * ny * vi;
      vb = (1. - 2. * ny * ny) * vi - 2. * nx * ny * ui;
      pb = pi;
      qb[0] = rhob;
      qb[1] = rhob * ub;
      qb[2] = rhob * vb;
      qb[3] = pb / (gamma - 1.0) + 0.5 * rhob * (ub * ub + vb * vb);
    }
  }
  return 0;
}

/* curved_boundaries.C:701-877 curved_boundary_normal_vector */
void orc_curved_normal(int bc, const double *x, double *nx, double *ny)
{
  double t;
  if (bc == 11 || bc == 12) {
    if (x[0] >= 0. && x[1] >= 0.) t = acos(x[0]);
    else if (x[0] >= 0. && x[1] < 0.) t = -acos(x[0]);
    else if (x[0] < 0. && x[1] >= 0.) t = acos(x[0]);
    else t = -acos(x[0]);
    if (bc == 11) { *nx = -cos(t); *ny = -sin(t); }
    else { *nx = cos(t); *ny = sin(t); }
    return;
  }
  if (bc == 13 || bc == 14) {
    t = atan2(x[1], x[0]);
    *nx = -cos(t); *ny = -sin(t);
    return;
  }
  if (bc == 15 || bc == 16 || bc == 21 || bc == 22) {
    t = atan2(x[1], x[0]);
    *nx = cos(t); *ny = sin(t);
    return;
  }
  if (bc == 17 || bc == 18 || bc == 19 || bc == 20) {
    int upper = (bc == 17 || bc == 18);
    if (fabs(x[0]) < 1.e-10) { *nx = 1.0; *ny = 0.0; return; }
    double y;
    if (upper)
      y = 0.08907 / sqrt(x[0]) - 0.07560 - 0.42192 * x[0] + 0.51174 * x[0] * x[0] -
          0.24864 * x[0] * x[0] * x[0];
    else
      y = -0.08907 / sqrt(x[0]) + 0.07560 + 0.42192 * x[0] - 0.51174 * x[0] * x[0] +
          0.24864 * x[0] * x[0] * x[0];
    double m = -1.0 / y;
    double len = sqrt(1.0 + m * m);
    *nx = 1.0 / len;
    *ny = m / len;
    if ((upper && *ny > 0.0) || (!upper && *ny < 0.0)) {
      *nx = -1.0 * (*nx);
      *ny = -1.0 * (*ny);
    }
  }
}

/* ------------------------------------------------------------------ */
/* residual.C:359-1230 + jacobian.C:681-962                             */
/* ------------------------------------------------------------------ */
static void boundary_jacobian(orc_grid *g, const orc_params *p, int ib, const double *QL,
                              const double *QR, double nx, double ny, double len)
{
  double gamma = p->gamma, Rm[16], d[4][4];
  roe_matrix(nx, ny, gamma, QL, QR, Rm);
  double rhoL = QL[0], uL = QL[1] / QL[0], vL = QL[2] / QL[0], EL = QL[3];
  double theta = uL * nx + vL * ny;
  double phi = 0.5 * (gamma - 1.) * (uL * uL + vL * vL);
  d[0][0] = 0.;
  d[0][1] = nx;
  d[0][2] = ny;
  d[0][3] = 0.;
  d[1][0] = phi * nx - uL * theta;
  d[1][1] = (2. - gamma) * uL * nx + theta;
  d[1][2] = uL * ny - (gamma - 1.) * vL * nx;
  d[1][3] = (gamma - 1.) * nx;
  d[2][0] = phi * ny - vL * theta;
  d[2][1] = vL * nx - (gamma - 1.) * uL * ny;
  d[2][2] = theta + (2. - gamma) * vL * ny;
  d[2][3] = (gamma - 1.) * ny;
  d[3][0] = (2. * phi - gamma * EL / rhoL) * theta;
  d[3][1] = (1. - gamma) * uL * theta + nx * (gamma * EL / rhoL - phi);
  d[3][2] = (1. - gamma) * vL * theta + ny * (gamma * EL / rhoL - phi);
  d[3][3] = gamma * theta;
  for (int i = 0; i < 4; i++)
    for (int k = 0; k < 4; k++) d[i][k] = 0.5 * (d[i][k] + Rm[i * 4 + k]) * len;
  int n = g->bedges[ib * 5];
  add_block(&g->LHS[(long)g->iau[n] * 16], d, 1.0);
}

int orc_boundary_residuals(orc_grid *g, const orc_params *p, int jupdate)
{
  int rc = orc_set_boundary_values(g, p);
  if (rc) return rc;
  int gauss = (p->order == 3 && g->citer > (p->foits + p->soits));
  double qL[4], qR[4], flux[4];
  for (int i = 1; i <= g->nbedges; i++) {
    int rn = g->bedges[i * 5], gn = g->bedges[i * 5 + 1] + g->nn;
    int bc = g->bbc[g->bedges[i * 5 + 3]];
    double nx = g->xn_bedges[i * 3], ny = g->xn_bedges[i * 3 + 1], len = g->xn_bedges[i * 3 + 2];
    if (gauss && bc > 10) {
      /* residual.C:1048-1143: Gauss-point fluxes are discarded; what
       * survives is the arc length and the node normal, which is also
       * written back into xn_bedges. */
      len = g->xgn_bedges[i * 9 + 2];
      orc_curved_normal(bc, &g->x[rn * 2], &nx, &ny);
      g->xn_bedges[i * 3] = nx;
      g->xn_bedges[i * 3 + 1] = ny;
    }
    for (int j = 0; j < NV; j++) { qL[j] = g->nQ[rn * NV + j]; qR[j] = g->nQ[gn * NV + j]; }
    orc_roe_flux(nx, ny, len, p->gamma, qL, qR, flux);
    if (jupdate) boundary_jacobian(g, p, i, qL, qR, nx, ny, len);
    for (int j = 0; j < NV; j++) g->R[rn * NV + j] += flux[j];
  }
  return 0;
}

/* ------------------------------------------------------------------ */
/* linear_algebra.C:122-401, 571-638                                     */
/* ------------------------------------------------------------------ */
static void lu4(double *A)
{
  for (int k = 0; k < 4; k++) {
    for (int i = k + 1; i < 4; i++) A[i * 4 + k] = A[i * 4 + k] / A[k * 4 + k];
    for (int j = k + 1; j < 4; j++)
      for (int i = k + 1; i < 4; i++) A[i * 4 + j] = A[i * 4 + j] - A[i * 4 + k] * A[k * 4 + j];
  }
}

static void gs_row(orc_grid *g, double *rhs1, int j)
{
  const double *LHS = g->LHS, *dQ = g->dQ;
  double M[16], y[4], xx[4];
  for (int k = g->ia[j]; k < g->ia[j + 1]; k++) {
    int c = g->ja[k];
    if (c == j) continue;
    const double *A = &LHS[(long)k * 16];
    const double *d = &dQ[c * NV];
    for (int r = 0; r < 4; r++)
      rhs1[j * NV + r] -= (A[r * 4] * d[0] + A[r * 4 + 1] * d[1] + A[r * 4 + 2] * d[2] +
                           A[r * 4 + 3] * d[3]);
  }
  memcpy(M, &LHS[(long)g->iau[j] * 16], sizeof(M));
  lu4(M);
  const double *b = &rhs1[j * NV];
  y[0] = b[0];
  y[1] = b[1] - M[4] * y[0];
  y[2] = b[2] - M[8] * y[0] - M[9] * y[1];
  y[3] = b[3] - M[12] * y[0] - M[13] * y[1] - M[14] * y[2];
  xx[3] = y[3] / M[15];
  xx[2] = (y[2] - M[11] * xx[3]) / M[10];
  xx[1] = (y[1] - M[6] * xx[2] - M[7] * xx[3]) / M[5];
  xx[0] = (y[0] - M[1] * xx[1] - M[2] * xx[2] - M[3] * xx[3]) / M[0];
  for (int r = 0; r < 4; r++) {
    double dx = xx[r] - g->dQ[j * NV + r];
    g->dQ[j * NV + r] += dx;
  }
}

double orc_linear_solve(orc_grid *g, const orc_params *p)
{
  int nn = g->nn;
  double RMS = 10.;
  double *rhs1 = (double *)malloc(sizeof(double) * (nn + 1) * NV);
  (void)p;
  for (int it = 0; it < p->subits; it++) {
    for (int j = 1; j <= nn; j++)
      for (int k = 0; k < NV; k++) rhs1[j * NV + k] = g->RHS[j * NV + k];
    if (it % 2 == 0)
      for (int j = 1; j <= nn; j++) gs_row(g, rhs1, j);
    else
      for (int j = nn; j >= 1; j--) gs_row(g, rhs1, j);
    RMS = 0.;
    for (int j = 1; j <= nn; j++) {
      double r[4];
      for (int k = 0; k < 4; k++) r[k] = g->RHS[j * NV + k];
      for (int k = g->ia[j]; k < g->ia[j + 1]; k++) {
        const double *A = &g->LHS[(long)k * 16];
        const double *d = &g->dQ[g->ja[k] * NV];
        for (int q = 0; q < 4; q++)
          r[q] -= (A[q * 4] * d[0] + A[q * 4 + 1] * d[1] + A[q * 4 + 2] * d[2] +
                   A[q * 4 + 3] * d[3]);
      }
      RMS += (r[0] * r[0] + r[1] * r[1] + r[2] * r[2] + r[3] * r[3]);
    }
    RMS /= (1. * nn);
    RMS = sqrt(RMS);
    if (RMS < 1.0E-15) break;
  }
  free(rhs1);
  return RMS;
}

/* ------------------------------------------------------------------ */
/* grid_io.C:1390-1697 Compute_Body_Forces (cached Gauss data)           */
/* ------------------------------------------------------------------ */
void orc_body_forces(orc_grid *g, const orc_params *p, double *F)
{
  double angle = p->alpha * M_PI / 180;
  double ca = cos(angle), sa = sin(angle);
  F[0] = 0.;
  F[1] = 0.;
  double q[4];
  for (int i = 1; i <= g->nbedges; i++) {
    int rn = g->bedges[i * 5];
    int bc = g->bbc[g->bedges[i * 5 + 3]];
    if (bc == 0 || (bc % 2 == 0)) continue;
    double t1 = 0., t2 = 0., len;
    if (bc <= 10) {
      double nx = -g->xn_bedges[i * 3], ny = -g->xn_bedges[i * 3 + 1];
      len = g->xn_bedges[i * 3 + 2];
      const double w[3] = {5. / 9., 8. / 9., 5. / 9.};
      for (int k = 0; k < 3; k++) {
        reconstruct_gauss_boundary(g, p, rn, &g->xg_bedges[i * 6 + 2 * k], q);
        double r = q[0], u = q[1] / r, v = q[2] / r, e = q[3];
        double P = (p->gamma - 1.) * (e - 0.5 * r * (u * u + v * v));
        t1 += (w[k] * (P * ny * ca - P * nx * sa));
        t2 += (w[k] * (P * nx * ca + P * ny * sa));
      }
    } else {
      len = g->xgn_bedges[i * 9 + 2];
      const double w[3] = {8. / 9., 5. / 9., 5. / 9.};
      for (int k = 0; k < 3; k++) {
        double nx = -g->xgn_bedges[i * 9 + k * 3], ny = -g->xgn_bedges[i * 9 + k * 3 + 1];
        reconstruct_gauss_boundary(g, p, rn, &g->xg_bedges[i * 6 + 2 * k], q);
        double r = q[0], u = q[1] / r, v = q[2] / r, e = q[3];
        double P = (p->gamma - 1.) * (e - 0.5 * r * (u * u + v * v));
        t1 += (w[k] * (P * ny * ca - P * nx * sa));
        t2 += (w[k] * (P * nx * ca + P * ny * sa));
      }
    }
    t1 = t1 * len * 0.5;
    t2 = t2 * len * 0.5;
    F[0] += t1;
    F[1] += t2;
  }
}

/* ------------------------------------------------------------------ */
/* solve.C:44-933 (steady implicit, orders 1 and 3, limiter 2)          */
/* ------------------------------------------------------------------ */
/* ------------------------------------------------------------------ */
/* Precision form: multicolour FP32 block Gauss-Seidel (no reference     */
/* counterpart; the FP64 sweep it replaces is linear_algebra.C:178-344)  */
/* ------------------------------------------------------------------ */
int orc_greedy_colors(const orc_grid *g, int *color)
{
  int nn = g->nn, ncol = 0;
  unsigned char used[256];
  for (int j = 1; j <= nn; j++) {
    memset(used, 0, sizeof(used));
    for (int k = g->ia[j]; k < g->ia[j + 1]; k++) {
      int c = g->ja[k];
      if (c < j) used[color[c]] = 1;
    }
    int col = 0;
    while (col < 255 && used[col]) col++;
    color[j] = col;
    if (col + 1 > ncol) ncol = col + 1;
  }
  return ncol;
}

static void gs_row_mixed(const orc_grid *g, const float *A32, const float *lu32, float *dq32,
                         int j)
{
  float b[4];
  for (int r = 0; r < 4; r++) b[r] = (float)g->RHS[j * NV + r];
  for (int k = g->ia[j]; k < g->ia[j + 1]; k++) {
    int c = g->ja[k];
    if (c == j) continue;
    const float *a = &A32[(long)k * 16];
    const float *d = &dq32[c * NV];
    for (int r = 0; r < 4; r++) {
      float t = a[r * 4] * d[0];
      t = fmaf(a[r * 4 + 1], d[1], t);
      t = fmaf(a[r * 4 + 2], d[2], t);
      t = fmaf(a[r * 4 + 3], d[3], t);
      b[r] = b[r] - t;
    }
  }
  const float *M = &lu32[j * 16];  /* LU factors, reciprocal pivots on the diagonal */
  float y0 = b[0];
  float y1 = fmaf(-M[4], y0, b[1]);
  float y2 = fmaf(-M[9], y1, fmaf(-M[8], y0, b[2]));
  float y3 = fmaf(-M[14], y2, fmaf(-M[13], y1, fmaf(-M[12], y0, b[3])));
  float x3 = y3 * M[15];
  float x2 = fmaf(-M[11], x3, y2) * M[10];
  float x1 = fmaf(-M[7], x3, fmaf(-M[6], x2, y1)) * M[5];
  float x0 = fmaf(-M[3], x3, fmaf(-M[2], x2, fmaf(-M[1], x1, y0))) * M[0];
  dq32[j * NV] = x0;
  dq32[j * NV + 1] = x1;
  dq32[j * NV + 2] = x2;
  dq32[j * NV + 3] = x3;
}

/* color == NULL: the reference's row order (forward 1..nn, backward nn..1,
 * in place, so earlier rows of the sweep are already updated). */
void orc_linear_solve_mixed(orc_grid *g, const orc_params *p, const int *color, int ncolors)
{
  int nn = g->nn;
  long nnz = g->ia[nn + 1];
  float *A32 = (float *)malloc(sizeof(float) * 16 * (nnz > 0 ? nnz : 1));
  float *lu32 = (float *)malloc(sizeof(float) * 16 * (nn + 1));
  float *dq32 = (float *)calloc((size_t)(nn + 1) * NV, sizeof(float));
  for (long k = 0; k < 16 * nnz; k++) A32[k] = (float)g->LHS[k];
  for (int j = 1; j <= nn; j++) {
    double M[16];
    memcpy(M, &g->LHS[(long)g->iau[j] * 16], sizeof(M));
    lu4(M);
    for (int q = 0; q < 16; q++) lu32[j * 16 + q] = (float)M[q];
    for (int q = 0; q < 4; q++) lu32[j * 16 + 5 * q] = (float)(1.0 / M[5 * q]);
  }
  for (int it = 0; it < p->subits; it++) {
    if (!color) {
      if (it % 2 == 0)
        for (int j = 1; j <= nn; j++) gs_row_mixed(g, A32, lu32, dq32, j);
      else
        for (int j = nn; j >= 1; j--) gs_row_mixed(g, A32, lu32, dq32, j);
      continue;
    }
    for (int ci = 0; ci < ncolors; ci++) {
      int col = (it % 2 == 0) ? ci : ncolors - 1 - ci;
      for (int j = 1; j <= nn; j++)
        if (color[j] == col) gs_row_mixed(g, A32, lu32, dq32, j);
    }
  }
  for (int j = 1; j <= nn; j++)
    for (int r = 0; r < NV; r++) g->dQ[j * NV + r] = (double)dq32[j * NV + r];
  free(A32);
  free(lu32);
  free(dq32);
}

/* FP32 sweeps in an arbitrary row order: forward sweeps visit order[0..nn-1],
 * backward sweeps the reverse (in place). */
void orc_linear_solve_mixed_order(orc_grid *g, const orc_params *p, const int *order)
{
  int nn = g->nn;
  long nnz = g->ia[nn + 1];
  float *A32 = (float *)malloc(sizeof(float) * 16 * (nnz > 0 ? nnz : 1));
  float *lu32 = (float *)malloc(sizeof(float) * 16 * (nn + 1));
  float *dq32 = (float *)calloc((size_t)(nn + 1) * NV, sizeof(float));
  for (long k = 0; k < 16 * nnz; k++) A32[k] = (float)g->LHS[k];
  for (int j = 1; j <= nn; j++) {
    double M[16];
    memcpy(M, &g->LHS[(long)g->iau[j] * 16], sizeof(M));
    lu4(M);
    for (int q = 0; q < 16; q++) lu32[j * 16 + q] = (float)M[q];
    for (int q = 0; q < 4; q++) lu32[j * 16 + 5 * q] = (float)(1.0 / M[5 * q]);
  }
  for (int it = 0; it < p->subits; it++) {
    if (it % 2 == 0)
      for (int i = 0; i < nn; i++) gs_row_mixed(g, A32, lu32, dq32, order[i]);
    else
      for (int i = nn - 1; i >= 0; i--) gs_row_mixed(g, A32, lu32, dq32, order[i]);
  }
  for (int j = 1; j <= nn; j++)
    for (int r = 0; r < NV; r++) g->dQ[j * NV + r] = (double)dq32[j * NV + r];
  free(A32);
  free(lu32);
  free(dq32);
}

static int solve_impl(orc_grid *g, const orc_params *p, int ts, double *dqnorm, int mixed,
                      const int *color, int ncolors, const int *order);

int orc_solve_mixed_order(orc_grid *g, const orc_params *p, int ts, double *dqnorm,
                          const int *order)
{
  return solve_impl(g, p, ts, dqnorm, 2, NULL, 0, order);
}

int orc_solve(orc_grid *g, const orc_params *p, int ts, double *dqnorm)
{
  return solve_impl(g, p, ts, dqnorm, 0, NULL, 0, NULL);
}

int orc_solve_mixed(orc_grid *g, const orc_params *p, int ts, double *dqnorm, const int *color,
                    int ncolors)
{
  return solve_impl(g, p, ts, dqnorm, 1, color, ncolors, NULL);
}

static int solve_impl(orc_grid *g, const orc_params *p, int ts, double *dqnorm, int mixed,
                      const int *color, int ncolors, const int *order)
{
  int nn = g->nn, rc;
  double dql2 = 0.;
  for (int n = 1; n <= nn; n++)
    for (int k = 0; k < 8; k++) g->grad[n * 8 + k] = 0.;
  for (int i = 0; i <= nn; i++)
    for (int k = 0; k < 36; k++) g->hess[i * 36 + k] = 0.;
  for (int i = 1; i <= nn + g->nn_ghost; i++)
    for (int j = 0; j < NV; j++) g->nQ[i * NV + j] = g->Q[i * NV + j];
  for (int m = 1; m <= p->iter; m++) {
    int jac = ((m - 1) % p->jufreq == 0) || m == 1;
    if (p->method == 0) jac = 0;
    for (int i = 1; i <= nn; i++)
      for (int j = 0; j < 8; j++) g->phi[i * 8 + j] = 1.;
    if ((rc = orc_build_matrix(g, p))) return 10 + rc;
    if ((p->order == 1 || p->order == 2) && ts > p->foits)
      orc_gradient_lsq(g);
    else if (p->order == 3 && ts > p->foits) {
      if (ts <= p->foits + p->soits) orc_gradient_lsq(g);
      else orc_derivatives_k2(g);
    }
    int do_lim = 0;
    if ((p->order == 1 || p->order == 2) && p->limit > 0 && ts > p->foits) do_lim = 1;
    if (p->order == 3 && p->limit > 0 && ts > (p->foits + p->soits)) do_lim = 1;
    if (do_lim) {
      if (p->limit != 2) return 20;
      if (orc_limiter_venkat(g, p)) return 21;
    }
    orc_interior_residuals(g, p, jac, ts);
    if ((rc = orc_boundary_residuals(g, p, jac))) return 30 + rc;
    for (int i = 0; i <= nn; i++)
      for (int j = 0; j < NV; j++) g->dQ[i * NV + j] = 0.;
    if (p->tacc != 0 || p->unsteady != 0) return 40;
    for (int i = 1; i <= nn; i++)
      for (int j = 0; j < NV; j++) g->RHS[i * NV + j] = -(g->R[i * NV + j]);
    if (mixed == 2)
      orc_linear_solve_mixed_order(g, p, order);
    else if (mixed)
      orc_linear_solve_mixed(g, p, color, ncolors);
    else
      orc_linear_solve(g, p);
    dql2 = 0.;
    for (int i = 1; i <= nn; i++)
      for (int j = 0; j < NV; j++) dql2 += (g->dQ[i * NV + j] * g->dQ[i * NV + j]);
    for (int i = 1; i <= nn; i++)
      for (int j = 0; j < NV; j++) g->nQ[i * NV + j] += g->dQ[i * NV + j];
  }
  for (int i = 1; i <= nn + g->nn_ghost; i++)
    for (int j = 0; j < NV; j++) g->pQ[i * NV + j] = g->Q[i * NV + j];
  for (int i = 1; i <= nn + g->nn_ghost; i++)
    for (int j = 0; j < NV; j++) g->Q[i * NV + j] = g->nQ[i * NV + j];
  *dqnorm = sqrt(dql2);
  return 0;
}
