/*
 * curved.c - analytic curved boundaries (see curved.h).
 *
 * Same formulas and the same floating-point operation order as
 * curved_boundaries.C, so host preprocessing reproduces the reference's
 * curved-boundary geometry bit for bit (the arc-length integral goes through
 * flow_quad_adaptive, the quadrature that also stands in for the
 * reference's GSL call).
 */
#include <math.h>
#include "curved.h"
#include "quadrature.h"

/* curved_boundaries.C:47-56 (closed trailing edge coefficient -0.1036) */
static double naca_y(double x, int bc)
{
  double y = 0.6 * (0.2969 * sqrt(x) - 0.1260 * x - 0.3516 * x * x + 0.2843 * x * x * x -
                    0.1036 * x * x * x * x);
  if (bc == 19 || bc == 20) y = -1.0 * y;
  return y;
}

/* curved_boundaries.C:58-74: |ds/dx| and its negative */
static double naca_slope(double x)
{
  return 0.08907 / sqrt(x) - 0.07560 - 0.42192 * x + 0.51174 * x * x - 0.24864 * x * x * x;
}

static double naca_arclen_integrand(double x, void *params)
{
  (void)params;
  double s = naca_slope(x);
  return sqrt(1.0 + s * s);
}

static double naca_arclen_deriv(double x)
{
  double s = naca_slope(x);
  return -1.0 * sqrt(1.0 + s * s);
}

static double circle_angle_acos(const double *x)
{
  if (x[0] >= 0. && x[1] >= 0.) return acos(x[0]);
  if (x[0] >= 0. && x[1] < 0.) return -acos(x[0]);
  if (x[0] < 0. && x[1] >= 0.) return acos(x[0]);
  return -acos(x[0]);
}

static int is_naca(int bc) { return bc >= 17 && bc <= 20; }

static double circle_radius(int bc)
{
  if (bc == 13 || bc == 14) return 2.;
  if (bc == 15 || bc == 16) return 3.;
  if (bc == 21 || bc == 22) return 300.;
  return 1.;
}

void flow_curved_normal(int bc, const double *x, double *nx, double *ny)
{
  double t;
  if (bc == 11 || bc == 12) {
    t = circle_angle_acos(x);
    if (bc == 11) { *nx = -cos(t); *ny = -sin(t); }
    else { *nx = cos(t); *ny = sin(t); }
    return;
  }
  if (bc == 13 || bc == 14) {
    t = atan2(x[1], x[0]);
    *nx = -cos(t);
    *ny = -sin(t);
    return;
  }
  if (bc == 15 || bc == 16 || bc == 21 || bc == 22) {
    t = atan2(x[1], x[0]);
    *nx = cos(t);
    *ny = sin(t);
    return;
  }
  if (is_naca(bc)) {
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

static double naca_length(double xa, double xb)
{
  double r = 0.0, e = 0.0;
  flow_quad_adaptive(naca_arclen_integrand, 0, xa, xb, 1.0e-8, 1.0e-8, 1000, &r, &e);
  return r;
}

void flow_curved_arclength(int bc, const double *xL, const double *xR, double *len)
{
  double tL, tR;
  if (bc == 11 || bc == 12) {
    tL = circle_angle_acos(xL);
    tR = circle_angle_acos(xR);
    if (tL < 0. && tR > 0.) tR = -1. * tR;
    else if (tL > 0. && tR < 0.) tL = -1. * tL;
    *len = fabs(tR - tL);
    return;
  }
  if (bc == 13 || bc == 14 || bc == 15 || bc == 16) {
    tL = atan2(xL[1], xL[0]);
    tR = atan2(xR[1], xR[0]);
    *len = fabs(tR - tL) * circle_radius(bc);
    return;
  }
  if (is_naca(bc)) {
    double xa = xL[0] > xR[0] ? xR[0] : xL[0];
    double xb = xL[0] > xR[0] ? xL[0] : xR[0];
    *len = naca_length(xa, xb);
    return;
  }
  if (bc == 21 || bc == 22) {
    tL = atan2(xL[1], xL[0]);
    tR = atan2(xR[1], xR[0]);
    if (tL < 0. && tR > 0.) tR = -1. * tR;
    else if (tL > 0. && tR < 0.) tL = -1. * tL;
    *len = fabs(tR - tL) * 300.;
  }
}

void flow_curved_midpoint(int bc, const double *xL, const double *xR, double *xM)
{
  double tL, tR, tM, r = circle_radius(bc);
  if (bc == 11 || bc == 12) {
    tL = circle_angle_acos(xL);
    tR = circle_angle_acos(xR);
  } else if (!is_naca(bc)) {
    tL = atan2(xL[1], xL[0]);
    tR = atan2(xR[1], xR[0]);
  } else {
    xM[0] = 0.5 * (xL[0] + xR[0]);
    xM[1] = naca_y(xM[0], bc);
    return;
  }
  if (tL < 0. && tR > 0.) tR = -1. * tR;
  else if (tL > 0. && tR < 0.) tL = -1. * tL;
  tM = 0.5 * (tL + tR);
  if (bc == 11 || bc == 12) {
    xM[0] = cos(tM);
    xM[1] = sin(tM);
  } else {
    xM[0] = r * cos(tM);
    xM[1] = r * sin(tM);
  }
}

void flow_curved_gauss_points(int bc, const double *xL, const double *xR, double *GP)
{
  const double t[3] = {0.0, sqrt(0.6), -1.0 * sqrt(0.6)};
  if (is_naca(bc)) {
    const double beta[3] = {0.5, (1.0 + sqrt(3. / 5.)) * 0.5, (1.0 - sqrt(3. / 5.)) * 0.5};
    double xa = xL[0] < xR[0] ? xL[0] : xR[0];
    double xb = xL[0] < xR[0] ? xR[0] : xL[0];
    for (int i = 0; i < 3; i++) {
      double Lt = naca_length(xa, xb);
      double xn = (xa + xb) * 0.5 + (xb - xa) * 0.5 * t[i];
      double xnp1 = xn;
      for (int j = 1; j <= 50; j++) {
        double L = naca_length(xa, xn);
        double f = (beta[i] * Lt) - L;
        double fp = naca_arclen_deriv(xn);
        double update = (f / fp);
        xnp1 = xn - (f / fp);
        while (xnp1 < xa || xnp1 > xb) {
          update = 0.5 * update;
          xnp1 = xn - update;
        }
        if (fabs(f) < 1.0E-12) break;
        xn = xnp1;
      }
      GP[i * 2 + 0] = xnp1;
      GP[i * 2 + 1] = naca_y(xnp1, bc);
    }
    return;
  }
  double thL, thR;
  if (bc == 11 || bc == 12) {
    thL = circle_angle_acos(xL);
    thR = circle_angle_acos(xR);
  } else {
    thL = atan2(xL[1], xL[0]);
    thR = atan2(xR[1], xR[0]);
  }
  if (thL < 0. && thR > 0.) thR = -1. * thR;
  else if (thL > 0. && thR < 0.) thL = -1. * thL;
  double r = circle_radius(bc);
  for (int i = 0; i < 3; i++) {
    double th = (thL + thR) * 0.5 + (thR - thL) * 0.5 * t[i];
    if (bc == 11 || bc == 12) {
      GP[2 * i] = cos(th);
      GP[2 * i + 1] = sin(th);
    } else {
      GP[2 * i] = r * cos(th);
      GP[2 * i + 1] = r * sin(th);
    }
  }
}
