/*
 * curved.h - analytic curved boundaries of the reference (bc 11..22).
 *
 * Reserved boundary conditions (curved_boundaries.C:24-45): 11/12 unit
 * circle, 13/14 R=2 circle, 15/16 R=3 circle, 17/18 NACA 0012 upper
 * surface, 19/20 lower surface, 21/22 R=300 circle; odd = inviscid wall,
 * even = far field.  The NACA surface is the closed-trailing-edge airfoil
 * y = 0.6 (0.2969 sqrt(x) - 0.1260 x - 0.3516 x^2 + 0.2843 x^3 - 0.1036 x^4)
 * that the reference hard-codes (curved_boundaries.C:47-74).
 */
#ifndef FLOW_CURVED_H
#define FLOW_CURVED_H

#ifdef __cplusplus
extern "C" {
#endif

/* Outward (out of the fluid) unit normal at boundary point x
 * (curved_boundaries.C:701-877). */
void flow_curved_normal(int bc, const double *x, double *nx, double *ny);

/* Arc length of the curve between xL and xR (curved_boundaries.C:1009-1155). */
void flow_curved_arclength(int bc, const double *xL, const double *xR, double *len);

/* Point halfway along the boundary between xL and xR
 * (curved_boundaries.C:91-328; for the NACA curves the reference returns the
 * curve point above the chord midpoint). */
void flow_curved_midpoint(int bc, const double *xL, const double *xR, double *xM);

/* The 3 Gauss points of the curve piece between xL and xR, equally spaced
 * in arc length at the Gauss-Legendre abscissae, centre point first
 * (curved_boundaries.C:345-700). */
void flow_curved_gauss_points(int bc, const double *xL, const double *xR, double *GP);

#ifdef __cplusplus
}
#endif

#endif
