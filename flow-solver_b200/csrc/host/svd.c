/*
 * svd.c - one-sided Jacobi SVD (Hestenes), see svd.h.
 *
 * Column pairs (p,q) of the working copy W = A V are rotated until every
 * pair is orthogonal to within 1e-15 relative; then sigma_j = |W_j|,
 * U_j = W_j / sigma_j.  Columns are sorted by descending sigma and U is
 * completed to a square orthonormal matrix with modified Gram-Schmidt
 * against the canonical basis.
 */
#include <math.h>
#include <string.h>
#include "svd.h"

#define SVD_MAXM 64
#define SVD_MAXN 16

int flow_svd_jacobi(int m, int n, const double *A, double *s, double *U,
                    double *VT, int full_u)
{
    if (m < n || n < 1 || m > SVD_MAXM || n > SVD_MAXN) return -1;
    double W[SVD_MAXM * SVD_MAXN];
    double V[SVD_MAXN * SVD_MAXN];
    memcpy(W, A, sizeof(double) * (size_t)m * n);
    for (int i = 0; i < n * n; i++) V[i] = 0.0;
    for (int i = 0; i < n; i++) V[i * n + i] = 1.0;

    for (int sweep = 0; sweep < 60; sweep++) {
        int rotated = 0;
        for (int p = 0; p < n - 1; p++) {
            for (int q = p + 1; q < n; q++) {
                double *wp = W + (size_t)p * m, *wq = W + (size_t)q * m;
                double alpha = 0.0, beta = 0.0, gamma = 0.0;
                for (int k = 0; k < m; k++) {
                    alpha += wp[k] * wp[k];
                    beta += wq[k] * wq[k];
                    gamma += wp[k] * wq[k];
                }
                if (fabs(gamma) <= 1e-15 * sqrt(alpha * beta) || gamma == 0.0)
                    continue;
                rotated = 1;
                double zeta = (beta - alpha) / (2.0 * gamma);
                double t = (zeta >= 0.0 ? 1.0 : -1.0) /
                           (fabs(zeta) + sqrt(1.0 + zeta * zeta));
                double c = 1.0 / sqrt(1.0 + t * t), sn = c * t;
                for (int k = 0; k < m; k++) {
                    double a = wp[k], b = wq[k];
                    wp[k] = c * a - sn * b;
                    wq[k] = sn * a + c * b;
                }
                double *vp = V + (size_t)p * n, *vq = V + (size_t)q * n;
                for (int k = 0; k < n; k++) {
                    double a = vp[k], b = vq[k];
                    vp[k] = c * a - sn * b;
                    vq[k] = sn * a + c * b;
                }
            }
        }
        if (!rotated) break;
    }

    /* singular values and sort order */
    double sig[SVD_MAXN];
    int order[SVD_MAXN];
    for (int j = 0; j < n; j++) {
        double nrm = 0.0;
        for (int k = 0; k < m; k++) nrm += W[j * m + k] * W[j * m + k];
        sig[j] = sqrt(nrm);
        order[j] = j;
    }
    for (int i = 1; i < n; i++) {
        int key = order[i], j = i - 1;
        while (j >= 0 && sig[order[j]] < sig[key]) { order[j + 1] = order[j]; j--; }
        order[j + 1] = key;
    }

    for (int j = 0; j < n; j++) {
        int src = order[j];
        s[j] = sig[src];
        double inv = sig[src] > 0.0 ? 1.0 / sig[src] : 0.0;
        for (int k = 0; k < m; k++) U[(size_t)j * m + k] = W[src * m + k] * inv;
        /* VT(j, c) = V(c, src), column-major with ldvt = n */
        for (int c = 0; c < n; c++) VT[(size_t)c * n + j] = V[src * n + c];
    }

    if (!full_u) return 0;

    /* complete U to m x m */
    int have = n;
    for (int e = 0; e < m && have < m; e++) {
        double v[SVD_MAXM];
        for (int k = 0; k < m; k++) v[k] = (k == e) ? 1.0 : 0.0;
        for (int pass = 0; pass < 2; pass++) {
            for (int j = 0; j < have; j++) {
                double d = 0.0;
                for (int k = 0; k < m; k++) d += U[(size_t)j * m + k] * v[k];
                for (int k = 0; k < m; k++) v[k] -= d * U[(size_t)j * m + k];
            }
        }
        double nrm = 0.0;
        for (int k = 0; k < m; k++) nrm += v[k] * v[k];
        nrm = sqrt(nrm);
        if (nrm < 1e-3) continue;
        for (int k = 0; k < m; k++) U[(size_t)have * m + k] = v[k] / nrm;
        have++;
    }
    return have == m ? 0 : 1;
}
