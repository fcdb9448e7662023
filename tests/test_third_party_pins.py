"""The two third-party numerical routines the reference links, pinned
against independent implementations (CPU only).

* LAPACK dgesvd_ (compute_derivatives.C:928, JOBU = JOBVT = 'A'): the k=2
  preprocessing factors every node's weighted m x 5 stencil system with the
  solver's own one-sided Jacobi SVD (host/svd.c), and the oracle's stand-in
  for dgesvd_ forwards to the same routine.  Here the system of every node
  of a curved k=2 mesh is rebuilt in numpy (the rows of
  compute_derivatives.C:859-917) and factored by LAPACK's dgesvd (scipy's
  binding) and by numpy.linalg.pinv; the stored singular values and the
  pseudo-inverse V S^-1 U1^T that the derivative kernel applies must agree.
* GSL gsl_integration_qags (curved_boundaries.C:238-256, 555-572, asked for
  1e-8 absolute and relative error): the curved-boundary arc lengths go
  through the solver's adaptive Gauss-Legendre quadrature (host/quadrature.c).
  Here NACA arc lengths and singular test integrals are compared with
  scipy.integrate.quad, QUADPACK's qags (the algorithm GSL's qags
  implements), run at a much tighter tolerance.
"""
import ctypes as C

import numpy as np
import pytest

# singular values: relative to the largest (seen: 1.5e-15 on 64x16)
SVD_RTOL = 1e-13
# pseudo-inverse entries: relative to the largest, for stencil systems with
# condition numbers up to ~2e3 (seen: 1.0e-14)
PINV_RTOL = 1e-12
# the reference asks qags for 1e-8 (abs and rel); seen: 2.3e-13 relative
QUAD_RTOL = 1e-10


def _stencil_systems(mesh):
    """Yield (node, A, U1, S, VT) with A the weighted reduced m x 5 system of
    compute_derivatives.C:859-917 and the factors the preprocessing stored."""
    nn = mesh.sizes["nn"]
    x = mesh.array("x").reshape(-1, 2)
    mo = mesh.array("moments").reshape(-1, 9)
    gnsn, gnnsn, gnnsn1 = mesh.array("gnsn"), mesh.array("gnnsn"), mesh.array("gnnsn1")
    off, U = mesh.array("svd_off"), mesh.array("svd_U")
    VT, S = mesh.array("svd_VT").reshape(-1, 5, 5), mesh.array("svd_S").reshape(-1, 5)
    for i in range(1, nn + 1):
        a0, a1 = gnnsn[gnnsn1[i] + 1], gnnsn[gnnsn1[i + 1]]
        m = a1 - a0
        nb = gnsn[a0:a1]
        d0, d1 = x[nb, 0] - x[i, 0], x[nb, 1] - x[i, 1]
        w = 1.0 / np.sqrt(d0 * d0 + d1 * d1)
        A = np.empty((m, 5))
        A[:, 0] = w * (d0 + mo[nb, 0] - mo[i, 0])
        A[:, 1] = w * (d1 + mo[nb, 1] - mo[i, 1])
        A[:, 2] = 0.5 * w * (d0 * d0 + 2.0 * mo[nb, 0] * d0 + mo[nb, 2] - mo[i, 2])
        A[:, 3] = 0.5 * w * (d1 * d1 + 2.0 * mo[nb, 1] * d1 + mo[nb, 3] - mo[i, 3])
        A[:, 4] = w * (mo[nb, 4] + mo[nb, 0] * d1 + mo[nb, 1] * d0 + d1 * d0 - mo[i, 4])
        U1 = U[off[i]:off[i] + 5 * m].reshape(5, m).T   # column-major m x 5
        yield i, A, U1, S[i], VT[i].T                   # VT column-major 5 x 5


@pytest.mark.parametrize("nc,nr", [(64, 16), (96, 24)])
def test_stencil_svd_matches_lapack_dgesvd_and_numpy(nc, nr):
    from scipy.linalg import lapack
    from flowgpu import workloads
    from flowgpu.prep import Mesh
    wl = workloads.Workload(f"svdpin{nc}x{nr}", nc, nr, True, 3, 0.8)
    mesh = Mesh.from_case(wl.write(), order=3)
    n = 0
    for i, A, U1, s, VT in _stencil_systems(mesh):
        u, s_ref, vt, info = lapack.dgesvd(A, full_matrices=1)
        assert info == 0
        assert np.max(np.abs(s - s_ref)) <= SVD_RTOL * s_ref[0], i
        P = VT.T @ np.diag(1.0 / s) @ U1.T
        P_lapack = vt.T @ np.diag(1.0 / s_ref) @ u[:, :5].T
        P_numpy = np.linalg.pinv(A)
        scale = np.max(np.abs(P_lapack))
        assert np.max(np.abs(P - P_lapack)) <= PINV_RTOL * scale, i
        assert np.max(np.abs(P - P_numpy)) <= PINV_RTOL * scale, i
        # the left factor's columns are orthonormal, as dgesvd's are
        assert np.max(np.abs(U1.T @ U1 - np.eye(5))) <= 1e-13, i
        n += 1
    assert n == mesh.sizes["nn"]
    mesh.close()


def _naca_y(x, bc):
    y = 0.6 * (0.2969 * np.sqrt(x) - 0.1260 * x - 0.3516 * x * x + 0.2843 * x ** 3
               - 0.1036 * x ** 4)
    return y if bc in (17, 18) else -y


def test_naca_arc_lengths_match_qags():
    from scipy.integrate import quad
    from flowgpu import capi
    L = capi.load()
    D2 = C.c_double * 2
    L.flow_curved_arclength.argtypes = [C.c_int, D2, D2, C.POINTER(C.c_double)]

    def integrand(x):  # |ds/dx| of the reference's surface (curved_boundaries.C:58-74)
        s = 0.08907 / np.sqrt(x) - 0.07560 - 0.42192 * x + 0.51174 * x * x - 0.24864 * x ** 3
        return np.sqrt(1.0 + s * s)

    xs = 0.5 * (1.0 - np.cos(np.linspace(0.0, np.pi, 129)))  # cosine-clustered wall nodes
    pieces = list(zip(xs[:-1], xs[1:])) + [(0.0, 1.0), (0.0, 0.5), (0.3, 0.9)]
    for bc in (17, 19):
        for a, b in pieces:
            out = C.c_double()
            L.flow_curved_arclength(bc, D2(b, _naca_y(b, bc)), D2(a, _naca_y(a, bc)),
                                    C.byref(out))
            ref, _err = quad(integrand, a, b, epsabs=1e-14, epsrel=1e-13, limit=500)
            assert abs(out.value - ref) <= QUAD_RTOL * ref, (bc, a, b, out.value, ref)


def test_adaptive_quadrature_on_singular_integrands():
    """flow_quad_adaptive itself, on integrands with the endpoint behaviour
    of the arc-length integrand (1/sqrt(x)) and worse (log x), at the
    tolerance the reference requests."""
    from scipy.integrate import quad
    from flowgpu import capi
    L = capi.load()
    QF = C.CFUNCTYPE(C.c_double, C.c_double, C.c_void_p)
    L.flow_quad_adaptive.argtypes = [QF, C.c_void_p, C.c_double, C.c_double, C.c_double,
                                     C.c_double, C.c_int, C.POINTER(C.c_double),
                                     C.POINTER(C.c_double)]
    cases = [(lambda x: 1.0 / np.sqrt(x), 0.0, 1.0), (lambda x: np.log(x), 0.0, 1.0),
             (lambda x: np.cos(x), 0.0, np.pi / 2), (lambda x: np.sqrt(x) * np.exp(-x), 0.0, 3.0)]
    for f, a, b in cases:
        r, e = C.c_double(), C.c_double()
        cb = QF(lambda x, _p, f=f: f(x))
        rc = L.flow_quad_adaptive(cb, None, a, b, 1e-8, 1e-8, 1000, C.byref(r), C.byref(e))
        ref, _ = quad(f, a, b, epsabs=1e-14, epsrel=1e-13, limit=500)
        assert rc == 0
        assert abs(r.value - ref) <= max(1e-8, 1e-8 * abs(ref))
