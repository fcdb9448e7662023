"""Known answers the reference checks with its debug switches and run-time
checks, on the oracle and the host preprocessing (CPU only):

* closure: the outward normals of every median-dual control volume sum to
  zero (cv_calc.C:379-640, cv_calc_check_closure);
* the k=1 least-squares gradient is exact for linear fields (gradient.C:
  326-336, the DEBUG_GRAD fields);
* the k=2 derivatives and point value are exact for quadratics given as
  control-volume averages (compute_derivatives.C:317-342, DEBUG_DERIVS);
* freestream preservation: with Q the freestream everywhere, the interior
  residual of a node without boundary faces vanishes to rounding.

The CUDA drop-in is held to the same answers in test_gpu_known_answers.py.
Tolerances are absolute and stated per test; a reconstruction that is not
exact misses them by many orders of magnitude (errors of O(h) or O(h^2)
times the field's derivatives, 1e-5 and up on these meshes)."""
import numpy as np
import pytest

from cases import (closure_leak, interior_nodes, kat_mesh as mesh_of, linear_state,
                   quad_derivs, quad_values, quadratic_state, KAT_KINDS as KINDS, LINEAR_COEF)

CLOSURE_TOL = 1e-14   # |sum of normals| / perimeter; observed <= 1e-16
LINEAR_TOL = 1e-10    # gradient of fields of size ~500; observed ~1e-12
# k=2 first and second derivatives: rounding of the field values (eps x |q|,
# |q| up to 600) divided by h^2 of the wall cells (h ~ 1e-2) gives up to ~6e-9;
# a scheme that is not exact for quadratics errs by >= 1e-5 on these fields
QUAD_D_TOL = 1e-7
QUAD_PV_TOL = 1e-11   # k=2 point value; observed ~1e-13
FREESTREAM_TOL = 1e-13  # interior residual; observed ~3e-15


def _oracle(mesh):
    from oracle import port
    return port.OracleGrid(mesh.sizes, mesh.arrays())


@pytest.mark.parametrize("kind", KINDS)
def test_control_volumes_close(kind):
    mesh, _ = mesh_of(kind, 3 if kind in ("curved", "cylinder") else 1)
    assert closure_leak(mesh).max() <= CLOSURE_TOL
    mesh.close()


@pytest.mark.parametrize("kind", KINDS)
def test_lsq_gradient_is_exact_for_linear_fields(kind):
    mesh, fp = mesh_of(kind, 1)
    og = _oracle(mesh)
    nn = mesh.sizes["nn"]
    Q = linear_state(mesh.initial_state(fp), og["x"], nn)
    og.set("nQ", Q)
    og.gradient()
    g = og["grad"].reshape(-1, 4, 2)[1:nn + 1]
    assert np.abs(g - LINEAR_COEF[None, :, 1:]).max() <= LINEAR_TOL
    mesh.close()


@pytest.mark.parametrize("kind", KINDS)
def test_k2_derivatives_are_exact_for_quadratics(kind):
    mesh, fp = mesh_of(kind, 3)
    og = _oracle(mesh)
    nn = mesh.sizes["nn"]
    Q = quadratic_state(mesh.initial_state(fp), og["x"], mesh.arrays()["moments"], nn)
    og.set("nQ", Q)
    og.derivatives()
    X = og["x"].reshape(-1, 2)[1:nn + 1]
    h = og["hess"].reshape(-1, 4, 9)[1:nn + 1, :, :5]
    pv = og["point_value"].reshape(-1, 4)[1:nn + 1]
    assert np.abs(h - quad_derivs(X)).max() <= QUAD_D_TOL
    assert np.abs(pv - quad_values(X)).max() <= QUAD_PV_TOL
    mesh.close()


@pytest.mark.parametrize("kind,order", [("triangles", 1), ("quads", 1), ("triangles", 3),
                                        ("curved", 3), ("mixed", 3), ("cylinder", 3)])
def test_freestream_is_preserved(kind, order):
    from oracle import port
    mesh, fp = mesh_of(kind, order)
    og = _oracle(mesh)
    p = port.params_from_flow(fp)
    nn, nbe = mesh.sizes["nn"], mesh.sizes["nbedges"]
    Q = mesh.initial_state(fp)
    og.set("Q", Q)
    og.set("nQ", Q)
    og.g.citer = 1
    og.build_matrix(p)
    if order == 1:
        og.gradient()
    else:
        og.derivatives()
    og.limiter(p)
    og.interior(p, 1, 1)
    R = og["R"].reshape(-1, 4)
    inner = interior_nodes(mesh.arrays()["bedges"], nbe, nn)
    assert len(inner) > nn // 2
    assert np.abs(R[inner]).max() <= FREESTREAM_TOL
    mesh.close()
