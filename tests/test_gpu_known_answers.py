"""The CUDA drop-in held to the reference's known answers, through the C ABI
(flow_set_state, flow_build_matrix, flow_reconstruct, flow_residuals):
the k=1 gradient exact for linear fields (gradient.C:326-336, DEBUG_GRAD),
the k=2 derivatives and point value exact for control-volume averages of
quadratics (compute_derivatives.C:317-342, DEBUG_DERIVS), and a freestream
state giving a zero interior residual at nodes without boundary faces.
The fields and tolerances are the ones test_known_answers.py applies to the
oracle."""
import numpy as np
import pytest

from cases import (interior_nodes, kat_mesh, linear_state, quad_derivs, quad_values,
                   quadratic_state, KAT_KINDS, LINEAR_COEF)
from test_known_answers import FREESTREAM_TOL, LINEAR_TOL, QUAD_D_TOL, QUAD_PV_TOL

pytestmark = pytest.mark.gpu


def _solver(mesh, fp):
    from flowgpu import capi
    return capi.Solver.from_mesh(mesh, fp, device=0)


@pytest.mark.parametrize("kind", KAT_KINDS)
def test_gradient_is_exact_for_linear_fields(kind):
    mesh, fp = kat_mesh(kind, 1)
    s = _solver(mesh, fp)
    nn = mesh.sizes["nn"]
    s.set_state(linear_state(mesh.initial_state(fp), mesh.array("x"), nn))
    s.reconstruct(2)
    g = s.get("grad").reshape(-1, 4, 2)[1:nn + 1]
    assert np.abs(g - LINEAR_COEF[None, :, 1:]).max() <= LINEAR_TOL
    assert s.status() == 0
    s.close()
    mesh.close()


@pytest.mark.parametrize("kind", KAT_KINDS)
def test_k2_derivatives_are_exact_for_quadratics(kind):
    mesh, fp = kat_mesh(kind, 3)
    s = _solver(mesh, fp)
    nn = mesh.sizes["nn"]
    x = mesh.array("x")
    s.set_state(quadratic_state(mesh.initial_state(fp), x, mesh.arrays()["moments"], nn))
    s.reconstruct(2)
    X = x.reshape(-1, 2)[1:nn + 1]
    h = s.get("hess").reshape(-1, 4, 9)[1:nn + 1, :, :5]
    pv = s.get("point_value").reshape(-1, 4)[1:nn + 1]
    assert np.abs(h - quad_derivs(X)).max() <= QUAD_D_TOL
    assert np.abs(pv - quad_values(X)).max() <= QUAD_PV_TOL
    assert s.status() == 0
    s.close()
    mesh.close()


@pytest.mark.parametrize("kind,order", [("triangles", 1), ("quads", 1), ("triangles", 3),
                                        ("curved", 3), ("mixed", 3), ("cylinder", 3)])
def test_freestream_is_preserved(kind, order):
    mesh, fp = kat_mesh(kind, order)
    s = _solver(mesh, fp)
    nn, nbe = mesh.sizes["nn"], mesh.sizes["nbedges"]
    s.set_state(mesh.initial_state(fp))
    s.build_matrix(1)
    s.reconstruct(1)
    s.residuals(1, 1)
    R = s.get("R").reshape(-1, 4)
    inner = interior_nodes(mesh.arrays()["bedges"], nbe, nn)
    assert np.abs(R[inner]).max() <= FREESTREAM_TOL
    s.close()
    mesh.close()
