"""The per-stage entry points of the C ABI against the reference's stage
functions, called one by one after one full step (the sequence of solve.C:
369-881): flow_build_matrix (build_matrix, init_memory.C:159-310),
flow_reconstruct (Compute_Gradient_LeastSquares or Compute_Derivatives, then
compute_limiter_venkatakrishnan), flow_residuals (build_interior_residuals and
build_boundary_residuals), flow_linear_solve (linear_solve,
linear_algebra.C:122-401) and flow_body_forces (Compute_Body_Forces).  Every
array each stage writes is bit-identical to the reference's; the returned
b - Ax RMS agrees to RMS_RTOL."""
import numpy as np
import pytest

from cases import make_case, ndiff

pytestmark = pytest.mark.gpu

# the b - Ax RMS of linear_solve is a sum over all rows, which the GPU reduces
# as a tree rather than in row order; every array is compared bit for bit
RMS_RTOL = 1e-12


@pytest.mark.parametrize("nc,nr,curved,order", [(64, 16, False, 1), (64, 16, True, 3)])
def test_stage_entry_points_match_the_reference(ref_lib, nc, nr, curved, order):
    from flowgpu import capi
    from flowgpu.prep import Mesh
    d, _, fp = make_case(nc, nr, curved, order)
    ref = ref_lib.RefSolver(d)
    mesh = Mesh.from_case(d, order=order)
    s = capi.Solver.from_mesh(mesh, fp, device=0)
    s.set_state(mesh.initial_state(fp))
    ref.solve(1)
    s.solve(1)
    nn = mesh.sizes["nn"]
    assert ndiff(ref.array("Q")[4:], s.get("Q")[4:]) == 0

    ref.set_citer(2)
    ref.build_matrix()
    s.build_matrix(2)
    assert ndiff(ref.array("LHS"), s.get("LHS")) == 0
    assert ndiff(ref.array("dt")[1:], s.get("dt")[1:]) == 0

    if order == 1:
        ref.gradient()
    else:
        ref.derivatives(3)
    ref.limiter()
    s.reconstruct(2)
    if order == 1:
        assert ndiff(ref.array("grad")[8:], s.get("grad")[8:]) == 0
    else:
        h_ref = ref.array("hess").reshape(-1, 4, 9)[1:nn + 1, :, :5]
        h_gpu = s.get("hess").reshape(-1, 4, 9)[1:nn + 1, :, :5]
        assert ndiff(h_ref, h_gpu) == 0
        assert ndiff(ref.array("point_value")[4:], s.get("point_value")[4:]) == 0
    assert ndiff(ref.array("phi")[8:], s.get("phi")[8:]) == 0

    ref.interior(1, 2)
    ref.boundary(1)
    s.residuals(1, 2)
    assert ndiff(ref.array("R")[4:], s.get("R")[4:]) == 0
    assert ndiff(ref.array("LHS"), s.get("LHS")) == 0
    assert ndiff(ref.array("xn_bedges")[3:], s.get("xn_bedges")[3:]) == 0  # row 0 unused
    assert ndiff(ref.array("nQ")[4:], s.get("nQ")[4:]) == 0  # ghost states

    ref.set_array("RHS", -ref.array("R"))
    ref.set_array("dQ", np.zeros_like(ref.array("dQ")))
    r_ref = ref.linear_solve()
    r_gpu = s.linear_solve()
    assert ndiff(ref.array("dQ")[4:], s.get("dQ")[4:]) == 0
    assert r_gpu == pytest.approx(r_ref, rel=RMS_RTOL)

    assert tuple(s.body_forces()) == tuple(ref.body_forces())
    assert s.status() == 0
    # summed in the reference's row order, the RMS is the reference's bits
    s.set_exact_rms(True)
    ref.set_array("dQ", np.zeros_like(ref.array("dQ")))
    assert s.linear_solve() == ref.linear_solve()
    assert ndiff(ref.array("dQ")[4:], s.get("dQ")[4:]) == 0
    s.close()
    mesh.close()
    ref.close()


@pytest.mark.parametrize("nc,nr,curved,order", [(64, 16, False, 1), (64, 16, True, 3)])
def test_split_residual_stages_and_host_reconstruction(ref_lib, nc, nr, curved, order):
    """build_interior_residuals and build_boundary_residuals one at a time
    (flow_residual_stage), in a context given the reference's own gradient,
    limiter and k=2 derivatives through flow_set: the arrays after each stage
    equal the reference's after the same stage, bit for bit.  For k=2 the
    context is made without device stencils (the derivatives are the
    host's), as a caller that keeps the reference's Compute_Derivatives
    makes it; its device k=2 steps refuse."""
    from flowgpu import capi
    from flowgpu.prep import Mesh
    d, _, fp = make_case(nc, nr, curved, order)
    ref = ref_lib.RefSolver(d)
    mesh = Mesh.from_case(d, order=order)
    sizes, arrays = mesh.sizes, mesh.arrays()
    if order == 3:
        for k in ("gnsn", "gnnsn", "gnnsn1", "svd_m", "svd_off", "svd_U", "svd_VT", "svd_S"):
            arrays[k] = None
    s = capi.Solver(sizes, arrays, fp, device=0)
    s.set_state(mesh.initial_state(fp))
    ref.solve(1)
    for name in ("Q", "nQ", "pQ", "xn_bedges"):  # the reference's state after step 1
        s.set(name, ref.array(name))
    if order == 3:
        with pytest.raises(capi.FlowError):
            s.reconstruct(2)  # k=2 derivatives on the device need the stencils
    ref.set_citer(2)
    ref.build_matrix()
    s.build_matrix(2)
    assert ndiff(ref.array("LHS"), s.get("LHS")) == 0
    if order == 1:
        ref.gradient()
    else:
        ref.derivatives(3)
    ref.limiter()
    names = ("grad", "phi") if order == 1 else ("hess", "point_value", "phi")
    for name in names:
        s.set(name, ref.array(name))
    ref.interior(1, 2)
    s.residual_stage(1, 2, capi.Solver.STAGE_INTERIOR)
    assert ndiff(ref.array("R")[4:], s.get("R")[4:]) == 0
    assert ndiff(ref.array("LHS"), s.get("LHS")) == 0
    ref.boundary(1)
    s.residual_stage(1, 2, capi.Solver.STAGE_BOUNDARY)
    assert ndiff(ref.array("R")[4:], s.get("R")[4:]) == 0
    assert ndiff(ref.array("LHS"), s.get("LHS")) == 0
    assert ndiff(ref.array("xn_bedges")[3:], s.get("xn_bedges")[3:]) == 0
    assert ndiff(ref.array("nQ")[4:], s.get("nQ")[4:]) == 0
    # the linear solve from the caller's LHS and RHS (LU factors formed anew)
    ref.set_array("RHS", -ref.array("R"))
    ref.set_array("dQ", np.zeros_like(ref.array("dQ")))
    s.set("LHS", ref.array("LHS"))
    s.set("RHS", ref.array("RHS"))
    r_ref = ref.linear_solve()
    r_gpu = s.linear_solve()
    assert ndiff(ref.array("dQ")[4:], s.get("dQ")[4:]) == 0
    assert r_gpu == pytest.approx(r_ref, rel=RMS_RTOL)
    assert s.get("cfl")[0] == ref.cfl()
    assert s.status() == 0
    s.close()
    mesh.close()
    ref.close()
