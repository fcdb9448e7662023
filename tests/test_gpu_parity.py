"""GPU parity: the CUDA library (through its C ABI) against the reference
solver compiled from its own sources (oracle/_ref), step by step.

Bar: bit-for-bit equality of every array the reference's solve() produces
(Q, R, LHS, dQ, phi, grad/hess, point values, the mutated boundary normals)
and of the lift/drag forces; the step norm ||dQ|| is reduced in a different
order on the GPU, so it is compared to 1e-12 relative."""
import numpy as np
import pytest

from cases import ParityCase, ndiff

pytestmark = pytest.mark.gpu


def _solver(case, sweep_mode=0):
    from flowgpu.capi import Solver
    s = Solver(case.sizes, case.arrays, case.fp, device=0)
    s.set_sweep_mode(sweep_mode)
    s.set_state(case.Q0)
    return s


@pytest.mark.parametrize("nc,nr,curved,order,steps,mode,quads,mach", [
    (32, 8, False, 1, 6, 0, False, None),
    (128, 32, False, 1, 4, 0, False, None),
    (32, 8, True, 3, 6, 0, False, None),
    (128, 32, True, 3, 4, 0, False, None),
    (128, 32, True, 3, 3, 1, False, None),
    (64, 16, False, 1, 3, 1, False, None),
    (64, 16, False, 3, 4, 0, False, 0.5),  # k=2 with straight walls
    (64, 16, False, 1, 4, 0, True, None),  # quadrilateral meshes
    (64, 16, False, 3, 4, 0, True, None),
    (64, 16, False, 1, 4, 0, "mixed", None),  # quadrilaterals inside, triangles outside
    (64, 16, False, 3, 4, 0, "mixed", None),
    (8, 3, False, 1, 6, 0, False, None),  # 24 nodes: smaller than one CTA of the node kernels
    (8, 3, False, 1, 4, 1, False, None),
    (12, 4, True, 3, 6, 0, False, None),  # 48 nodes, k=2 (8x3 is too small for the k=2 stencils)
])
def test_steps_bitwise(ref_lib, nc, nr, curved, order, steps, mode, quads, mach):
    """mode 0: grid-wide ordered sweep; mode 1: one-CTA ordered sweep."""
    _steps_bitwise(ParityCase(nc, nr, curved, order, quads=quads, mach=mach), steps, mode)


@pytest.mark.parametrize("order", [1, 3])
def test_steps_on_a_circular_wall_bitwise(ref_lib, order):
    """Triangles around the unit circle: the reference's curved wall bc 11."""
    _steps_bitwise(ParityCase(48, 12, True, order, cylinder=True), 5, 0)


@pytest.mark.parametrize("curved,order,params", [
    (True, 3, {"iter": 3, "jufreq": 2}),  # Newton iterations, Jacobian every 2nd
    (False, 1, {"reorder": 0}),           # no Cuthill-McKee renumbering
    (True, 3, {"subits": 3}),             # an odd number of sweeps
    (True, 3, {"limit": 0}),              # no limiter
    (False, 1, {"limit": 0}),
])
def test_parameter_variants_bitwise(ref_lib, curved, order, params):
    _steps_bitwise(ParityCase(32, 8, curved, order, **params), 5, 0)


@pytest.mark.parametrize("curved,order,foits,soits", [
    (True, 3, 3, 0), (False, 1, 3, 0),
    (True, 3, 0, 3), (True, 3, 2, 2),  # k=2 after second-order start-up steps
])
def test_steps_after_start_up_steps_bitwise(ref_lib, curved, order, foits, soits):
    """foits first-order steps (and soits second-order ones for k=2), then
    the scheme of the order."""
    from cases import startup_parity_case
    _steps_bitwise(startup_parity_case(32, 8, curved, order, foits, soits), 7, 0)


def _steps_bitwise(case, steps, mode):
    order = case.fp.order
    gpu = _solver(case, mode)
    nn = case.sizes["nn"]
    for ts in range(1, steps + 1):
        case.ref_step()
        dq, rr = gpu.solve(ts)
        ref = case.ref
        for name in ("LHS", "xn_bedges"):
            assert ndiff(ref.array(name), gpu.get(name)) == 0, (name, ts)
        for name in ("Q", "nQ", "pQ"):  # entry 0 is unused (and uninitialised) in the reference
            assert ndiff(ref.array(name)[4:], gpu.get(name)[4:]) == 0, (name, ts)
        for name in ("R", "dQ", "phi", "grad"):
            a, b = ref.array(name), gpu.get(name)
            w = a.size // (nn + 1)
            assert ndiff(a[w:], b[w:]) == 0, (name, ts)
        if order == 3:
            a, b = ref.array("hess"), gpu.get("hess")
            a = a.reshape(-1, 4, 9)[1:, :, :5]
            b = b.reshape(-1, 4, 9)[1:, :, :5]
            assert ndiff(a, b) == 0, ("hess", ts)
            pv = ref.array("point_value")  # allocated at the reference's first k=2 step
            if pv.size:
                assert ndiff(pv[4:], gpu.get("point_value")[4:]) == 0, ("point_value", ts)
        if ts > 1:
            R = ref.array("R").reshape(-1, 4)[1:, 0]
            assert rr == pytest.approx(np.sqrt((R * R).sum()), rel=1e-12)
        assert gpu.body_forces() == ref.body_forces()
    assert gpu.status() == 0


def test_transonic_k2_at_full_size_bitwise(ref_lib):
    """The plain drop-in check at its own size: 512 x 128 O-grid (65,536
    nodes), k=2, M 0.8, curved NACA walls (the curved boundary path of
    residual.C:1103-1143 and the k=2 derivatives of
    compute_derivatives.C:1438-1534), three steps bit for bit."""
    _steps_bitwise(ParityCase(512, 128, True, 3, mach=0.8), 3, 0)


@pytest.mark.parametrize("nc,nr,curved,order,mach,steps", [
    (128, 32, False, 1, 0.5, 300),   # the k=1 case: 128 x 32, M 0.5
    (128, 32, True, 3, 0.8, 200),    # k=2, curved walls, M 0.8
])
def test_long_residual_history(ref_lib, nc, nr, curved, order, mach, steps):
    """The drop-in reproduces the reference's residual-drop history: every
    step's ||R_rho|| over a long run (the GPU forms the norm as a tree
    reduction: 1e-12 relative), and the state after the last step bit for
    bit (so every step's sweeps took the reference's path, including the
    b - Ax RMS test of linear_algebra.C:348-387)."""
    case = ParityCase(nc, nr, curved, order, mach=mach)
    gpu = _solver(case)
    r_gpu, _dq = gpu.run(1, steps)
    r_ref = []
    for ts in range(1, steps + 1):
        case.ref_step()
        R = case.ref.array("R").reshape(-1, 4)[1:, 0]
        r_ref.append(np.sqrt((R * R).sum()))
    r_ref = np.asarray(r_ref)
    np.testing.assert_allclose(np.asarray(r_gpu), r_ref, rtol=1e-12, atol=0.)
    assert r_ref[-1] < r_ref[0]  # the history falls
    assert ndiff(case.ref.array("Q")[4:], gpu.get("Q")[4:]) == 0
    assert gpu.body_forces() == case.ref.body_forces()
    assert gpu.status() == 0


@pytest.mark.parametrize("nc,nr,curved,order,steps", [
    (128, 32, False, 1, 4), (128, 32, True, 3, 4), (12, 4, True, 3, 4), (8, 3, False, 1, 4),
])
@pytest.mark.parametrize("variant", [3, 4, 5, 6, 7])
def test_node_kernel_variants_bitwise(ref_lib, nc, nr, curved, order, steps, variant):
    """Node variant 3 (gathers staged in shared memory), 4 (16 lanes a node),
    5-7 (variants 0, 1 and 4 with the limiter that divides no zero and by no
    zero), step by step against the reference, including meshes smaller than one
    tile of 32 nodes."""
    case = ParityCase(nc, nr, curved, order)
    gpu = _solver(case)
    gpu.set_variants(variant, 0)
    nn = case.sizes["nn"]
    for ts in range(1, steps + 1):
        case.ref_step()
        gpu.solve(ts)
        assert ndiff(case.ref.array("Q")[4:], gpu.get("Q")[4:]) == 0, ts
        for name in ("phi", "grad"):
            a, b = case.ref.array(name), gpu.get(name)
            w = a.size // (nn + 1)
            assert ndiff(a[w:], b[w:]) == 0, (name, ts)
        assert ndiff(case.ref.array("LHS"), gpu.get("LHS")) == 0, ts
    assert gpu.status() == 0
