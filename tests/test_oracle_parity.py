"""The C restatement (oracle/flow_oracle.c) against the reference compiled from
its own sources (oracle/_ref): bit-for-bit on every array of several steps,
for k=1 (linear walls) and k=2 (curved NACA walls).  CPU only."""
import numpy as np
import pytest

from cases import ParityCase, ndiff
from oracle import port


@pytest.mark.parametrize("nc,nr,curved,order,steps,quads,mach", [
    (32, 8, False, 1, 8, False, None),
    (32, 8, True, 3, 8, False, None),
    (64, 16, True, 3, 4, False, None),
    (64, 16, False, 1, 4, False, None),
    (64, 16, False, 3, 6, False, 0.5),  # k=2 with straight walls
    (64, 16, False, 1, 6, True, None),  # quadrilateral meshes
    (64, 16, False, 3, 6, True, None),
    (64, 16, False, 1, 5, "mixed", None),  # quadrilaterals inside, triangles outside
    (64, 16, False, 3, 5, "mixed", None),
    (8, 3, False, 1, 6, False, None),   # 24 nodes: smaller than one CTA of the node kernels
    (12, 4, True, 3, 6, False, None),   # 48 nodes, k=2 (8x3 is too small for the k=2 stencils)
])
def test_oracle_matches_reference(ref_lib, nc, nr, curved, order, steps, quads, mach):
    _oracle_steps(ParityCase(nc, nr, curved, order, quads=quads, mach=mach), steps)


@pytest.mark.parametrize("order", [1, 3])
def test_oracle_matches_reference_on_a_circular_wall(ref_lib, order):
    """Triangles around the unit circle: the reference's curved wall bc 11."""
    _oracle_steps(ParityCase(48, 12, True, order, cylinder=True), 6)


@pytest.mark.parametrize("curved,order,params", [
    (True, 3, {"iter": 3, "jufreq": 2}),  # Newton iterations, Jacobian every 2nd
    (False, 1, {"reorder": 0}),           # no Cuthill-McKee renumbering
    (True, 3, {"subits": 3}),             # an odd number of sweeps
    (True, 3, {"limit": 0}),              # no limiter
    (False, 1, {"limit": 0}),
])
def test_oracle_matches_reference_parameter_variants(ref_lib, curved, order, params):
    _oracle_steps(ParityCase(32, 8, curved, order, **params), 6)


@pytest.mark.parametrize("curved,order,foits,soits", [
    (True, 3, 3, 0), (False, 1, 3, 0),
    (True, 3, 0, 3), (True, 3, 2, 2),  # k=2 after second-order start-up steps
])
def test_oracle_matches_reference_after_start_up_steps(ref_lib, curved, order, foits, soits):
    """foits first-order steps (and soits second-order ones for k=2), then
    the scheme of the order."""
    from cases import startup_parity_case
    _oracle_steps(startup_parity_case(32, 8, curved, order, foits, soits), 7)


def _oracle_steps(case, steps):
    og = port.OracleGrid(case.sizes, case.arrays)
    p = port.params_from_flow(case.fp)
    nn = case.sizes["nn"]
    for ts in range(1, steps + 1):
        case.ref_step()
        dq = og.solve(p, ts)
        ref = case.ref
        for name in ("LHS", "xn_bedges"):
            assert ndiff(ref.array(name), og[name]) == 0, (name, ts)
        for name in ("Q", "nQ", "pQ"):  # entry 0 is unused (and uninitialised) in the reference
            assert ndiff(ref.array(name)[4:], og[name][4:]) == 0, (name, ts)
        for name in ("R", "dQ", "phi", "grad", "hess"):
            a, b = ref.array(name), og[name]
            w = a.size // (nn + 1)
            assert ndiff(a[w:], b[w:]) == 0, (name, ts)
        assert og.body_forces(p) == ref.body_forces()
        if ts == 1:
            assert dq == case.dq1


def test_stage_functions_match(ref_lib):
    """build_matrix, limiter and residual stages one by one (k=1)."""
    case = ParityCase(32, 8, False, 1)
    og = port.OracleGrid(case.sizes, case.arrays)
    p = port.params_from_flow(case.fp)
    ref = case.ref
    # bring both to the reference's state after step 1, then run stage by stage
    og.set("Q", ref.array("Q")); og.set("nQ", ref.array("nQ"))
    ref.set_citer(2); og.g.citer = 2
    ref.build_matrix(); og.build_matrix(p)
    assert ndiff(ref.array("LHS"), og["LHS"]) == 0
    assert ndiff(ref.array("dt")[1:], og["dt"][1:]) == 0
    ref.gradient(); og.gradient()
    assert ndiff(ref.array("grad")[8:], og["grad"][8:]) == 0
    ref.limiter(); og.limiter(p)
    assert ndiff(ref.array("phi")[8:], og["phi"][8:]) == 0
    ref.interior(1, 2); og.interior(p, 1, 2)
    ref.boundary(1); og.boundary(p, 1)
    assert ndiff(ref.array("R")[4:], og["R"][4:]) == 0
    assert ndiff(ref.array("LHS"), og["LHS"]) == 0
    rhs = -ref.array("R")
    ref.set_array("RHS", rhs); og.set("RHS", rhs)
    ref.set_array("dQ", np.zeros_like(ref.array("dQ"))); og.set("dQ", np.zeros_like(og["dQ"]))
    r1 = ref.linear_solve(); r2 = og.linear_solve(p)
    assert ndiff(ref.array("dQ")[4:], og["dQ"][4:]) == 0
    assert r1 == r2


def test_roe_flux_consistency():
    """Roe_flux_centered(q, q) is the physical Euler flux (flux.C:537-538)."""
    rng = np.random.default_rng(0)
    for _ in range(50):
        rho = rng.uniform(0.5, 2.0); u, v = rng.uniform(-1, 1, 2); p = rng.uniform(0.3, 2.0)
        E = p / 0.4 + 0.5 * rho * (u * u + v * v)
        q = np.array([rho, rho * u, rho * v, E])
        th = rng.uniform(0, 2 * np.pi); nx, ny = np.cos(th), np.sin(th); L = rng.uniform(0.1, 2)
        f = port.roe_flux(nx, ny, L, 1.4, q, q)
        un = u * nx + v * ny
        ref = np.array([rho * un, rho * u * un + p * nx, rho * v * un + p * ny, un * (E + p)]) * L
        assert np.allclose(f, ref, rtol=1e-13, atol=1e-14)
