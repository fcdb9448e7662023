"""The CUDA path, fed by the library's own preprocessing of the stored mesh,
reproduces the golden vectors recorded from the reference (bit for bit; the
step norm ||dQ|| is reduced in another order on the GPU: 1e-12 relative)."""
import numpy as np
import pytest

from test_golden import CASES, load_case, params_of

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("name", CASES)
def test_gpu_reproduces_golden(name, mode, tmp_path):
    from flowgpu.capi import Solver
    from flowgpu.prep import Mesh
    z, d = load_case(name, tmp_path)
    fp = params_of(d)
    mesh = Mesh.from_case(d, order=int(z["order"]))
    nn = mesh.sizes["nn"]
    s = Solver.from_mesh(mesh, fp, device=0)
    s.set_sweep_mode(mode)
    s.set_state(mesh.initial_state(fp))
    iau = mesh.array("iau")
    for ts in range(1, int(z["steps"]) + 1):
        dq, _ = s.solve(ts)
        assert np.array_equal(s.get("R")[4:].reshape(nn, 4), z["R"][ts - 1]), ts
        assert np.array_equal(s.get("dQ")[4:].reshape(nn, 4), z["dQ"][ts - 1]), ts
        assert dq == pytest.approx(z["dq_norm"][ts - 1], rel=1e-12)
        assert s.body_forces() == tuple(z["forces"][ts - 1])
        if ts == 1:
            L = s.get("LHS").reshape(-1, 16)
            assert np.array_equal(L[iau[1:nn + 1]], z["diag1"])
    assert np.array_equal(s.get("Q")[4:].reshape(-1, 4), z["Q"])
    assert s.status() == 0


def test_converge_restarts_identically(tmp_path):
    """flow_set_state starts a fresh solve: two runs to the same drop take the
    same number of steps and end in the same state (the curved-wall normals
    rewritten by the k=2 boundary pass are reset too)."""
    from flowgpu.capi import Solver
    from flowgpu.prep import Mesh
    z, d = load_case("ogrid32x8_k2", tmp_path)
    fp = params_of(d)
    mesh = Mesh.from_case(d, order=3)
    s = Solver.from_mesh(mesh, fp, device=0)
    Q0 = mesh.initial_state(fp)
    out = []
    for _ in range(2):
        s.set_state(Q0)
        n, r0, r1 = s.converge(1, 5000, 1e-6)
        out.append((n, s.get("Q"), s.body_forces()))
    assert out[0][0] == out[1][0]
    assert np.array_equal(out[0][1], out[1][1])
    assert out[0][2] == out[1][2]
