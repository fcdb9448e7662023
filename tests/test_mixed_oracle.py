"""The oracle's precision-form pieces on the CPU: the greedy colouring is a
proper colouring of the block pattern, and the multicolour FP32 solve drives
the nonlinear residual down like the FP64 one."""
import numpy as np
import pytest


def _grid(nc, nr, curved, order):
    from flowgpu import workloads
    from flowgpu.prep import Mesh
    from oracle import port
    wl = workloads.Workload(f"orc{nc}x{nr}", nc, nr, curved, order, 0.8 if order == 3 else 0.5,
                            subits=4)
    mesh = Mesh.from_case(wl.write(), order=order)
    fp = wl.params()
    og = port.OracleGrid(mesh.sizes, mesh.arrays())
    og.set("Q", mesh.initial_state(fp))
    return mesh, og, port.params_from_flow(fp)


def test_greedy_colouring_is_proper():
    mesh, og, _ = _grid(64, 16, True, 3)
    col, nc = og.colors()
    ia, ja = og["ia"], og["ja"]
    nn = mesh.sizes["nn"]
    assert 3 <= nc <= 12
    for j in range(1, nn + 1):
        for k in range(ia[j], ia[j + 1]):
            c = ja[k]
            if c != j:
                assert col[c] != col[j]
            # greedy: colour is the smallest not held by an earlier neighbour
        earlier = {col[ja[k]] for k in range(ia[j], ia[j + 1]) if ja[k] < j}
        assert col[j] == min(set(range(nc + 1)) - earlier)


@pytest.mark.parametrize("approx", [0, 1])
def test_mixed_solve_reduces_the_residual(approx):
    """With the forward-difference face Jacobians and with the approximate
    Roe ones rounded to FP32 (jac_approx)."""
    mesh, og, p = _grid(32, 8, True, 3)
    p.jac_approx = approx
    nn = mesh.sizes["nn"]
    norms = []
    for ts in range(1, 41):
        og.solve_mixed(p, ts)
        R = og["R"].reshape(-1, 4)[1:nn + 1, 0]
        norms.append(float(np.sqrt((R * R).sum())))
    assert np.all(np.isfinite(norms))
    assert norms[-1] < 1e-3 * norms[0]
