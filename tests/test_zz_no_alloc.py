"""flow_linear_residual_noalloc: the b - A x RMS of a caller-held BCSR system,
computed in a static __device__ scratch array with no device allocation.

Its result is checked against the RMS that flow_linear_solve (the context
entry point, whose scratch the context allocates) returns for the same
matrix, right-hand side and dQ, on several calls in a row: a large system, a
smaller one (stale scratch rows of the first call must not leak in), then the
first again.  This file runs last so that it is exercised both alone and
after every other GPU test in the same process.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1e-12  # the tests' tolerance for reductions whose order may differ


def _system(nc, nr, order):
    """A Jacobian system of pseudo-time step 2, solved by flow_linear_solve."""
    from flowgpu import capi, workloads
    from flowgpu.prep import Mesh
    wl = workloads.Workload(f"noalloc{nc}x{nr}", nc, nr, True, order, 0.8)
    mesh = Mesh.from_case(wl.write(), order=order)
    p = wl.params()
    s = capi.Solver.from_mesh(mesh, p, device=0)
    s.set_state(mesh.initial_state(p))
    s.solve(1)
    s.build_matrix(2)
    s.reconstruct(2)
    s.residuals(1, 2)
    rms = s.linear_solve()
    nn = mesh.sizes["nn"]
    out = {"nn": nn, "rms": rms, "ia": mesh.array("ia").astype(np.int32),
           "ja": mesh.array("ja").astype(np.int32), "LHS": s.get("LHS"),
           "RHS": s.get("RHS"), "dQ": s.get("dQ")}
    s.close()
    mesh.close()
    return out


def _on_device(sysd):
    """The system's arrays in the caller's own device memory (torch's)."""
    import torch
    dev = torch.device("cuda", 0)
    t = {k: torch.from_numpy(sysd[k]).to(dev) for k in ("ia", "ja", "LHS", "RHS", "dQ")}
    torch.cuda.synchronize()
    return t


def _noalloc(sysd, t):
    import torch
    from flowgpu import capi
    nnz = int(sysd["ia"][sysd["nn"] + 1])
    stream = torch.cuda.current_stream(torch.device("cuda", 0)).cuda_stream
    return capi.linear_residual_noalloc(t["ia"].data_ptr(), t["ja"].data_ptr(),
                                        t["LHS"].data_ptr(), t["RHS"].data_ptr(),
                                        t["dQ"].data_ptr(), sysd["nn"], nnz, stream)


def test_noalloc_residual_matches_linear_solve_on_calls_in_a_row():
    import torch
    torch.cuda.set_device(0)
    big = _system(64, 16, 3)
    small = _system(32, 8, 1)
    assert big["nn"] > small["nn"]
    tb, ts = _on_device(big), _on_device(small)
    # the first call loads the module (a one-time set-up); from then on the
    # calls take no device memory: neither the device's free bytes nor
    # torch's allocated bytes move
    first = _noalloc(big, tb)
    assert first == pytest.approx(big["rms"], rel=RTOL, abs=0.)
    torch.cuda.synchronize()
    free0, alloc0 = torch.cuda.mem_get_info(0)[0], torch.cuda.memory_allocated(0)
    for sysd, t in ((big, tb), (small, ts), (big, tb)):
        got = _noalloc(sysd, t)
        assert np.isfinite(got) and got > 0.
        assert got == pytest.approx(sysd["rms"], rel=RTOL, abs=0.)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(0)[0] == free0
    assert torch.cuda.memory_allocated(0) == alloc0


def test_noalloc_rejects_rows_beyond_the_scratch():
    import torch
    from flowgpu import capi
    torch.cuda.set_device(0)
    buf = torch.zeros(64, dtype=torch.float64, device="cuda")
    p = buf.data_ptr()
    with pytest.raises(capi.FlowError) as ei:
        capi.linear_residual_noalloc(p, p, p, p, p, capi.NOALLOC_MAX_ROWS + 1, 0)
    assert "static scratch" in str(ei.value)
