"""Failure detection on the GPU without a fault: a sweep whose first row is
never computed makes its dependents' bounded waits run out; the kernel
reports FLOW_ERR_SWEEP_TIMEOUT and ends, and the context goes on to give
the same next step as a context that never ran the test."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_sweep_wait_runs_out_and_the_context_stays_usable():
    from flowgpu import capi, workloads
    from flowgpu.prep import Mesh
    wl = workloads.Workload("selftest", 64, 16, True, 3, 0.8)
    mesh = Mesh.from_case(wl.write(), order=3)
    fp = wl.params()
    a = capi.Solver.from_mesh(mesh, fp, device=0)
    b = capi.Solver.from_mesh(mesh, fp, device=0)
    for s in (a, b):
        s.set_state(mesh.initial_state(fp))
        s.solve(1)
    st = a.selftest_sweep_timeout(max_spin=4096)
    assert st & capi.ERR_SWEEP_TIMEOUT
    assert a.status() == 0
    a.solve(2)
    b.solve(2)
    assert a.status() == 0 and b.status() == 0
    assert np.array_equal(a.get("Q"), b.get("Q"))
    a.close()
    b.close()
