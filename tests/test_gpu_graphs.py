"""Chunks of steps replayed from CUDA graphs (step index and CFL ramp on the
device) give the same iterates, bit for bit, as steps launched one by one,
in the FP64 drop-in and in the precision form."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,order,subits", [(0, 3, 2), (1, 3, 4), (0, 1, 2), (1, 1, 3),
                                                    (2, 3, 2), (2, 1, 3), (3, 3, 4), (3, 1, 3)])
def test_graph_chunks_match_eager_steps(precision, order, subits):
    from flowgpu import capi, workloads
    from flowgpu.prep import Mesh
    wl = workloads.Workload("graphs", 64, 16, order == 3, order, 0.8 if order == 3 else 0.5,
                            subits=subits)
    mesh = Mesh.from_case(wl.write(), order=order)
    fp = wl.params()
    out = []
    for graphs in (False, True):
        s = capi.Solver.from_mesh(mesh, fp, device=0)
        s.set_precision(precision)
        s.set_graphs(graphs)
        s.set_state(mesh.initial_state(fp))
        steps, r0, r1 = s.converge(1, 300, 1e-10, chunk=16, check=False)
        out.append((steps, r0, r1, s.get("Q"), s.get("dQ"), s.body_forces(), s.status()))
        s.close()
    (n0, a0, b0, q0, d0, f0, st0), (n1, a1, b1, q1, d1, f1, st1) = out
    assert st0 == st1 and (st0 == 0 or st0 == 256)
    assert n0 == n1 and a0 == a1 and b0 == b1
    assert np.array_equal(q0, q1) and np.array_equal(d0, d1)
    assert f0 == f1


@pytest.mark.parametrize("precision", [0, 3])
def test_failed_capture_falls_back_to_eager_launches(precision):
    """A chunk whose graph capture fails (here discarded on purpose through
    the host-side hook flow_set_capture_fault) is launched kernel by kernel
    instead: the iterates are those of the run whose captures succeed, and
    the fallback is counted."""
    from flowgpu import capi, workloads
    from flowgpu.prep import Mesh
    wl = workloads.Workload("capfault", 64, 16, True, 3, 0.8, subits=4 if precision else 2)
    mesh = Mesh.from_case(wl.write(), order=3)
    fp = wl.params()
    out = []
    for faults in (0, 3):
        s = capi.Solver.from_mesh(mesh, fp, device=0)
        s.set_precision(precision)
        s.set_state(mesh.initial_state(fp))
        s.set_capture_fault(faults)
        steps, r0, r1 = s.converge(1, 200, 1e-10, chunk=16, check=False)
        out.append((steps, r0, r1, s.get("Q"), s.body_forces(), s.status(),
                    s.capture_fallbacks()))
        s.close()
    (n0, a0, b0, q0, f0, st0, fb0), (n1, a1, b1, q1, f1, st1, fb1) = out
    assert fb0 == 0 and fb1 == 3
    assert st0 == st1 and n0 == n1 and a0 == a1 and b0 == b1
    assert np.array_equal(q0, q1) and f0 == f1
