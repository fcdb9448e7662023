"""The kernel variants the autotuner chooses between give bit-identical
iterates, and autotuning leaves the solution state as it found it."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,order", [(0, 3), (3, 3), (0, 1), (3, 1)])
def test_variants_are_bit_identical_and_autotune_restores_state(precision, order):
    """Variant 3 of the node kernel is the shared-memory-staged one, 4 the
    16-lane one, 5-7 variants 0, 1 and 4 with the limiter that divides no
    zero and by no zero."""
    from flowgpu import capi, workloads
    from flowgpu.prep import Mesh
    wl = workloads.Workload("tune", 64, 16, order == 3, order, 0.8 if order == 3 else 0.5,
                            subits=2 if precision == 0 else 4)
    mesh = Mesh.from_case(wl.write(), order=order)
    fp = wl.params()
    runs = []
    for v in [(0, 0), (1, 1), (2, 2), (3, 0), (4, 2), (5, 0), (6, 1), (7, 0), None]:
        s = capi.Solver.from_mesh(mesh, fp, device=0)
        s.set_precision(precision)
        s.set_state(mesh.initial_state(fp))
        s.run(1, 3)
        if v is None:
            q_before = s.get("Q")
            chosen, ms = s.autotune(ts=4, steps=2)
            assert 0 <= chosen[0] <= 7 and 0 <= chosen[1] <= 2 and all(t > 0 for t in ms)
            assert ms[3] < 1e30  # the staged kernel fits this mesh and was timed
            assert np.array_equal(q_before, s.get("Q"))
        else:
            s.set_variants(*v)
        rh, dh = s.run(4, 5)
        runs.append((s.get("Q"), list(rh)))
        assert s.status() == 0
        s.close()
    for q, rh in runs[1:]:
        assert np.array_equal(q, runs[0][0]) and rh == runs[0][1]


@pytest.mark.parametrize("allow_df", [False, True])
def test_sweep_shape_autotune_restores_state_and_keeps_the_iterates(allow_df):
    """flow_autotune_sweep times the mode 3 sweep shapes (ring of 64/32/16-row
    sub-levels; one launch per sweep when allowed), keeps the fastest, and
    leaves the state as it was; the steps after it are those of the default
    shape, bit for bit."""
    from flowgpu import capi, workloads
    from flowgpu.prep import Mesh
    wl = workloads.Workload("tunesweep", 96, 24, True, 3, 0.8, subits=4)
    mesh = Mesh.from_case(wl.write(), order=3)
    fp = wl.params()
    runs = []
    for tune in (False, True):
        s = capi.Solver.from_mesh(mesh, fp, device=0)
        s.set_precision(3)
        s.set_state(mesh.initial_state(fp))
        s.run(1, 3)
        if tune:
            q_before = s.get("Q")
            choice, ms = s.autotune_sweep(ts=4, steps=2, allow_df=allow_df)
            assert choice % 1000 in (64, 32, 16) and (allow_df or choice < 1000)
            assert ms[0] < 1e30 and (allow_df or ms[3] == 1e30)
            assert np.array_equal(q_before, s.get("Q"))
        rh, _ = s.run(4, 5)
        runs.append((s.get("Q"), list(rh)))
        assert s.status() == 0
        s.close()
    assert np.array_equal(runs[0][0], runs[1][0]) and runs[0][1] == runs[1][1]
