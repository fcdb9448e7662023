"""The kernel variants the autotuner chooses between give bit-identical
iterates, and autotuning leaves the solution state as it found it."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [0, 3])
def test_variants_are_bit_identical_and_autotune_restores_state(precision):
    from flowgpu import capi, workloads
    from flowgpu.prep import Mesh
    wl = workloads.Workload("tune", 64, 16, True, 3, 0.8, subits=2 if precision == 0 else 4)
    mesh = Mesh.from_case(wl.write(), order=3)
    fp = wl.params()
    runs = []
    for v in [(0, 0), (1, 1), (2, 2), None]:
        s = capi.Solver.from_mesh(mesh, fp, device=0)
        s.set_precision(precision)
        s.set_state(mesh.initial_state(fp))
        s.run(1, 3)
        if v is None:
            q_before = s.get("Q")
            chosen, ms = s.autotune(ts=4, steps=2)
            assert all(0 <= x <= 2 for x in chosen) and all(t > 0 for t in ms)
            assert np.array_equal(q_before, s.get("Q"))
        else:
            s.set_variants(*v)
        rh, dh = s.run(4, 5)
        runs.append((s.get("Q"), list(rh)))
        assert s.status() == 0
        s.close()
    for q, rh in runs[1:]:
        assert np.array_equal(q, runs[0][0]) and rh == runs[0][1]
