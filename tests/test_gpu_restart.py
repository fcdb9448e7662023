"""Restart files on the GPU: after the same steps the library's
flow_write_restart writes the bytes of the reference's write_mesh, and a
solve resumed from that file (flow_prep_read + flow_prep_restart_state, then
steps citer+1 ...) matches the reference's resumed solve bit for bit."""
import os

import numpy as np
import pytest

from cases import ParityCase, ndiff
from test_restart import restart_case

pytestmark = pytest.mark.gpu


class _RefMesh:
    """The reference's connectivity and boundaries in the shape the library's
    writers take (Mesh.elements / segments / array)."""

    def __init__(self, ref):
        self.ref = ref
        self.x = ref.array("x")

    def array(self, name):
        return self.x

    def elements(self):
        quad = self.ref.array("c2n_quad")
        return self.ref.array("c2n_tri"), quad if quad.size else np.zeros(4, dtype=np.int32)

    def segments(self):
        segs = self.ref.segments()
        bbc = self.ref.array("bbc")
        nbs = np.array([0] + [len(s) for s in segs], dtype=np.int32)
        seg = np.array([n for s in segs for pair in s for n in pair], dtype=np.int32)
        return len(segs), bbc, nbs, seg


@pytest.mark.parametrize("curved,order", [(False, 1), (True, 3)])
def test_restart_file_matches_the_reference(ref_lib, curved, order, tmp_path):
    from flowgpu.capi import Solver
    case = ParityCase(32, 8, curved, order)
    gpu = Solver(case.sizes, case.arrays, case.fp, device=0)
    gpu.set_state(case.Q0)
    for ts in (1, 2, 3):
        gpu.solve(ts)
    d, fp = restart_case(case, 3, str(tmp_path / "restart"))
    mine = str(tmp_path / "mine.mesh")
    gpu.write_restart(_RefMesh(case.ref), mine)
    with open(mine, "rb") as a, open(os.path.join(d, "grid.mesh"), "rb") as b:
        assert a.read() == b.read()
    gpu.close()


def test_resumed_solve_matches_the_reference(ref_lib, tmp_path):
    """k=1: both resume from the same restart file (the reference re-reads
    it with isrestart = 1, its step loop going on at citer + 1)."""
    from flowgpu.capi import Solver
    from flowgpu.prep import Mesh
    case = ParityCase(32, 8, False, 1)
    d, fp = restart_case(case, 3, str(tmp_path / "restart"))
    ref2 = ref_lib.RefSolver(d)
    m = Mesh.from_case(d, order=1, reorder=0)
    Q, citer, _ = m.restart_state()
    gpu = Solver.from_mesh(m, case.fp, device=0)
    gpu.set_state(Q)
    for ts in range(citer + 1, citer + 5):
        ref2.solve(ts)
        gpu.solve(ts)
        assert ndiff(ref2.array("Q")[4:], gpu.get("Q")[4:]) == 0, ts
        assert ndiff(ref2.array("LHS"), gpu.get("LHS")) == 0, ts
    assert gpu.status() == 0
    gpu.close()
    m.close()
    ref2.close()
