"""Restart files on the CPU: a restart written by the reference's own
write_mesh (mesh_io.C:300-393) is read back by the library's preprocessing
(flow_prep_read + flow_prep_restart_state) into the state, step and CFL the
reference reads with isrestart = 1 (mesh_io.C:217-262, ic.C:84-96)."""
import os
import shutil

import numpy as np
import pytest

from cases import ParityCase


def restart_case(case, steps, d):
    """Run the reference `steps` steps, write its restart file into a new
    case directory set up for a restart (isrestart = 1); returns the dir."""
    from flowgpu import meshgen
    for _ in range(steps):  # the first call books step 1, run at set-up
        case.ref_step()
    os.makedirs(d, exist_ok=True)
    case.ref.write_mesh(os.path.join(d, "grid.mesh"))
    shutil.copy(os.path.join(case.dir, "bc.dat"), os.path.join(d, "bc.dat"))
    fp = meshgen.FlowParams(**{k: getattr(case.fp, k) for k in meshgen.FlowParams.FIELDS})
    fp.isrestart = 1
    meshgen.write_params(os.path.join(d, "euler.params"), fp)
    return d, fp


@pytest.mark.parametrize("curved,order", [(False, 1), (True, 3)])
def test_restart_block_reads_back_as_the_reference_reads_it(ref_lib, curved, order, tmp_path):
    from flowgpu.prep import Mesh
    case = ParityCase(32, 8, curved, order)
    d, fp = restart_case(case, 3, str(tmp_path / "restart"))
    ref2 = ref_lib.RefSolver(d)  # the reference's own restart set-up
    m = Mesh.from_case(d, order=order, reorder=0)
    Q, citer, cfl = m.restart_state()
    assert citer == 3 and cfl == case.ref.cfl()
    assert np.array_equal(Q[4:], ref2.array("Q")[4:])
    assert np.array_equal(m.array("x")[2:], ref2.array("x")[2:])
    m.close()
    ref2.close()


def test_mesh_without_restart_block(tmp_path):
    from flowgpu import workloads
    from flowgpu.prep import Mesh
    wl = workloads.Workload("norestart", 32, 8, False, 1, 0.5)
    m = Mesh.from_case(wl.write(str(tmp_path)), order=1)
    assert m.restart_state() is None
    m.close()
