"""The reference's own driver (main.C, unmodified) over the shims and
libflowgpu.so, against the reference as shipped.  oracle/build_ref_exe.sh
builds the executables from the reference's sources:
* field_solver_gpu: solve() replaced whole (flow-solver_b200/shim/solve_gpu.C);
* field_solver_stages: the reference's own solve() with build_matrix,
  build_interior_residuals, build_boundary_residuals and linear_solve
  replaced (flow-solver_b200/shim/stages_gpu.C).
Each runs the same case (k=1 straight walls, k=2 curved walls) for 8
pseudo-time steps in its own directory, and every file the run writes is
compared:
* residuals.dat holds the step norm ||dQ|| that solve() returns, which the
  GPU reduces in a different order: compared to 1e-12 relative;
* time.dat holds wall-clock times: only its presence is compared;
* every other file (surface pressure, body forces, the Tecplot and restart
  files the reference's writers make from the state the shim copies back,
  the command file) byte for byte.
Both runs end the way the reference's own run ends (its teardown frees an
array twice after every file is written): the return codes are compared."""
import os
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

from cases import make_case

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_EXE = os.path.join(ROOT, "oracle", "_ref", "field_solver")
GPU_EXES = {"whole": os.path.join(ROOT, "oracle", "_ref", "field_solver_gpu"),
            "stages": os.path.join(ROOT, "oracle", "_ref", "field_solver_stages")}
NORM_RTOL = 1e-12


def _run(exe, case_dir):
    work = tempfile.mkdtemp(prefix="exe_")
    shutil.rmtree(work)
    shutil.copytree(case_dir, work)
    r = subprocess.run([exe, "grid.mesh"], cwd=work, capture_output=True, text=True, timeout=300)
    return r, work


def _numbers_close(a, b):
    ta, tb = a.split(), b.split()
    assert len(ta) == len(tb)
    for x, y in zip(ta, tb):
        try:
            fx, fy = float(x), float(y)
        except ValueError:
            assert x == y
            continue
        assert fy == pytest.approx(fx, rel=NORM_RTOL, abs=0.0)


@pytest.mark.parametrize("shim", ["whole", "stages"])
@pytest.mark.parametrize("curved,order", [(False, 1), (True, 3)])
def test_reference_driver_over_the_shim_writes_the_reference_files(shim, curved, order):
    GPU_EXE = GPU_EXES[shim]
    if not (os.path.exists(REF_EXE) and os.path.exists(GPU_EXE)):
        pytest.skip("oracle/build_ref_exe.sh has not been run")
    d, _, _ = make_case(64, 16, curved, order, nsteps=8)
    r_ref, w_ref = _run(REF_EXE, d)
    r_gpu, w_gpu = _run(GPU_EXE, d)
    assert "Finished Iteration 8" in r_ref.stdout
    assert "FATAL" not in r_gpu.stdout, r_gpu.stdout[-2000:]
    assert r_gpu.returncode == r_ref.returncode, (r_gpu.stdout[-2000:], r_gpu.stderr[-2000:])
    names = sorted(os.listdir(w_ref))
    assert names == sorted(os.listdir(w_gpu))
    assert "body_forces.dat" in names and "grid_solution.mesh" in names
    for n in names:
        if n == "time.dat":
            continue
        a = open(os.path.join(w_ref, n), "rb").read()
        b = open(os.path.join(w_gpu, n), "rb").read()
        if n == "residuals.dat":
            _numbers_close(a.decode(), b.decode())
        else:
            assert a == b, n
    steps = np.loadtxt(os.path.join(w_gpu, "residuals.dat"))
    assert steps.shape[0] == 8
