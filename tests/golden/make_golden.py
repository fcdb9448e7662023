"""Generate the golden vectors of tests/golden/ from the reference solver.

    python tests/golden/make_golden.py

Runs the reference built from its own sources (oracle/_ref/libflowref.so) on
small seeded O-grids and records, per pseudo-time step, the residual R, the
update dQ, ||dQ||, the lift/drag forces and the diagonal LHS blocks of the
first step, and the final state Q.  The mesh, bc.dat and euler.params are
stored with the vectors, so the fixtures do not depend on the generator.
"""
import io
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "flow-solver_b200")]

from flowgpu import meshgen  # noqa: E402
from oracle.ref import RefSolver  # noqa: E402

CASES = {
    "ogrid32x8_k1": dict(nc=32, nr=8, curved=False, order=1, mach=0.5, seed=7, steps=5),
    "ogrid32x8_k2": dict(nc=32, nr=8, curved=True, order=3, mach=0.8, seed=7, steps=5),
}


def make(name, nc, nr, curved, order, mach, seed, steps):
    g = meshgen.make_ogrid(nc, nr, seed=seed, curved=curved)
    fp = meshgen.FlowParams(order=order, mach=mach, ramp=1111)
    d = tempfile.mkdtemp(prefix="golden_")
    meshgen.write_case(d, g, fp)
    ref = RefSolver(d)
    nn = ref.scalars()["nn"]
    out = {"mesh": open(os.path.join(d, "grid.mesh")).read(),
           "bc": open(os.path.join(d, "bc.dat")).read(),
           "params": open(os.path.join(d, "euler.params")).read()}
    R, dQ, dqn, F = [], [], [], []
    for ts in range(1, steps + 1):
        dqn.append(ref.solve(ts))
        R.append(ref.array("R")[4:].reshape(nn, 4))
        dQ.append(ref.array("dQ")[4:].reshape(nn, 4))
        F.append(ref.body_forces())
        if ts == 1:
            ia, iau = ref.array("ia"), ref.array("iau")
            L = ref.array("LHS").reshape(-1, 16)
            diag1 = L[iau[1:nn + 1]]
    Q = ref.array("Q")[4:].reshape(-1, 4)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), R=np.array(R), dQ=np.array(dQ),
                        dq_norm=np.array(dqn), forces=np.array(F), diag1=diag1, Q=Q,
                        mesh=np.array(out["mesh"]), bc=np.array(out["bc"]),
                        params=np.array(out["params"]), order=order, steps=steps)
    print(name, "nn", nn, "steps", steps, "forces", F[-1])


if __name__ == "__main__":
    for k, v in CASES.items():
        make(k, **v)
