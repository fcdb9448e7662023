"""Golden vectors recorded from the reference solver (tests/golden/*.npz,
made by tests/golden/make_golden.py): the oracle's C restatement, fed by the
library's own preprocessing of the stored mesh, reproduces them bit for bit.
CPU only; needs neither the reference sources nor a GPU."""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
CASES = sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz"))


def load_case(name, tmp_path):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    d = tmp_path / name
    d.mkdir()
    (d / "grid.mesh").write_text(str(z["mesh"]))
    (d / "bc.dat").write_text(str(z["bc"]))
    (d / "euler.params").write_text(str(z["params"]))
    return z, str(d)


def params_of(casedir):
    from flowgpu import meshgen
    vals = [l.strip() for l in open(os.path.join(casedir, "euler.params")) if not l.startswith("#")]
    fp = meshgen.FlowParams()
    for name, v in zip(meshgen.FlowParams.FIELDS, vals):
        setattr(fp, name, float(v) if isinstance(getattr(fp, name), float) else int(v))
    return fp


@pytest.mark.parametrize("name", CASES)
def test_oracle_reproduces_golden(name, tmp_path):
    from flowgpu.prep import Mesh
    from oracle import port
    z, d = load_case(name, tmp_path)
    fp = params_of(d)
    mesh = Mesh.from_case(d, order=int(z["order"]))
    sizes = dict(mesh.sizes)
    arrays = mesh.arrays()
    arrays["Q"] = mesh.initial_state(fp)
    og = port.OracleGrid(sizes, arrays)
    p = port.params_from_flow(fp)
    nn = sizes["nn"]
    for ts in range(1, int(z["steps"]) + 1):
        dq = og.solve(p, ts)
        assert np.array_equal(og["R"][4:].reshape(nn, 4), z["R"][ts - 1]), ts
        assert np.array_equal(og["dQ"][4:].reshape(nn, 4), z["dQ"][ts - 1]), ts
        assert dq == z["dq_norm"][ts - 1]
        assert og.body_forces(p) == tuple(z["forces"][ts - 1])
        if ts == 1:
            L = og["LHS"].reshape(-1, 16)
            assert np.array_equal(L[og["iau"][1:nn + 1]], z["diag1"])
    assert np.array_equal(og["Q"][4:].reshape(-1, 4), z["Q"])
