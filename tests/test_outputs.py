"""Solution writers on the CPU: the oracle's restatement (oracle/outputs.py)
against the reference's own write_surface_cp, write_tecplot_solutionC and
write_tecplot_solutionP (grid_io.C:102-331, 841-1375) byte for byte, on
states after a few reference steps and on a perturbed state; and the
renumbered connectivity and boundary segments that the library's
preprocessing hands to its writers against the reference's."""
import os
import tempfile

import numpy as np
import pytest

from cases import make_case


def _ref_after(ref_lib, nc, nr, curved, order, steps):
    d, _, fp = make_case(nc, nr, curved, order)
    r = ref_lib.RefSolver(d)
    for ts in range(1, steps + 1):
        r.solve(ts)
    return d, fp, r


def _compare(r, fp, tag):
    from oracle import outputs
    sc = r.scalars()
    nn = sc["nn"]
    Q, x = r.array("Q"), r.array("x")
    bbc = r.array("bbc")
    segs = r.segments()
    out = tempfile.mkdtemp(prefix=f"writers_{tag}_")
    r.write_surface_cp(out)
    mine = outputs.surface_cp_files(Q, x, bbc, segs, fp.gamma, fp.mach)
    written = sorted(f for f in os.listdir(out) if f.startswith("surface_"))
    assert written == sorted(f"surface_{b}_pressure.dat" for b in mine)
    assert mine, "no inviscid boundary"
    for b, data in mine.items():
        with open(os.path.join(out, f"surface_{b}_pressure.dat"), "rb") as f:
            assert f.read() == data, f"surface file of boundary {b} differs"
    tri, quad = r.array("c2n_tri"), r.array("c2n_quad")
    if quad.size == 0:
        quad = np.zeros(4, dtype=np.int32)
    for prim in (False, True):
        path = os.path.join(out, f"tecplot_{int(prim)}.dat")
        r.write_tecplot(path, prim)
        with open(path, "rb") as f:
            ref_bytes = f.read()
        assert outputs.tecplot_bytes(Q, x, nn, tri, quad, prim, fp.gamma) == ref_bytes
    return mine


@pytest.mark.parametrize("nc,nr,curved,order,steps", [(128, 32, False, 1, 3),
                                                       (64, 16, True, 3, 3)])
def test_oracle_writers_match_the_reference(ref_lib, nc, nr, curved, order, steps):
    d, fp, r = _ref_after(ref_lib, nc, nr, curved, order, steps)
    files = _compare(r, fp, f"{nc}x{nr}")
    # a solved state has a pressure field that varies along the wall
    for data in files.values():
        cps = [float(l.split()[1]) for l in data.decode().splitlines()]
        assert len(cps) > 8 and max(cps) > min(cps)
    r.close()


def test_oracle_writers_on_a_perturbed_state_with_ties(ref_lib):
    """Random positive states; three wall nodes share one x, two of them
    also one state (identical lines) and the third another (the sort's tie
    rule orders it by its bytes)."""
    d, fp, r = _ref_after(ref_lib, 64, 16, False, 1, 1)
    rng = np.random.Generator(np.random.PCG64(11))
    Q = r.array("Q").reshape(-1, 4)
    Q[1:, 0] = rng.uniform(0.5, 1.5, len(Q) - 1)
    Q[1:, 1:3] = rng.uniform(-0.6, 0.6, (len(Q) - 1, 2))
    Q[1:, 3] = rng.uniform(2.0, 3.0, len(Q) - 1)
    segs = r.segments()
    wall = next(s for b, s in enumerate(segs, 1) if r.array("bbc")[b] % 2)
    a, c, e = wall[0][0], wall[len(wall) // 2][0], wall[len(wall) // 3][0]
    Q[c] = Q[a]
    x = r.array("x").reshape(-1, 2)
    x[c, 0] = x[a, 0]
    x[e, 0] = x[a, 0]
    r.set_array("Q", Q.ravel())
    r.set_array("x", x.ravel())
    _compare(r, fp, "perturbed")
    r.close()


@pytest.mark.parametrize("curved,order", [(False, 1), (True, 3)])
def test_prep_connectivity_and_segments_match_the_reference(ref_lib, curved, order):
    from flowgpu.prep import Mesh
    d, _, fp = make_case(64, 16, curved, order)
    r = ref_lib.RefSolver(d)
    m = Mesh.from_case(d, order=order)
    tri, quad = m.elements()
    assert np.array_equal(tri[3:], r.array("c2n_tri")[3:])
    assert len(quad) == 4
    nb, bbc, nbs, seg = m.segments()
    ref_segs = r.segments()
    assert nb == len(ref_segs)
    assert np.array_equal(bbc[1:], r.array("bbc")[1:])
    assert [int(n) for n in nbs[1:]] == [len(s) for s in ref_segs]
    flat = [n for s in ref_segs for pair in s for n in pair]
    assert np.array_equal(seg, np.asarray(flat, dtype=np.int32))
    m.close()
    r.close()


def test_oracle_writers_on_a_quadrilateral_mesh(ref_lib, tmp_path):
    """Quadrilaterals switch the Tecplot zone type, write no triangles and use
    the reference's other pressure form in write_tecplot_solutionP."""
    from cases import make_quad_case
    d = str(tmp_path / "quads")
    fp = make_quad_case(64, 16, 3, d)
    r = ref_lib.RefSolver(d)
    assert r.scalars()["nquad"] > 0 and r.scalars()["ntri"] == 0
    rng = np.random.Generator(np.random.PCG64(2))
    Q = r.array("Q").reshape(-1, 4)
    Q[1:, 0] = rng.uniform(0.5, 1.5, len(Q) - 1)
    Q[1:, 1:3] = rng.uniform(-0.5, 0.5, (len(Q) - 1, 2))
    Q[1:, 3] = rng.uniform(2.0, 3.0, len(Q) - 1)
    r.set_array("Q", Q.ravel())
    _compare(r, fp, "quads")
    r.close()
