"""Solution writers on the GPU, through the C ABI: after the same FP64 steps
as the reference (whose state the drop-in reproduces bit for bit),
flow_write_surface_cp and flow_write_tecplot write the same bytes as the
reference's write_surface_cp, write_tecplot_solutionC and
write_tecplot_solutionP (grid_io.C), and flow_surface_cp's nodes and
pressure coefficients equal the oracle's bit for bit."""
import os
import tempfile

import numpy as np
import pytest

from cases import make_case

pytestmark = pytest.mark.gpu


def _pair(ref_lib, nc, nr, curved, order, steps):
    from flowgpu import capi
    from flowgpu.prep import Mesh
    d, _, fp = make_case(nc, nr, curved, order)
    ref = ref_lib.RefSolver(d)
    mesh = Mesh.from_case(d, order=order)
    s = capi.Solver.from_mesh(mesh, fp, device=0)
    s.set_state(mesh.initial_state(fp))
    for ts in range(1, steps + 1):
        ref.solve(ts)
        s.solve(ts)
    return fp, ref, mesh, s


def _same_files(dir_a, dir_b, names):
    for n in names:
        with open(os.path.join(dir_a, n), "rb") as fa, open(os.path.join(dir_b, n), "rb") as fb:
            assert fa.read() == fb.read(), n


@pytest.mark.parametrize("nc,nr,curved,order,steps", [(128, 32, False, 1, 3),
                                                       (64, 16, True, 3, 3)])
def test_writers_match_the_reference(ref_lib, nc, nr, curved, order, steps):
    from oracle import outputs
    fp, ref, mesh, s = _pair(ref_lib, nc, nr, curved, order, steps)
    Q = s.get("Q")
    assert np.array_equal(Q[4:], ref.array("Q")[4:])  # entry 0 unused by the reference
    nb, bbc, nbs, seg = mesh.segments()
    segs = ref.segments()
    for b in range(1, nb + 1):
        nodes, cp = s.surface_cp(mesh, b)
        want = outputs.boundary_nodes(segs[b - 1])
        assert nodes.tolist() == want
        assert np.array_equal(cp, outputs.surface_cp(Q, want, fp.gamma, fp.mach))
    ref_dir = tempfile.mkdtemp(prefix="ref_out_")
    gpu_dir = tempfile.mkdtemp(prefix="gpu_out_")
    ref.write_surface_cp(ref_dir)
    s.write_surface_cp(mesh, gpu_dir)
    names = sorted(os.listdir(ref_dir))
    assert names and names == sorted(os.listdir(gpu_dir))
    _same_files(ref_dir, gpu_dir, names)
    for prim in (False, True):
        name = f"tecplot_{'primitive' if prim else 'conserved'}.dat"
        ref.write_tecplot(os.path.join(ref_dir, name), prim)
        s.write_tecplot(mesh, os.path.join(gpu_dir, name), prim)
        _same_files(ref_dir, gpu_dir, [name])
    s.close()
    mesh.close()
    ref.close()


def test_surface_cp_rejects_bad_arguments(ref_lib):
    import ctypes as C
    from flowgpu import capi
    fp, ref, mesh, s = _pair(ref_lib, 32, 8, False, 1, 1)
    nb, bbc, nbs, seg = mesh.segments()
    with pytest.raises(capi.FlowError):
        s.surface_cp(mesh, nb + 1)
    # output arrays shorter than the boundary's node list
    nodes = np.zeros(2, dtype=np.int32)
    cp = np.zeros(2)
    cnt = C.c_int(0)
    L = capi.load()
    rc = L.flow_surface_cp(s.ctx, C.byref(s.p), nb, nbs.ctypes.data_as(capi.IP),
                           seg.ctypes.data_as(capi.IP), 1, nodes.ctypes.data_as(capi.IP),
                           cp.ctypes.data_as(capi.DP), 2, C.byref(cnt))
    assert rc == capi.ERR_ARG and cnt.value > 2
    # a segment naming a node beyond nn is refused on the host
    bad = seg.copy()
    bad[0] = mesh.sizes["nn"] + 1
    rc = L.flow_surface_cp(s.ctx, C.byref(s.p), nb, nbs.ctypes.data_as(capi.IP),
                           bad.ctypes.data_as(capi.IP), 1, nodes.ctypes.data_as(capi.IP),
                           cp.ctypes.data_as(capi.DP), 2, C.byref(cnt))
    assert rc == capi.ERR_ARG and b"outside" in L.flow_last_error()
    assert s.status() == 0
    s.close()
    mesh.close()
    ref.close()


def test_tecplot_writer_quadrilateral_branch(ref_lib, tmp_path):
    """flow_write_tecplot given quadrilaterals besides the triangles: the
    quadrilateral zone, triangles written as degenerate quadrilaterals, and
    the reference's other pressure form; against the oracle for the
    context's state."""
    import ctypes as C
    from flowgpu import capi
    from oracle import outputs
    fp, ref, mesh, s = _pair(ref_lib, 32, 8, False, 1, 2)
    Q = s.get("Q")
    x = mesh.array("x")
    nn = mesh.sizes["nn"]
    tri, _ = mesh.elements()
    quad = np.concatenate([np.zeros(4, dtype=np.int32),
                           (np.arange(4 * 9, dtype=np.int32) * 7) % nn + 1])
    L = capi.load()
    for prim in (False, True):
        path = tmp_path / f"quads_{int(prim)}.dat"
        rc = L.flow_write_tecplot(s.ctx, C.byref(s.p), str(path).encode(), int(prim),
                                  x.ctypes.data_as(capi.DP), len(tri) // 3 - 1,
                                  tri.ctypes.data_as(capi.IP), len(quad) // 4 - 1,
                                  quad.ctypes.data_as(capi.IP))
        assert rc == 0
        assert path.read_bytes() == outputs.tecplot_bytes(Q, x, nn, tri, quad, prim, fp.gamma)
    s.close()
    mesh.close()
    ref.close()
