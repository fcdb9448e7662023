"""Host preprocessing (include/flow_prep.h) against the reference's own set-up
(read_mesh, Cuthill_McKee, maps, geometry, cv_calc, Build_CRS, edge weights,
k=2 stencils and SVD factors): integer arrays identical, floating-point
arrays bit-identical.  CPU only."""
import numpy as np
import pytest

from cases import ParityCase


def _prep(case):
    from flowgpu.prep import Mesh
    return Mesh.from_case(case.dir, order=case.fp.order)


INT_KEYS = ("edges", "subedges", "bedges", "bbc", "node_order", "ia", "iau", "ja")
FLOAT_KEYS = ("x", "cv_area", "el_cent", "xn_subedges", "xm_subedges", "xg_subedges",
              "xg_bedges", "xgn_bedges")


@pytest.mark.parametrize("nc,nr,curved,order,quads", [
    (32, 8, False, 1, False), (64, 16, False, 1, False), (32, 8, True, 3, False),
    (64, 16, True, 3, False),
    (128, 64, True, 3, False),  # 8192 nodes: stencils and SVD factored on host threads
    (64, 16, False, 1, True), (64, 16, False, 3, True),  # quadrilateral meshes
    (64, 16, False, 3, "mixed"),  # quadrilaterals inside, triangles outside
    (48, 12, True, 1, "cylinder"), (48, 12, True, 3, "cylinder"),  # circular wall, bc 11
])
def test_prep_matches_reference_setup(ref_lib, nc, nr, curved, order, quads):
    case = (ParityCase(nc, nr, curved, order, cylinder=True) if quads == "cylinder"
            else ParityCase(nc, nr, curved, order, quads=quads))
    mesh = _prep(case)
    mine = mesh.arrays()
    assert mesh.sizes["nn"] == case.sizes["nn"]
    assert mesh.sizes["nsubedges"] == case.sizes["nsubedges"]
    assert np.array_equal(mesh.node_map()[1:], case.ref.array("nn_map")[1:])
    for k in INT_KEYS + FLOAT_KEYS:
        a, b = case.arrays[k], mine[k]
        if k == "x" or k == "node_order":
            assert np.array_equal(a[2 if k == "x" else 1:], b[2 if k == "x" else 1:]), k
        else:
            off = {"edges": 2, "subedges": 2, "bedges": 5, "bbc": 1, "ia": 0, "iau": 1, "ja": 0,
                   "cv_area": 1, "el_cent": 2, "xn_subedges": 3, "xm_subedges": 2,
                   "xg_subedges": 6, "xg_bedges": 6, "xgn_bedges": 9}[k]
            assert np.array_equal(a[off:], b[off:]), k
    assert np.array_equal(case.xnb0[3:], mine["xn_bedges"][3:])
    if order == 1:
        assert np.array_equal(case.arrays["edge_weight"][4:], mine["edge_weight"][4:])
    else:
        assert np.array_equal(case.arrays["moments"][9:], mine["moments"][9:])
        for k in ("gnsn", "gnnsn", "gnnsn1", "svd_m"):
            assert np.array_equal(case.arrays[k][:mine[k].size], mine[k]), k
        assert np.array_equal(case.arrays["svd_S"][5:], mine["svd_S"][5:])
        assert np.array_equal(case.arrays["svd_VT"][25:], mine["svd_VT"][25:])
        nn = case.sizes["nn"]
        for i in range(1, nn + 1):
            m = mine["svd_m"][i]
            a = case.arrays["svd_U"][case.arrays["svd_off"][i]:][:5 * m]
            b = mine["svd_U"][mine["svd_off"][i]:][:5 * m]
            assert np.array_equal(a, b), i
    Q = mesh.initial_state(case.fp)
    assert np.array_equal(Q[4:], case.Q0[4:])


@pytest.mark.parametrize("curved,order", [(False, 1), (True, 3)])
def test_in_memory_grid_gives_the_arrays_of_its_mesh_file(curved, order, tmp_path):
    """Mesh.from_grid (flow_prep_build on the generator's arrays) and
    Mesh.from_case (the written mesh file through flow_prep_read) give the
    same preprocessed arrays, bit for bit."""
    from flowgpu import workloads
    from flowgpu.prep import Mesh
    wl = workloads.Workload("mem", 64, 16, curved, order, 0.7)
    a = Mesh.from_case(wl.write(str(tmp_path)), order=order)
    b = Mesh.from_grid(wl.grid(), order=order)
    assert a.sizes == b.sizes
    A, B = a.arrays(), b.arrays()
    assert A.keys() == B.keys()
    for k in A:
        if A[k] is None:
            assert B[k] is None, k
        else:
            assert np.array_equal(A[k], B[k]), k
    for x, y in zip(a.elements(), b.elements()):
        assert np.array_equal(x, y)
    for x, y in zip(a.segments()[1:], b.segments()[1:]):
        assert np.array_equal(x, y)
    fp = wl.params()
    assert np.array_equal(a.initial_state(fp), b.initial_state(fp))
    a.close()
    b.close()


def test_generator_rejects_a_boundary_segment_with_the_domain_on_its_right():
    from flowgpu import meshgen
    g = meshgen.make_ogrid(64, 16, seed=1)
    bc, segs = g.boundaries[0]
    g.boundaries[0] = (bc, segs[:, ::-1].copy())
    with pytest.raises(ValueError, match="domain on its right"):
        meshgen._check_segments(g)


def test_concurrent_in_memory_preprocessing_is_deterministic():
    """flow_prep_build called from several Python threads at once (as the
    serving workers do), each splitting its stencils and SVD over host
    threads, gives the arrays a one-at-a-time build gives."""
    import concurrent.futures as cf
    from flowgpu import workloads
    from flowgpu.prep import Mesh
    wls = [workloads.Workload(f"conc{i}", 128, 64 + 8 * i, i % 2 == 0, 3 if i % 2 == 0 else 1,
                              0.7, seed=20 + i) for i in range(4)]
    grids = [wl.grid() for wl in wls]

    def build(i):
        m = Mesh.from_grid(grids[i], order=wls[i].order)
        out = m.arrays()
        m.close()
        return out

    alone = [build(i) for i in range(len(wls))]
    with cf.ThreadPoolExecutor(max_workers=4) as ex:
        together = list(ex.map(build, range(len(wls))))
    for a, b in zip(alone, together):
        assert a.keys() == b.keys()
        for k in a:
            assert (a[k] is None and b[k] is None) or np.array_equal(a[k], b[k]), k
