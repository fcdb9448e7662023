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


@pytest.mark.parametrize("nc,nr,curved,order", [
    (32, 8, False, 1), (64, 16, False, 1), (32, 8, True, 3), (64, 16, True, 3),
])
def test_prep_matches_reference_setup(ref_lib, nc, nr, curved, order):
    case = ParityCase(nc, nr, curved, order)
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
