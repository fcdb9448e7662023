"""Host preprocessing through libflowgpu.so (include/flow_prep.h): a mesh file
in the reference's format -> the grid arrays of the nonlinear iteration."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import capi

def _lib():
    """The library handle; capi.load() sets the preprocessing prototypes."""
    return capi.load()


def read_bc(path: str) -> list[int]:
    """bc.dat: one boundary-condition id per line (mesh_io.C:282-297)."""
    with open(path) as f:
        return [int(line.split()[0]) for line in f if line.strip()]


class Mesh:
    """A preprocessed mesh owned by the library (flow_mesh)."""

    def __init__(self, mesh_path: str, bbc, order: int, reorder: int = 1):
        self.L = _lib()
        bc = np.ascontiguousarray(bbc, dtype=np.int32)
        st = C.c_int(0)
        self.h = self.L.flow_prep_read(mesh_path.encode(), bc.ctypes.data_as(capi.IP), len(bc),
                                       int(reorder), int(order), C.byref(st))
        if not self.h:
            raise capi.FlowError(st.value or 1, "flow_prep_read: " +
                                 self.L.flow_prep_last_error().decode())
        self.order = order
        self.view = capi.FlowGridView()
        self.L.flow_prep_view(self.h, C.byref(self.view))

    @classmethod
    def from_grid(cls, g, order: int, reorder: int = 1):
        """From a generated grid in memory (flowgpu.meshgen.OGrid: x, 1-based
        triangles, (bc, segments) per boundary) through flow_prep_build: the
        same arrays flow_prep_read gives for the grid's mesh file, without the
        file."""
        self = cls.__new__(cls)
        self.L = _lib()
        x = np.ascontiguousarray(g.x, dtype=np.float64)
        tri = np.ascontiguousarray(g.tris, dtype=np.int32)
        nbs = np.array([len(segs) for _, segs in g.boundaries], dtype=np.int32)
        seg = np.ascontiguousarray(np.concatenate([np.asarray(segs, dtype=np.int32).reshape(-1, 2)
                                                   for _, segs in g.boundaries]))
        bbc = np.array([bc for bc, _ in g.boundaries], dtype=np.int32)
        quad = np.zeros(4, dtype=np.int32)
        st = C.c_int(0)
        self.h = self.L.flow_prep_build(int(x.shape[0]), x.ctypes.data_as(capi.DP), int(tri.shape[0]),
                                        tri.ctypes.data_as(capi.IP), 0, quad.ctypes.data_as(capi.IP),
                                        len(nbs), nbs.ctypes.data_as(capi.IP),
                                        seg.ctypes.data_as(capi.IP), bbc.ctypes.data_as(capi.IP),
                                        int(reorder), int(order), C.byref(st))
        if not self.h:
            raise capi.FlowError(st.value or 1, "flow_prep_build: " +
                                 self.L.flow_prep_last_error().decode())
        self.order = order
        self.view = capi.FlowGridView()
        self.L.flow_prep_view(self.h, C.byref(self.view))
        return self

    @classmethod
    def from_case(cls, casedir: str, order: int, mesh_name: str = "grid.mesh", reorder: int = 1):
        return cls(os.path.join(casedir, mesh_name), read_bc(os.path.join(casedir, "bc.dat")),
                   order, reorder)

    def close(self):
        if getattr(self, "h", None):
            self.L.flow_prep_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def sizes(self) -> dict:
        v = self.view
        return {"nn": v.nn, "nn_ghost": v.nn_ghost, "nedges": v.nedges,
                "nsubedges": v.nsubedges, "nbedges": v.nbedges, "nb": v.nb, "nelem": v.nelem}

    def initial_state(self, params) -> np.ndarray:
        v = self.view
        Q = np.zeros((v.nn + v.nn_ghost + 1) * 4)
        p = capi.params_struct(params)
        self.L.flow_prep_initial_state(self.h, C.byref(p), Q.ctypes.data_as(capi.DP))
        return Q

    def array(self, name: str) -> np.ndarray:
        """Copy of one array of the view, in the reference layout."""
        v = self.view
        nn, ng, ne, ns, nb = v.nn, v.nn_ghost, v.nedges, v.nsubedges, v.nbedges
        nnz = int(np.ctypeslib.as_array(v.ia, shape=(nn + 2,))[nn + 1])
        lens = {"edges": (ne + 1) * 2, "subedges": (ns + 1) * 2, "bedges": (nb + 1) * 5,
                "bedge_seg": (nb + 1) * 2, "bbc": v.nb + 1, "node_order": nn + ng + 1,
                "ia": nn + 2, "iau": nn + 1, "ja": nnz, "x": (nn + ng + 1) * 2,
                "cv_area": nn + 1, "el_cent": (v.nelem + 1) * 2, "xn_subedges": (ns + 1) * 3,
                "xm_subedges": (ns + 1) * 2, "xg_subedges": (ns + 1) * 6,
                "xn_bedges": (nb + 1) * 3, "xg_bedges": (nb + 1) * 6, "xgn_bedges": (nb + 1) * 9,
                "edge_weight": (ne + 1) * 4, "moments": (nn + 1) * 9, "gnnsn1": nn + 2,
                "svd_m": nn + 1, "svd_VT": (nn + 1) * 25, "svd_S": (nn + 1) * 5}
        if name in ("gnnsn", "gnsn", "svd_U", "svd_off"):
            g1 = np.ctypeslib.as_array(v.gnnsn1, shape=(nn + 2,))
            if name == "gnnsn":
                lens[name] = int(g1[nn + 1]) + 1
            elif name == "gnsn":
                gn = np.ctypeslib.as_array(v.gnnsn, shape=(int(g1[nn + 1]) + 1,))
                lens[name] = int(gn[g1[nn + 1]])
            elif name == "svd_off":
                lens[name] = nn + 1
            else:
                m = np.ctypeslib.as_array(v.svd_m, shape=(nn + 1,))
                lens[name] = int(5 * m.sum())
        ptr = getattr(v, name)
        if not ptr:
            return None
        return np.ctypeslib.as_array(ptr, shape=(lens[name],)).copy()

    def arrays(self) -> dict:
        names = ["edges", "subedges", "bedges", "bedge_seg", "bbc", "node_order", "ia", "iau",
                 "ja", "x", "cv_area", "el_cent", "xn_subedges", "xm_subedges", "xg_subedges",
                 "xn_bedges", "xg_bedges", "xgn_bedges", "edge_weight", "moments"]
        if self.order == 3:
            names += ["gnsn", "gnnsn", "gnnsn1", "svd_m", "svd_off", "svd_U", "svd_VT", "svd_S"]
        return {n: self.array(n) for n in names}

    def elements(self):
        """Renumbered connectivity (GRID::c2n[Tri], c2n[Quad]): 1-based rows,
        row 0 unused, as flat int32 arrays."""
        nt, nq = C.c_int(), C.c_int()
        tp, qp = capi.IP(), capi.IP()
        self.L.flow_prep_elements(self.h, C.byref(nt), C.byref(tp), C.byref(nq), C.byref(qp))
        tri = np.ctypeslib.as_array(tp, shape=((nt.value + 1) * 3,)).copy()
        quad = np.ctypeslib.as_array(qp, shape=((nq.value + 1) * 4,)).copy()
        return tri, quad

    def segments(self):
        """nb, bbc and nbs (index 0 unused) and every boundary's renumbered
        segment node pairs in order, flat int32 (GRID::bs)."""
        nb = C.c_int()
        bp, np_, sp = capi.IP(), capi.IP(), capi.IP()
        self.L.flow_prep_segments(self.h, C.byref(nb), C.byref(bp), C.byref(np_), C.byref(sp))
        bbc = np.ctypeslib.as_array(bp, shape=(nb.value + 1,)).copy()
        nbs = np.ctypeslib.as_array(np_, shape=(nb.value + 1,)).copy()
        n = 2 * int(nbs[1:].sum())
        seg = (np.ctypeslib.as_array(sp, shape=(n,)).copy() if n
               else np.zeros(1, dtype=np.int32))
        return nb.value, bbc, nbs, seg

    def restart_state(self):
        """(Q, last step, its CFL) from the file's restart block, or None."""
        v = self.view
        Q = np.zeros((v.nn + v.nn_ghost + 1) * 4)
        citer, cfl = C.c_int(0), C.c_double(0.)
        rc = self.L.flow_prep_restart_state(self.h, Q.ctypes.data_as(capi.DP), Q.size,
                                            C.byref(citer), C.byref(cfl))
        if rc == 128:  # FLOW_ERR_NOT_FOUND: no restart block
            return None
        if rc:
            raise capi.FlowError(rc, "flow_prep_restart_state")
        return Q, citer.value, cfl.value

    def node_map(self) -> np.ndarray:
        return np.ctypeslib.as_array(self.L.flow_prep_node_map(self.h), shape=(self.view.nn + 1,)).copy()
