"""ctypes access to the C restatement of the hot path (oracle/flow_oracle.c).

Test infrastructure only.  ``OracleGrid`` owns numpy arrays in the
reference's layout (1-based, array-of-structs) and a matching ``orc_grid``
struct; ``from_reference`` fills them from a set-up ``oracle.ref.RefSolver``.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libflow_oracle.so")

_lib = None

IP = C.POINTER(C.c_int)
DP = C.POINTER(C.c_double)
LP = C.POINTER(C.c_long)


class OrcParams(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("iter", "jufreq", "ramp", "subits", "unsteady", "tacc",
                                       "method", "order", "foits", "soits", "toits", "limit")] + \
               [(n, C.c_double) for n in ("CFL", "gamma", "alpha", "mach", "mintime")] + \
               [("jac_approx", C.c_int)]


_GRID_INTS = ("nn", "nn_ghost", "nedges", "nsubedges", "nbedges", "nb")
_GRID_IPTR = ("edges", "subedges", "bedges", "bedge_seg", "bbc", "node_order", "ia", "iau", "ja")
_GRID_DPTR1 = ("x", "cv_area", "el_cent", "xn_subedges", "xm_subedges", "xg_subedges",
               "xn_bedges", "xg_bedges", "xgn_bedges", "edge_weight", "moments")
_GRID_IPTR2 = ("gnsn", "gnnsn", "gnnsn1")
_GRID_STATE = ("Q", "nQ", "pQ", "dQ", "R", "grad", "hess", "phi", "point_value", "dt",
               "ev_con", "LHS", "RHS")


class OrcGrid(C.Structure):
    _fields_ = ([(n, C.c_int) for n in _GRID_INTS]
                + [(n, IP) for n in _GRID_IPTR]
                + [(n, DP) for n in _GRID_DPTR1]
                + [(n, IP) for n in _GRID_IPTR2]
                + [("svd_off", LP), ("svd_m", IP), ("svd_U", DP), ("svd_VT", DP), ("svd_S", DP)]
                + [(n, DP) for n in _GRID_STATE]
                + [("cfl", C.c_double), ("citer", C.c_int)])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("oracle/_build/libflow_oracle.so is not built (oracle/build_oracle.sh)")
        L = C.CDLL(LIB_PATH)
        gp, pp = C.POINTER(OrcGrid), C.POINTER(OrcParams)
        L.orc_build_matrix.argtypes = [gp, pp]
        L.orc_gradient_lsq.argtypes = [gp]
        L.orc_derivatives_k2.argtypes = [gp]
        L.orc_limiter_venkat.argtypes = [gp, pp]
        L.orc_interior_residuals.argtypes = [gp, pp, C.c_int, C.c_int]
        L.orc_set_boundary_values.argtypes = [gp, pp]
        L.orc_boundary_residuals.argtypes = [gp, pp, C.c_int]
        L.orc_linear_solve.argtypes = [gp, pp]
        L.orc_linear_solve.restype = C.c_double
        L.orc_body_forces.argtypes = [gp, pp, DP]
        L.orc_solve.argtypes = [gp, pp, C.c_int, DP]
        L.orc_greedy_colors.argtypes = [gp, IP]
        L.orc_linear_solve_mixed.argtypes = [gp, pp, IP, C.c_int]
        L.orc_solve_mixed.argtypes = [gp, pp, C.c_int, DP, IP, C.c_int]
        L.orc_solve_mixed_order.argtypes = [gp, pp, C.c_int, DP, IP]
        L.orc_roe_flux.argtypes = [C.c_double] * 4 + [DP, DP, DP]
        L.orc_curved_normal.argtypes = [C.c_int, DP, DP, DP]
        _lib = L
    return _lib


def params_from_vector(v) -> OrcParams:
    """v: the 25-entry vector of RefSolver.params() (euler.params order + cfl)."""
    p = OrcParams()
    p.iter, p.jufreq, p.CFL, p.ramp = int(v[1]), int(v[2]), v[3], int(v[4])
    p.gamma, p.alpha, p.mach, p.subits = v[5], v[6], v[7], int(v[8])
    p.unsteady, p.tacc, p.mintime, p.method = int(v[9]), int(v[10]), v[11], int(v[12])
    p.order, p.foits, p.soits, p.toits = int(v[13]), int(v[14]), int(v[15]), int(v[16])
    p.limit = int(v[18])
    return p


def params_from_flow(fp) -> OrcParams:
    """fp: a flowgpu.meshgen.FlowParams."""
    p = OrcParams()
    for n in ("iter", "jufreq", "ramp", "subits", "unsteady", "tacc", "method", "order", "foits",
              "soits", "toits", "limit"):
        setattr(p, n, int(getattr(fp, n)))
    for n in ("CFL", "gamma", "alpha", "mach", "mintime"):
        setattr(p, n, float(getattr(fp, n)))
    return p


def _iptr(a):
    return a.ctypes.data_as(IP) if a is not None and a.size else None


def _dptr(a):
    return a.ctypes.data_as(DP) if a is not None and a.size else None


class OracleGrid:
    """numpy-backed orc_grid.  ``arrays`` keys follow the reference's names."""

    def __init__(self, sizes: dict, arrays: dict):
        self.L = lib()
        self.a = {}
        for k, v in arrays.items():
            if v is None:
                continue
            dt = np.float64 if v.dtype.kind == "f" else (np.int64 if k == "svd_off" else np.int32)
            self.a[k] = np.ascontiguousarray(v, dtype=dt).copy()
        nn, ng = sizes["nn"], sizes["nn_ghost"]
        nnz = int(self.a["ia"][nn + 1])
        zeros = {"Q": (nn + ng + 1) * 4, "nQ": (nn + ng + 1) * 4, "pQ": (nn + ng + 1) * 4,
                 "dQ": (nn + 1) * 4, "R": (nn + 1) * 4, "grad": (nn + 1) * 8,
                 "hess": (nn + 1) * 36, "phi": (nn + 1) * 8, "point_value": (nn + 1) * 4,
                 "dt": nn + 1, "ev_con": nn + 1, "LHS": nnz * 16, "RHS": (nn + 1) * 4}
        for k, n in zeros.items():
            if k not in self.a:
                self.a[k] = np.zeros(n)
        g = OrcGrid()
        for n in _GRID_INTS:
            setattr(g, n, int(sizes[n]))
        for n in _GRID_IPTR + _GRID_IPTR2 + ("svd_m",):
            setattr(g, n, _iptr(self.a.get(n)))
        for n in _GRID_DPTR1 + _GRID_STATE + ("svd_U", "svd_VT", "svd_S"):
            setattr(g, n, _dptr(self.a.get(n)))
        off = self.a.get("svd_off")
        g.svd_off = off.ctypes.data_as(LP) if off is not None else None
        g.citer = 0
        g.cfl = 0.0
        self.g = g
        self.sizes = dict(sizes)

    def __getitem__(self, k):
        return self.a[k]

    def set(self, k, v):
        self.a[k][...] = np.asarray(v, dtype=self.a[k].dtype).reshape(self.a[k].shape)

    # ---- stages ----
    def solve(self, p: OrcParams, ts: int) -> float:
        self.g.citer = ts
        dq = C.c_double()
        rc = self.L.orc_solve(C.byref(self.g), C.byref(p), ts, C.byref(dq))
        if rc:
            raise RuntimeError(f"oracle solve failed with code {rc}")
        return dq.value

    def body_forces(self, p: OrcParams):
        f = (C.c_double * 2)()
        self.L.orc_body_forces(C.byref(self.g), C.byref(p), f)
        return f[0], f[1]

    def build_matrix(self, p):
        return self.L.orc_build_matrix(C.byref(self.g), C.byref(p))

    def gradient(self):
        self.L.orc_gradient_lsq(C.byref(self.g))

    def derivatives(self):
        self.L.orc_derivatives_k2(C.byref(self.g))

    def limiter(self, p):
        return self.L.orc_limiter_venkat(C.byref(self.g), C.byref(p))

    def interior(self, p, jupdate, ts):
        self.L.orc_interior_residuals(C.byref(self.g), C.byref(p), jupdate, ts)

    def boundary(self, p, jupdate):
        return self.L.orc_boundary_residuals(C.byref(self.g), C.byref(p), jupdate)

    def linear_solve(self, p):
        return self.L.orc_linear_solve(C.byref(self.g), C.byref(p))

    # ---- precision form (FP32 blocks, multicolour sweeps) ----
    def colors(self):
        """Greedy colouring of the block pattern: (color[0..nn], ncolors)."""
        if getattr(self, "_colors", None) is None:
            col = np.zeros(self.sizes["nn"] + 1, dtype=np.int32)
            nc = self.L.orc_greedy_colors(C.byref(self.g), col.ctypes.data_as(IP))
            self._colors = (col, nc)
        return self._colors

    def linear_solve_mixed(self, p, ordered: bool = False):
        col, nc = self.colors()
        cp = None if ordered else col.ctypes.data_as(IP)
        self.L.orc_linear_solve_mixed(C.byref(self.g), C.byref(p), cp, nc)

    def solve_mixed_order(self, p: OrcParams, ts: int, order) -> float:
        """Precision form step with the sweeps visiting rows in `order`."""
        o = np.ascontiguousarray(order, dtype=np.int32)
        self.g.citer = ts
        dq = C.c_double()
        rc = self.L.orc_solve_mixed_order(C.byref(self.g), C.byref(p), ts, C.byref(dq),
                                          o.ctypes.data_as(IP))
        if rc:
            raise RuntimeError(f"oracle solve failed with code {rc}")
        return dq.value

    def solve_mixed(self, p: OrcParams, ts: int, ordered: bool = False) -> float:
        """Precision form step: multicolour sweeps, or (ordered) the
        reference's row order, with FP32 blocks."""
        col, nc = self.colors()
        self.g.citer = ts
        dq = C.c_double()
        cp = None if ordered else col.ctypes.data_as(IP)
        rc = self.L.orc_solve_mixed(C.byref(self.g), C.byref(p), ts, C.byref(dq), cp, nc)
        if rc:
            raise RuntimeError(f"oracle solve failed with code {rc}")
        return dq.value


def roe_flux(nx, ny, length, gamma, ql, qr):
    ql = np.ascontiguousarray(ql, dtype=np.float64)
    qr = np.ascontiguousarray(qr, dtype=np.float64)
    out = np.zeros(4)
    lib().orc_roe_flux(nx, ny, length, gamma, _dptr(ql), _dptr(qr), _dptr(out))
    return out


GEOMETRY_KEYS = ("edges", "subedges", "bedges", "bbc", "node_order", "ia", "iau", "ja", "x",
                 "cv_area", "el_cent", "xn_subedges", "xm_subedges", "xg_subedges", "xn_bedges",
                 "xg_bedges", "xgn_bedges", "edge_weight", "Moments", "gnsn", "gnnsn", "gnnsn1")


def reference_arrays(ref, with_svd: bool = False) -> tuple[dict, dict]:
    """Pull sizes and the geometry/topology arrays out of a RefSolver."""
    sc = ref.scalars()
    a = {k: ref.array(k) for k in GEOMETRY_KEYS}
    a["moments"] = a.pop("Moments")
    segs = ref.segments()
    b = a["bedges"].reshape(-1, 5)
    seg = np.zeros((sc["nbedges"] + 1, 2), dtype=np.int32)
    for i in range(1, sc["nbedges"] + 1):
        seg[i] = segs[b[i, 3] - 1][b[i, 4] - 1]
    a["bedge_seg"] = seg.ravel()
    ew = a["edge_weight"]
    if ew.size == 0:
        a["edge_weight"] = np.zeros((sc["nedges"] + 1) * 4)
    for k in ("Q",):
        a[k] = ref.array(k)
    if with_svd:
        nn = sc["nn"]
        size = ref.array("SVD_size").reshape(-1, 3)
        m = np.zeros(nn + 1, dtype=np.int32)
        off = np.zeros(nn + 1, dtype=np.int64)
        U, VT, S = [], np.zeros((nn + 1) * 25), np.zeros((nn + 1) * 5)
        pos = 0
        for i in range(1, nn + 1):
            f = ref.svd(i)
            if f is None:
                continue
            u, vt, s = f
            m[i] = int(size[i, 0])
            off[i] = pos
            U.append(u)
            pos += u.size
            VT[i * 25:(i + 1) * 25] = vt
            S[i * 5:(i + 1) * 5] = s
        a["svd_m"], a["svd_off"] = m, off
        a["svd_U"] = np.concatenate(U) if U else np.zeros(1)
        a["svd_VT"], a["svd_S"] = VT, S
    return sc, a
