"""ctypes access to oracle/_ref/libflowref.so (the unmodified reference solver
plus the set-up harness in ref_harness.cpp).

Test infrastructure: imported by tests/ and by bench.py's CPU-baseline leg
only, as the checker / the reference arm.  Arrays come back as numpy copies
in the reference's own layout (1-based, array-of-structs).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libflowref.so")

_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError("oracle/_ref/libflowref.so is not built (run oracle/build_ref.sh)")
        L = C.CDLL(LIB_PATH)
        vp, ip, dp = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double)
        L.ref_open.restype = vp
        L.ref_open.argtypes = [C.c_char_p, C.c_char_p]
        L.ref_close.argtypes = [vp]
        L.ref_solve.restype = C.c_double
        L.ref_solve.argtypes = [vp, C.c_int]
        L.ref_body_forces.argtypes = [vp, dp]
        L.ref_set_citer.argtypes = [vp, C.c_int]
        for n in ("ref_build_matrix", "ref_gradient", "ref_limiter", "ref_set_boundary_values",
                  "ref_grow_stencils", "ref_alloc_work"):
            getattr(L, n).argtypes = [vp]
        L.ref_derivatives.argtypes = [vp, C.c_int]
        L.ref_interior.argtypes = [vp, C.c_int, C.c_int]
        L.ref_boundary.argtypes = [vp, C.c_int]
        L.ref_linear_solve.restype = C.c_double
        L.ref_linear_solve.argtypes = [vp]
        L.ref_scalars.argtypes = [vp, ip]
        L.ref_params.argtypes = [vp, dp]
        L.ref_array.restype = C.c_long
        L.ref_array.argtypes = [vp, C.c_char_p, C.POINTER(C.c_void_p), ip]
        L.ref_segment.argtypes = [vp, C.c_int, C.c_int, ip]
        L.ref_nbs.restype = C.c_int
        L.ref_nbs.argtypes = [vp, C.c_int]
        L.ref_svd.restype = C.c_int
        L.ref_svd.argtypes = [vp, C.c_int, C.POINTER(dp), C.POINTER(dp), C.POINTER(dp)]
        L.ref_cfl.restype = C.c_double
        L.ref_cfl.argtypes = [vp]
        L.ref_set_quiet.argtypes = [C.c_int]
        L.ref_write_surface_cp.restype = C.c_int
        L.ref_write_surface_cp.argtypes = [vp, C.c_char_p]
        L.ref_write_tecplot.argtypes = [vp, C.c_char_p, C.c_int]
        L.ref_write_mesh.argtypes = [vp, C.c_char_p]
        _lib = L
    return _lib


SCALARS = ("nn", "nn_ghost", "nedges", "nsubedges", "nbedges", "nb", "ntri", "nquad", "citer",
           "nnz", "gnnsn_len", "gnsn_len", "nsegments", "nsn_len")


class RefSolver:
    """One reference GRID/SYS_MEM/PARAMS set up from a case directory."""

    def __init__(self, casedir: str, mesh_name: str = "grid.mesh"):
        self.L = lib()
        self.h = self.L.ref_open(casedir.encode(), mesh_name.encode())
        if not self.h:
            raise RuntimeError(f"reference set-up failed for {casedir}")

    def close(self):
        if self.h:
            self.L.ref_close(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- scalars / arrays ----
    def scalars(self) -> dict:
        out = (C.c_int * 14)()
        self.L.ref_scalars(self.h, out)
        return dict(zip(SCALARS, list(out)))

    def array(self, name: str) -> np.ndarray:
        ptr = C.c_void_p()
        kind = C.c_int()
        n = self.L.ref_array(self.h, name.encode(), C.byref(ptr), C.byref(kind))
        if n < 0:
            raise KeyError(name)
        if n == 0 or not ptr.value:
            return np.zeros(0, dtype=np.float64 if kind.value == 0 else np.int32)
        ct = C.c_double if kind.value == 0 else C.c_int
        buf = C.cast(ptr, C.POINTER(ct * n)).contents
        return np.frombuffer(buf, dtype=np.float64 if kind.value == 0 else np.int32).copy()

    def set_array(self, name: str, values: np.ndarray):
        ptr = C.c_void_p()
        kind = C.c_int()
        n = self.L.ref_array(self.h, name.encode(), C.byref(ptr), C.byref(kind))
        if n <= 0:
            raise KeyError(name)
        dt = np.float64 if kind.value == 0 else np.int32
        v = np.ascontiguousarray(values, dtype=dt).ravel()
        if v.size != n:
            raise ValueError(f"{name}: expected {n} values, got {v.size}")
        C.memmove(ptr.value, v.ctypes.data, v.nbytes)

    def params(self) -> np.ndarray:
        out = (C.c_double * 25)()
        self.L.ref_params(self.h, out)
        return np.array(out)

    def segments(self):
        """[(b, [(n0, n1), ...]), ...] 1-based boundary segments bs[b][s]."""
        sc = self.scalars()
        res = []
        pair = (C.c_int * 2)()
        for b in range(1, sc["nb"] + 1):
            segs = []
            for s in range(1, self.L.ref_nbs(self.h, b) + 1):
                self.L.ref_segment(self.h, b, s, pair)
                segs.append((pair[0], pair[1]))
            res.append(segs)
        return res

    def svd(self, node: int):
        U = C.POINTER(C.c_double)()
        VT = C.POINTER(C.c_double)()
        S = C.POINTER(C.c_double)()
        m = self.L.ref_svd(self.h, node, C.byref(U), C.byref(VT), C.byref(S))
        if m == 0:
            return None
        u = np.ctypeslib.as_array(U, shape=(m * m,)).copy()
        vt = np.ctypeslib.as_array(VT, shape=(25,)).copy()
        s = np.ctypeslib.as_array(S, shape=(5,)).copy()
        return u, vt, s

    # ---- stages ----
    def solve(self, ts: int) -> float:
        return self.L.ref_solve(self.h, ts)

    def body_forces(self):
        f = (C.c_double * 2)()
        self.L.ref_body_forces(self.h, f)
        return f[0], f[1]

    def set_citer(self, c: int):
        self.L.ref_set_citer(self.h, c)

    def alloc_work(self):
        self.L.ref_alloc_work(self.h)

    def build_matrix(self):
        self.L.ref_build_matrix(self.h)

    def gradient(self):
        self.L.ref_gradient(self.h)

    def derivatives(self, order: int = 3):
        self.L.ref_derivatives(self.h, order)

    def limiter(self):
        self.L.ref_limiter(self.h)

    def interior(self, jupdate: int, ts: int):
        self.L.ref_interior(self.h, jupdate, ts)

    def boundary(self, jupdate: int):
        self.L.ref_boundary(self.h, jupdate)

    def set_boundary_values(self):
        self.L.ref_set_boundary_values(self.h)

    def linear_solve(self) -> float:
        return self.L.ref_linear_solve(self.h)

    def grow_stencils(self):
        self.L.ref_grow_stencils(self.h)

    def cfl(self) -> float:
        return self.L.ref_cfl(self.h)

    # ---- writers (grid_io.C) ----
    def write_surface_cp(self, directory: str):
        """write_surface_cp run in `directory` (its sort under LC_ALL=C)."""
        if self.L.ref_write_surface_cp(self.h, directory.encode()) != 0:
            raise RuntimeError(f"cannot enter {directory}")

    def write_mesh(self, path: str):
        """write_mesh: the mesh and the restart block of the current state."""
        self.L.ref_write_mesh(self.h, path.encode())

    def write_tecplot(self, path: str, primitive: bool = False):
        self.L.ref_write_tecplot(self.h, path.encode(), 1 if primitive else 0)
