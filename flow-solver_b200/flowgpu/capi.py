"""ctypes binding of libflowgpu.so (include/flow_gpu.h).

The solver only runs through the CUDA library: importing works without a
GPU, but constructing a ``Solver`` fails loudly when the library or a CUDA
device is missing.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import threading
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(HERE), "lib", "libflowgpu.so")

IP = C.POINTER(C.c_int)
DP = C.POINTER(C.c_double)
LP = C.POINTER(C.c_long)

ERRORS = {1: "ARG", 2: "CUDA", 4: "EIGEN", 8: "DT", 16: "LIMITER", 32: "BC",
          64: "SWEEP_TIMEOUT", 128: "NOT_FOUND", 256: "NOT_CONVERGED", 512: "BUDGET",
          1024: "STALLED"}
ERR_ARG = 1
ERR_NOT_CONVERGED = 256
ERR_BUDGET = 512
ERR_STALLED = 1024
ERR_SWEEP_TIMEOUT = 64
ERR_EIGEN = 4
ERR_DT = 8
ERR_LIMITER = 16
ERR_BC = 32
ERR_NONPHYSICAL = ERR_EIGEN | ERR_DT | ERR_LIMITER | ERR_BC

# exported symbols, in include/flow_gpu.h order
SYMBOLS = ("flow_create", "flow_destroy", "flow_set_state", "flow_solve", "flow_run",
           "flow_converge", "flow_converge_batch", "flow_build_matrix", "flow_reconstruct",
           "flow_residuals", "flow_residual_stage", "flow_linear_solve", "flow_body_forces", "flow_surface_cp",
           "flow_write_surface_cp", "flow_write_tecplot", "flow_write_restart", "flow_get",
           "flow_size", "flow_set",
           "flow_set_sweep_mode", "flow_set_precision", "flow_precision_of", "flow_set_chunk", "flow_set_sweep_ring", "flow_set_sweep_dataflow", "flow_chunk_starts", "flow_set_graphs",
           "flow_set_capture_fault", "flow_capture_fallbacks", "flow_set_jacobian",
           "flow_set_exact_rms", "flow_set_sweep_pairs",
           "flow_autotune", "flow_autotune_sweep", "flow_set_variants", "flow_set_sweep_schedule", "flow_save_state", "flow_restore_state", "flow_set_timing",
           "flow_kernel_times", "flow_stream", "flow_status", "flow_clear_status",
           "flow_last_error", "flow_launch_count", "flow_last_device_ms",
           "flow_linear_residual_noalloc", "flow_arena_create", "flow_arena_destroy",
           "flow_arena_free_bytes", "flow_arena_largest_free", "flow_create_in",
           "flow_ctx_device_bytes", "flow_server_create", "flow_server_destroy",
           "flow_server_submit", "flow_server_stage", "flow_server_start", "flow_server_progress", "flow_server_result",
           "flow_server_release", "flow_server_running", "flow_server_last_error",
           "flow_server_set_autotune", "flow_server_set_stall",
           "flow_server_set_sweep_schedule", "flow_set_stream_priority",
           "flow_server_set_priority_policy", "flow_server_set_jacobian",
           "flow_server_set_recovery", "flow_server_set_stall_rule",
           "flow_selftest_sweep_timeout")


class FlowParamsC(C.Structure):
    """struct flow_params (mirrors the reference's PARAMS)."""
    _fields_ = [("nsteps", C.c_int), ("iter", C.c_int), ("jufreq", C.c_int),
                ("CFL", C.c_double), ("ramp", C.c_int), ("gamma", C.c_double),
                ("alpha", C.c_double), ("mach", C.c_double), ("subits", C.c_int),
                ("unsteady", C.c_int), ("tacc", C.c_int), ("mintime", C.c_double),
                ("method", C.c_int), ("order", C.c_int), ("foits", C.c_int), ("soits", C.c_int),
                ("toits", C.c_int), ("isrestart", C.c_int), ("limit", C.c_int),
                ("reorder", C.c_int), ("ic", C.c_int), ("p_or_cv", C.c_int),
                ("start_post_pro", C.c_int), ("post_pro_freq", C.c_int)]


_VIEW_INTS = ("nn", "nn_ghost", "nedges", "nsubedges", "nbedges", "nb", "nelem")
_VIEW_IPTR = ("edges", "subedges", "bedges", "bedge_seg", "bbc", "node_order", "ia", "iau", "ja")
_VIEW_DPTR = ("x", "cv_area", "el_cent", "xn_subedges", "xm_subedges", "xg_subedges",
              "xn_bedges", "xg_bedges", "xgn_bedges", "edge_weight", "moments")
_VIEW_IPTR2 = ("gnsn", "gnnsn", "gnnsn1", "svd_m")


class FlowGridView(C.Structure):
    _fields_ = ([(n, C.c_int) for n in _VIEW_INTS]
                + [(n, IP) for n in _VIEW_IPTR]
                + [(n, DP) for n in _VIEW_DPTR]
                + [(n, IP) for n in _VIEW_IPTR2[:3]]
                + [("svd_m", IP), ("svd_off", LP), ("svd_U", DP), ("svd_VT", DP),
                   ("svd_S", DP)])


_lib = None


def library_path() -> str:
    return LIB_PATH


_load_lock = threading.Lock()


def load():
    """Load libflowgpu.so (raises if it has not been built).  Thread-safe:
    every caller gets the one handle, with every prototype set."""
    global _lib
    if _lib is not None:
        return _lib
    with _load_lock:
        if _lib is None:
            _lib = _load_locked()
    return _lib


def _load_locked():
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with flow-solver_b200/build.py")
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    PP = C.POINTER(FlowParamsC)
    L.flow_create.restype = vp
    L.flow_create.argtypes = [C.POINTER(FlowGridView), PP, C.c_int, IP]
    L.flow_destroy.argtypes = [vp]
    L.flow_set_state.argtypes = [vp, DP]
    L.flow_solve.argtypes = [vp, PP, C.c_int, DP, DP]
    L.flow_run.argtypes = [vp, PP, C.c_int, C.c_int, DP, DP]
    L.flow_converge.argtypes = [vp, PP, C.c_int, C.c_int, C.c_double, C.c_int, IP, DP, DP]
    L.flow_converge_batch.argtypes = [C.POINTER(vp), C.c_int, PP, C.c_int, C.c_int, C.c_double,
                                      C.c_int, IP, IP]
    L.flow_build_matrix.argtypes = [vp, PP, C.c_int]
    L.flow_reconstruct.argtypes = [vp, PP, C.c_int]
    L.flow_residuals.argtypes = [vp, PP, C.c_int, C.c_int]
    L.flow_residual_stage.argtypes = [vp, PP, C.c_int, C.c_int, C.c_int]
    L.flow_linear_solve.argtypes = [vp, PP, DP]
    L.flow_body_forces.argtypes = [vp, PP, DP]
    L.flow_surface_cp.argtypes = [vp, PP, C.c_int, IP, IP, C.c_int, IP, DP, C.c_int, IP]
    L.flow_write_surface_cp.argtypes = [vp, PP, C.c_char_p, C.c_int, IP, IP, IP, DP]
    L.flow_write_tecplot.argtypes = [vp, PP, C.c_char_p, C.c_int, DP, C.c_int, IP, C.c_int, IP]
    L.flow_write_restart.argtypes = [vp, PP, C.c_char_p, DP, C.c_int, IP, C.c_int, IP, C.c_int,
                                     IP, IP]
    L.flow_get.argtypes = [vp, C.c_char_p, DP, C.c_long]
    L.flow_size.restype = C.c_long
    L.flow_size.argtypes = [vp, C.c_char_p]
    L.flow_set.argtypes = [vp, C.c_char_p, DP, C.c_long]
    L.flow_set_sweep_mode.argtypes = [vp, C.c_int]
    L.flow_set_precision.argtypes = [vp, C.c_int]
    L.flow_precision_of.argtypes = [vp]
    L.flow_set_graphs.argtypes = [vp, C.c_int]
    L.flow_set_capture_fault.argtypes = [vp, C.c_int]
    L.flow_set_jacobian.argtypes = [vp, C.c_int]
    L.flow_set_exact_rms.argtypes = [vp, C.c_int]
    L.flow_set_sweep_pairs.argtypes = [vp, C.c_int]
    L.flow_capture_fallbacks.restype = C.c_long
    L.flow_capture_fallbacks.argtypes = [vp]
    L.flow_set_chunk.argtypes = [vp, C.c_int, C.c_int]
    L.flow_set_sweep_ring.argtypes = [vp, C.c_int]
    L.flow_set_sweep_dataflow.argtypes = [vp, C.c_int]
    L.flow_autotune.argtypes = [vp, PP, C.c_int, C.c_int, IP, DP]
    L.flow_set_variants.argtypes = [vp, C.c_int, C.c_int]
    L.flow_autotune_sweep.argtypes = [vp, PP, C.c_int, C.c_int, C.c_int, IP, DP]
    L.flow_set_sweep_schedule.argtypes = [vp, C.c_int, C.c_int]
    L.flow_chunk_starts.argtypes = [vp, IP, C.c_int, IP, IP]
    L.flow_save_state.argtypes = [vp]
    L.flow_restore_state.argtypes = [vp]
    L.flow_set_timing.argtypes = [vp, C.c_int]
    L.flow_kernel_times.argtypes = [vp, LP, DP, C.c_int]
    L.flow_stream.restype = vp
    L.flow_stream.argtypes = [vp]
    L.flow_status.argtypes = [vp]
    L.flow_clear_status.argtypes = [vp]
    L.flow_last_error.restype = C.c_char_p
    L.flow_launch_count.restype = C.c_long
    L.flow_launch_count.argtypes = [vp]
    L.flow_last_device_ms.restype = C.c_double
    L.flow_last_device_ms.argtypes = [vp]
    L.flow_linear_residual_noalloc.argtypes = [vp, vp, vp, vp, vp, C.c_int, C.c_long, vp, DP]
    L.flow_arena_create.restype = vp
    L.flow_arena_create.argtypes = [C.c_int, C.c_longlong, IP]
    L.flow_arena_destroy.argtypes = [vp]
    L.flow_arena_free_bytes.restype = C.c_longlong
    L.flow_arena_free_bytes.argtypes = [vp]
    L.flow_arena_largest_free.restype = C.c_longlong
    L.flow_arena_largest_free.argtypes = [vp]
    L.flow_create_in.restype = vp
    L.flow_create_in.argtypes = [vp, C.POINTER(FlowGridView), PP, IP]
    L.flow_ctx_device_bytes.restype = C.c_longlong
    L.flow_ctx_device_bytes.argtypes = [vp]
    L.flow_server_create.restype = vp
    L.flow_server_create.argtypes = [vp, C.c_int, C.c_int, IP]
    L.flow_server_destroy.argtypes = [vp]
    L.flow_server_submit.argtypes = [vp, C.POINTER(FlowGridView), PP, DP, C.c_int, C.c_double,
                                     C.c_int, C.c_longlong, IP]
    L.flow_server_stage.argtypes = [vp, C.POINTER(FlowGridView), PP, DP, C.c_int, C.c_double,
                                    C.c_int, C.c_longlong, C.c_int, IP]
    L.flow_server_start.argtypes = [vp, C.c_int]
    L.flow_server_progress.argtypes = [vp, C.c_int, C.POINTER(FlowCompletion), C.c_int, IP]
    L.flow_server_result.argtypes = [vp, C.c_int, DP, C.c_long, DP]
    L.flow_server_release.argtypes = [vp, C.c_int]
    L.flow_server_running.argtypes = [vp]
    L.flow_server_last_error.restype = C.c_char_p
    L.flow_server_set_autotune.argtypes = [vp, C.c_int]
    L.flow_server_set_stall.argtypes = [vp, C.c_int]
    L.flow_server_set_sweep_schedule.argtypes = [vp, C.c_int, C.c_int, C.c_longlong]
    L.flow_set_stream_priority.argtypes = [vp, C.c_int]
    L.flow_server_set_priority_policy.argtypes = [vp, C.c_int]
    L.flow_server_set_jacobian.argtypes = [vp, C.c_int]
    L.flow_server_set_recovery.argtypes = [vp, C.c_int]
    L.flow_server_set_stall_rule.argtypes = [vp, C.c_double, C.c_double]
    L.flow_selftest_sweep_timeout.argtypes = [vp, C.c_long, IP]
    # host preprocessing (include/flow_prep.h)
    L.flow_prep_read.restype = vp
    L.flow_prep_read.argtypes = [C.c_char_p, IP, C.c_int, C.c_int, C.c_int, IP]
    L.flow_prep_build.restype = vp
    L.flow_prep_build.argtypes = [C.c_int, DP, C.c_int, IP, C.c_int, IP, C.c_int, IP, IP, IP,
                                  C.c_int, C.c_int, IP]
    L.flow_prep_view.argtypes = [vp, C.POINTER(FlowGridView)]
    L.flow_prep_initial_state.argtypes = [vp, C.POINTER(FlowParamsC), DP]
    L.flow_prep_node_map.restype = IP
    L.flow_prep_node_map.argtypes = [vp]
    L.flow_prep_elements.argtypes = [vp, IP, C.POINTER(IP), IP, C.POINTER(IP)]
    L.flow_prep_restart_state.argtypes = [vp, DP, C.c_long, IP, DP]
    L.flow_prep_segments.argtypes = [vp, IP, C.POINTER(IP), C.POINTER(IP), C.POINTER(IP)]
    L.flow_prep_free.argtypes = [vp]
    L.flow_prep_last_error.restype = C.c_char_p
    return L


def linear_residual_noalloc(ia: int, ja: int, lhs: int, rhs: int, x: int, nn: int, nnz: int,
                            stream: int | None = None) -> float:
    """b - A x RMS of a BCSR system in caller-held device memory (device
    pointers as ints), through flow_linear_residual_noalloc: no device
    allocation, static scratch of FLOW_NOALLOC_MAX_ROWS rows."""
    L = load()
    r = C.c_double()
    _check(L.flow_linear_residual_noalloc(ia, ja, lhs, rhs, x, int(nn), int(nnz), stream,
                                          C.byref(r)), "flow_linear_residual_noalloc")
    return r.value


NOALLOC_MAX_ROWS = 262144


class FlowCompletion(C.Structure):
    _fields_ = [("tag", C.c_longlong), ("slot", C.c_int), ("status", C.c_int),
                ("steps", C.c_int), ("r_first", C.c_double), ("r_last", C.c_double),
                ("device_ms", C.c_double), ("launches", C.c_longlong),
                ("recovered_at", C.c_int)]


class Arena:
    """flow_arena: one device allocation that contexts are carved from."""

    def __init__(self, nbytes: int, device: int = 0):
        self.L = load()
        st = C.c_int(0)
        self.h = self.L.flow_arena_create(int(device), int(nbytes), C.byref(st))
        if not self.h:
            raise FlowError(st.value or 2, "flow_arena_create " + self.L.flow_last_error().decode())
        self.device = device

    def free_bytes(self) -> int:
        return self.L.flow_arena_free_bytes(self.h)

    def largest_free(self) -> int:
        return self.L.flow_arena_largest_free(self.h)

    def close(self):
        if getattr(self, "h", None):
            self.L.flow_arena_destroy(self.h)
            self.h = None


class Server:
    """flow_server: continuous batching of steady solves in an arena.

    submit() returns a slot or None when the arena / slot table is full
    (FLOW_ERR_BUDGET); progress() returns retired solves as dicts."""

    def __init__(self, arena: Arena, chunk: int = 32, max_slots: int = 64, autotune: int = 0,
                 stall: int = 0, ramp_sweeps: int = 0, ramp_min_nodes: int = 250000,
                 priority_policy: int = 0, jacobian: int = 0, recovery: bool = True,
                 stall_drop: float = 10., stall_per_sqrt: float = 0.):
        self.L = load()
        st = C.c_int(0)
        self.arena = arena
        self.h = self.L.flow_server_create(arena.h, int(chunk), int(max_slots), C.byref(st))
        if not self.h:
            raise FlowError(st.value or 1, "flow_server_create")
        if autotune:
            _check(self.L.flow_server_set_autotune(self.h, int(autotune)), "autotune")
        if stall:
            _check(self.L.flow_server_set_stall(self.h, int(stall)), "stall")
        if ramp_sweeps:
            _check(self.L.flow_server_set_sweep_schedule(self.h, int(ramp_sweeps), 0,
                                                         int(ramp_min_nodes)), "sweep schedule")
        if priority_policy:
            _check(self.L.flow_server_set_priority_policy(self.h, int(priority_policy)),
                   "priority policy")
        if jacobian:
            _check(self.L.flow_server_set_jacobian(self.h, int(jacobian)), "jacobian")
        if not recovery:
            _check(self.L.flow_server_set_recovery(self.h, 0), "recovery")
        if stall_drop != 10. or stall_per_sqrt:
            _check(self.L.flow_server_set_stall_rule(self.h, float(stall_drop),
                                                     float(stall_per_sqrt)), "stall rule")
        self._keep = {}
        self._out = (FlowCompletion * 64)()

    def submit(self, mesh, params, Q0, precision: int = 1, drop: float = 1e-10,
               max_steps: int = 20000, tag: int = 0, hold: bool = False):
        """hold: stage only (inputs uploaded); start(slot) launches it."""
        p = params_struct(params)
        q = np.ascontiguousarray(Q0, dtype=np.float64)
        slot = C.c_int(-1)
        rc = self.L.flow_server_stage(self.h, C.byref(mesh.view), C.byref(p),
                                      q.ctypes.data_as(DP), int(precision), float(drop),
                                      int(max_steps), int(tag), int(bool(hold)), C.byref(slot))
        if rc == ERR_BUDGET:
            return None
        if rc:
            err = self.L.flow_server_last_error().decode()
            if slot.value >= 0:  # a start that failed leaves a finished slot behind
                self.L.flow_server_release(self.h, slot.value)
            raise FlowError(rc, "flow_server_submit " + err)
        self._keep[slot.value] = (mesh, p)
        return slot.value

    def start(self, slot: int):
        _check(self.L.flow_server_start(self.h, int(slot)), "flow_server_start")

    def progress(self, wait_us: int = 0) -> list:
        n = C.c_int(0)
        _check(self.L.flow_server_progress(self.h, int(wait_us), self._out, len(self._out),
                                           C.byref(n)), "flow_server_progress")
        return [{"tag": c.tag, "slot": c.slot, "status": c.status, "steps": c.steps,
                 "r_first": c.r_first, "r_last": c.r_last, "device_ms": c.device_ms,
                 "launches": c.launches, "recovered_at": c.recovered_at}
                for c in self._out[:n.value]]

    def result(self, slot: int, want_q: bool = True):
        mesh, p = self._keep[slot]
        v = mesh.view
        q = np.zeros((v.nn + v.nn_ghost + 1) * 4) if want_q else None
        f = (C.c_double * 2)()
        _check(self.L.flow_server_result(self.h, slot, q.ctypes.data_as(DP) if want_q else None,
                                         q.size if want_q else 0, f), "flow_server_result")
        return q, (f[0], f[1])

    def release(self, slot: int):
        _check(self.L.flow_server_release(self.h, slot), "flow_server_release")
        self._keep.pop(slot, None)

    def running(self) -> int:
        return self.L.flow_server_running(self.h)

    def close(self):
        if getattr(self, "h", None):
            self.L.flow_server_destroy(self.h)
            self.h = None


def params_struct(fp) -> FlowParamsC:
    """fp: flowgpu.meshgen.FlowParams (or any object with the PARAMS fields)."""
    p = FlowParamsC()
    for name, ct in FlowParamsC._fields_:
        v = getattr(fp, name)
        setattr(p, name, float(v) if ct is C.c_double else int(v))
    return p


class FlowError(RuntimeError):
    def __init__(self, code: int, what: str = ""):
        names = [n for b, n in ERRORS.items() if code & b]
        msg = f"flow_gpu error {code} ({'|'.join(names) or '?'})"
        if what:
            msg += f": {what}"
        super().__init__(msg)
        self.code = code


def converge_batch(solvers, ts0: int = 1, max_steps: int = 20000, drop: float = 1e-10,
                   chunk: int = 64, check: bool = True):
    """flow_converge_batch over several Solver objects; returns (steps, status) lists."""
    L = load()
    n = len(solvers)
    arr = (C.c_void_p * n)(*[s.ctx for s in solvers])
    steps = (C.c_int * n)()
    st = (C.c_int * n)()
    rc = L.flow_converge_batch(arr, n, C.byref(solvers[0].p), ts0, max_steps, drop, chunk,
                               steps, st)
    if check:
        _check(rc, "flow_converge_batch")
    return list(steps), list(st)


def _check(rc: int, what: str = ""):
    if rc:
        err = load().flow_last_error()
        raise FlowError(rc, (what + " " + (err.decode() if err else "")).strip())


class Solver:
    """One device-resident mesh + state (a flow_ctx).

    ``arrays`` holds the grid in the reference's layout (see
    ``FlowGridView``); ``sizes`` its counts.
    """

    def __init__(self, sizes: dict, arrays: dict, params, device: int = 0):
        self.L = load()
        self._keep = {}
        v = FlowGridView()
        for n in _VIEW_INTS:
            setattr(v, n, int(sizes[n]))
        for n in _VIEW_IPTR + _VIEW_IPTR2:
            a = arrays.get(n)
            if a is not None:
                a = np.ascontiguousarray(a, dtype=np.int32)
                self._keep[n] = a
                setattr(v, n, a.ctypes.data_as(IP))
        for n in _VIEW_DPTR + ("svd_U", "svd_VT", "svd_S"):
            a = arrays.get(n)
            if a is not None:
                a = np.ascontiguousarray(a, dtype=np.float64)
                self._keep[n] = a
                setattr(v, n, a.ctypes.data_as(DP))
        off = arrays.get("svd_off")
        if off is not None:
            off = np.ascontiguousarray(off, dtype=np.int64)
            self._keep["svd_off"] = off
            v.svd_off = off.ctypes.data_as(LP)
        self.params = params
        self.p = params_struct(params)
        st = C.c_int(0)
        self.ctx = self.L.flow_create(C.byref(v), C.byref(self.p), int(device), C.byref(st))
        self._keep = None  # the library copied everything it needs
        if not self.ctx:
            _check(st.value or 1, "flow_create")
        self.sizes = dict(sizes)

    @classmethod
    def from_mesh(cls, mesh, params, device: int = 0):
        """Build from a flowgpu.prep.Mesh (the library's own preprocessing)."""
        self = cls.__new__(cls)
        self.L = load()
        self._keep = None
        self.params = params
        self.p = params_struct(params)
        st = C.c_int(0)
        self.ctx = self.L.flow_create(C.byref(mesh.view), C.byref(self.p), int(device), C.byref(st))
        if not self.ctx:
            _check(st.value or 1, "flow_create")
        self.sizes = mesh.sizes
        return self

    def close(self):
        if getattr(self, "ctx", None):
            self.L.flow_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def get_into(self, name: str, out: np.ndarray):
        """flow_get into a caller-owned float64 buffer (e.g. pinned memory)."""
        n = self.L.flow_size(self.ctx, name.encode())
        if n < 0 or out.dtype != np.float64 or out.size < n or not out.flags.c_contiguous:
            raise ValueError(f"bad output buffer for {name}")
        _check(self.L.flow_get(self.ctx, name.encode(), out.ctypes.data_as(DP), n), f"get {name}")

    def set_params(self, params):
        self.params = params
        self.p = params_struct(params)

    def set_state(self, Q: np.ndarray):
        Q = np.ascontiguousarray(Q, dtype=np.float64)
        _check(self.L.flow_set_state(self.ctx, Q.ctypes.data_as(DP)), "flow_set_state")

    def solve(self, ts: int):
        dq, rr = C.c_double(), C.c_double()
        _check(self.L.flow_solve(self.ctx, C.byref(self.p), ts, C.byref(dq), C.byref(rr)),
               f"flow_solve ts={ts}")
        return dq.value, rr.value

    def run(self, ts0: int, nsteps: int):
        rh = np.zeros(max(nsteps, 1))
        dh = np.zeros(max(nsteps, 1))
        _check(self.L.flow_run(self.ctx, C.byref(self.p), ts0, nsteps, rh.ctypes.data_as(DP),
                               dh.ctypes.data_as(DP)), "flow_run")
        return rh[:nsteps], dh[:nsteps]

    def converge(self, ts0: int = 1, max_steps: int = 20000, drop: float = 1e-10,
                 chunk: int = 64, check: bool = True):
        """Steps until ||R_rho|| drops by `drop`; returns (steps, r_first, r_last)."""
        n, r0, r1 = C.c_int(), C.c_double(), C.c_double()
        rc = self.L.flow_converge(self.ctx, C.byref(self.p), ts0, max_steps, drop, chunk,
                                  C.byref(n), C.byref(r0), C.byref(r1))
        if check:
            _check(rc, "flow_converge")
        return n.value, r0.value, r1.value

    def build_matrix(self, citer: int):
        _check(self.L.flow_build_matrix(self.ctx, C.byref(self.p), citer), "flow_build_matrix")

    def reconstruct(self, ts: int):
        _check(self.L.flow_reconstruct(self.ctx, C.byref(self.p), ts), "flow_reconstruct")

    def residuals(self, jupdate: int, ts: int):
        _check(self.L.flow_residuals(self.ctx, C.byref(self.p), jupdate, ts), "flow_residuals")

    STAGE_INTERIOR, STAGE_BOUNDARY = 1, 2

    def residual_stage(self, jupdate: int, ts: int, stage: int):
        """build_interior_residuals (stage 1) or build_boundary_residuals (2)."""
        _check(self.L.flow_residual_stage(self.ctx, C.byref(self.p), jupdate, ts, stage),
               "flow_residual_stage")

    def linear_solve(self) -> float:
        r = C.c_double()
        _check(self.L.flow_linear_solve(self.ctx, C.byref(self.p), C.byref(r)), "flow_linear_solve")
        return r.value

    def body_forces(self):
        f = (C.c_double * 2)()
        _check(self.L.flow_body_forces(self.ctx, C.byref(self.p), f), "flow_body_forces")
        return f[0], f[1]

    def surface_cp(self, mesh, b: int):
        """Nodes of boundary b in first-appearance order and their pressure
        coefficients (flow_surface_cp, computed on the device)."""
        nb, bbc, nbs, seg = mesh.segments()
        cap = int(nbs[b]) * 2 if 1 <= b <= nb else 0
        nodes = np.zeros(max(cap, 1), dtype=np.int32)
        cp = np.zeros(max(cap, 1))
        cnt = C.c_int(0)
        _check(self.L.flow_surface_cp(self.ctx, C.byref(self.p), nb, nbs.ctypes.data_as(IP),
                                      seg.ctypes.data_as(IP), int(b), nodes.ctypes.data_as(IP),
                                      cp.ctypes.data_as(DP), cap, C.byref(cnt)), "flow_surface_cp")
        return nodes[:cnt.value].copy(), cp[:cnt.value].copy()

    def write_surface_cp(self, mesh, directory: str):
        """surface_<b>_pressure.dat of every inviscid boundary into directory
        (write_surface_cp)."""
        nb, bbc, nbs, seg = mesh.segments()
        x = mesh.array("x")
        _check(self.L.flow_write_surface_cp(self.ctx, C.byref(self.p), directory.encode(), nb,
                                            bbc.ctypes.data_as(IP), nbs.ctypes.data_as(IP),
                                            seg.ctypes.data_as(IP), x.ctypes.data_as(DP)),
               "flow_write_surface_cp")

    def write_tecplot(self, mesh, path: str, primitive: bool = False):
        """Tecplot solution file of the current state (write_tecplot_solutionC,
        or write_tecplot_solutionP with primitive=True)."""
        tri, quad = mesh.elements()
        x = mesh.array("x")
        _check(self.L.flow_write_tecplot(self.ctx, C.byref(self.p), path.encode(),
                                         1 if primitive else 0, x.ctypes.data_as(DP),
                                         len(tri) // 3 - 1, tri.ctypes.data_as(IP),
                                         len(quad) // 4 - 1, quad.ctypes.data_as(IP)),
               "flow_write_tecplot")

    def write_restart(self, mesh, path: str):
        """The mesh with the restart block of the current state (write_mesh)."""
        tri, quad = mesh.elements()
        nb, bbc, nbs, seg = mesh.segments()
        x = mesh.array("x")
        _check(self.L.flow_write_restart(self.ctx, C.byref(self.p), path.encode(),
                                         x.ctypes.data_as(DP), len(tri) // 3 - 1,
                                         tri.ctypes.data_as(IP), len(quad) // 4 - 1,
                                         quad.ctypes.data_as(IP), nb, nbs.ctypes.data_as(IP),
                                         seg.ctypes.data_as(IP)), "flow_write_restart")

    def get(self, name: str) -> np.ndarray:
        n = self.L.flow_size(self.ctx, name.encode())
        if n < 0:
            raise KeyError(name)
        out = np.zeros(n)
        _check(self.L.flow_get(self.ctx, name.encode(), out.ctypes.data_as(DP), n), f"get {name}")
        return out

    def set(self, name: str, values: np.ndarray):
        """Copy a named array into the context (flow_set, reference layout)."""
        v = np.ascontiguousarray(values, dtype=np.float64)
        _check(self.L.flow_set(self.ctx, name.encode(), v.ctypes.data_as(DP), v.size),
               f"set {name}")

    def set_precision(self, mode: int):
        """0: FP64 reference-order drop-in; 1: FP32 blocks, multicolour sweeps;
        2: FP32 blocks, sweeps in the reference's row order; 3: FP32 blocks,
        coloured chunks of the reference order."""
        _check(self.L.flow_set_precision(self.ctx, int(mode)), "flow_set_precision")

    def set_chunk(self, rows: int = 0, levels: int = 0):
        """Chunk limits of precision mode 3 (0: defaults)."""
        _check(self.L.flow_set_chunk(self.ctx, int(rows), int(levels)), "flow_set_chunk")

    def set_sweep_ring(self, rows: int = 0):
        """Sub-level rows of the mode 3 sweep's prefetch ring (64, 32, 16)."""
        _check(self.L.flow_set_sweep_ring(self.ctx, int(rows)), "flow_set_sweep_ring")

    def set_sweep_dataflow(self, on: bool = True):
        """One launch per mode 3 sweep, chunks started by their dependencies."""
        _check(self.L.flow_set_sweep_dataflow(self.ctx, 1 if on else 0),
               "flow_set_sweep_dataflow")

    def chunk_starts(self):
        """(first row of each mode 3 chunk plus nn+1, number of colours)."""
        n, k = C.c_int(), C.c_int()
        _check(self.L.flow_chunk_starts(self.ctx, None, 0, C.byref(n), C.byref(k)),
               "flow_chunk_starts")
        out = np.zeros(n.value + 1, dtype=np.int32)
        _check(self.L.flow_chunk_starts(self.ctx, out.ctypes.data_as(IP), out.size, C.byref(n),
                                        C.byref(k)), "flow_chunk_starts")
        return out, k.value

    def autotune(self, ts: int = 2, steps: int = 4):
        """Pick the fastest kernel variants on this mesh; returns
        ((node_prepare variant, flux variant), per-variant ms)."""
        v = (C.c_int * 2)()
        ms = (C.c_double * 11)()
        _check(self.L.flow_autotune(self.ctx, C.byref(self.p), int(ts), int(steps), v, ms),
               "flow_autotune")
        return (v[0], v[1]), [round(x, 4) for x in ms]

    def autotune_sweep(self, ts: int = 2, steps: int = 4, allow_df: bool = False):
        """Pick the fastest mode 3 sweep shape; returns (rows + 1000*one_launch, ms)."""
        ch = C.c_int(0)
        ms = (C.c_double * 4)()
        _check(self.L.flow_autotune_sweep(self.ctx, C.byref(self.p), int(ts), int(steps),
                                          int(bool(allow_df)), C.byref(ch), ms),
               "flow_autotune_sweep")
        return ch.value, [round(x, 4) for x in ms]

    def set_sweep_schedule(self, sweeps: int, until_step: int = 0):
        """`sweeps` Gauss-Seidel sweeps up to `until_step` (0: end of the CFL ramp)."""
        _check(self.L.flow_set_sweep_schedule(self.ctx, int(sweeps), int(until_step)),
               "flow_set_sweep_schedule")

    def selftest_sweep_timeout(self, max_spin: int = 4096) -> int:
        """Run a sweep whose first row never runs; returns the status bits it
        left (FLOW_ERR_SWEEP_TIMEOUT when the bounded waits work)."""
        st = C.c_int(0)
        _check(self.L.flow_selftest_sweep_timeout(self.ctx, int(max_spin), C.byref(st)),
               "flow_selftest_sweep_timeout")
        return st.value

    def set_variants(self, node_prepare: int, flux: int):
        _check(self.L.flow_set_variants(self.ctx, int(node_prepare), int(flux)),
               "flow_set_variants")

    def set_graphs(self, on: bool):
        """Replay full chunks of flow_converge steps from CUDA graphs (default on)."""
        _check(self.L.flow_set_graphs(self.ctx, int(bool(on))), "flow_set_graphs")

    def set_jacobian(self, mode: int):
        """Precision-form face Jacobians: 0 forward differences, 1 approximate Roe."""
        _check(self.L.flow_set_jacobian(self.ctx, int(mode)), "flow_set_jacobian")

    def set_sweep_pairs(self, on: bool):
        """Mode 3: a colour's two passes in a row as one launch (default on)."""
        _check(self.L.flow_set_sweep_pairs(self.ctx, int(bool(on))), "flow_set_sweep_pairs")

    def set_exact_rms(self, on: bool):
        """Sum every b-Ax RMS in the reference's row order (flow_set_exact_rms)."""
        _check(self.L.flow_set_exact_rms(self.ctx, int(bool(on))), "flow_set_exact_rms")

    def set_capture_fault(self, count: int):
        """Test hook: discard the next `count` chunk captures (eager fallback)."""
        _check(self.L.flow_set_capture_fault(self.ctx, int(count)), "flow_set_capture_fault")

    def capture_fallbacks(self) -> int:
        """Chunks launched eagerly after a failed (or discarded) capture."""
        return self.L.flow_capture_fallbacks(self.ctx)

    def set_sweep_mode(self, mode: int):
        _check(self.L.flow_set_sweep_mode(self.ctx, int(mode)), "flow_set_sweep_mode")

    def save_state(self):
        _check(self.L.flow_save_state(self.ctx), "flow_save_state")

    def restore_state(self):
        _check(self.L.flow_restore_state(self.ctx), "flow_restore_state")

    def set_timing(self, on: bool):
        _check(self.L.flow_set_timing(self.ctx, int(bool(on))), "flow_set_timing")

    KERNEL_CLASSES = ("node_prepare", "subedge_flux", "boundary", "assemble", "sweep",
                      "lin_residual", "other")

    def kernel_times(self) -> dict:
        n = len(self.KERNEL_CLASSES)
        cnt = (C.c_long * n)()
        ms = (C.c_double * n)()
        _check(self.L.flow_kernel_times(self.ctx, cnt, ms, n), "flow_kernel_times")
        return {k: (cnt[i], ms[i]) for i, k in enumerate(self.KERNEL_CLASSES)}

    def stream(self) -> int:
        return self.L.flow_stream(self.ctx)

    def status(self) -> int:
        return self.L.flow_status(self.ctx)

    def launch_count(self) -> int:
        return self.L.flow_launch_count(self.ctx)

    def last_device_ms(self) -> float:
        return self.L.flow_last_device_ms(self.ctx)
