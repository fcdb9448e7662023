"""The C ABI library loads without a GPU and exports every function that
include/flow_gpu.h declares; argument checking works without a device."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    txt = open(os.path.join(ROOT, "include", "flow_gpu.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(flow_[a-z_]+)\s*\(", txt)))


def test_header_lists_the_binding_symbols():
    from flowgpu import capi
    assert set(declared_functions()) == set(capi.SYMBOLS)


def test_library_exports_every_declared_symbol():
    from flowgpu import capi
    lib = ctypes.CDLL(capi.library_path())
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_null_arguments_are_rejected_without_a_device():
    from flowgpu import capi
    L = capi.load()
    st = ctypes.c_int(0)
    assert L.flow_create(None, None, 0, ctypes.byref(st)) is None
    assert st.value == 1
    assert L.flow_solve(None, None, 1, None, None) == 1
    assert L.flow_size(None, b"Q") == -1
    assert b"null" in L.flow_last_error()


def test_setters_reject_bad_arguments_without_a_device():
    from flowgpu import capi
    L = capi.load()
    assert L.flow_set_sweep_ring(None, 64) == 1
    assert b"rows not 0, 16, 32 or 64" in L.flow_last_error()
    assert L.flow_set_chunk(None, 0, 0) == 1
    assert L.flow_surface_cp(None, None, 0, None, None, 1, None, None, 0, None) == 1
    assert L.flow_write_tecplot(None, None, None, 0, None, 0, None, 0, None) == 1
