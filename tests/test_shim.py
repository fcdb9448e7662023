"""The reference-side shim (flow-solver_b200/shim/solve_gpu.C: solve(),
Compute_Body_Forces() and write_surface_cp() forwarded to the C ABI) compiles against the reference's own headers and
include/flow_gpu.h with the reference's compiler flags (Makefile:19,
-ansi -pedantic; long long in the C ABI is allowed).  Skipped where the
reference's headers are not present.  CPU only."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM = os.path.join(ROOT, "flow-solver_b200", "shim", "solve_gpu.C")


STAGES = os.path.join(ROOT, "flow-solver_b200", "shim", "stages_gpu.C")


@pytest.mark.parametrize("src", [SHIM, STAGES])
def test_shim_compiles_against_the_reference_headers(src):
    import __graft_entry__
    ref_include = os.path.join(__graft_entry__.reference_dir(), "include")
    if not os.path.isdir(ref_include):
        pytest.skip("the reference's headers are not present")
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no g++")
    cmd = [gxx, "-ansi", "-pedantic", "-Wall", "-Wno-deprecated", "-Wno-long-long", "-Werror",
           "-fsyntax-only", "-I", ref_include, "-I", os.path.join(ROOT, "include"), src]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_stage_shim_keeps_the_reference_signatures():
    src = open(STAGES).read()
    for sig, target in [
            ("void build_matrix(GRID *grid, PARAMS p, SYS_MEM *smem)", "flow_build_matrix"),
            ("void build_interior_residuals(GRID *grid, SYS_MEM *smem, PARAMS p, int jupdate, "
             "int ts)", "FLOW_STAGE_INTERIOR"),
            ("void build_boundary_residuals(GRID *grid, SYS_MEM *smem, PARAMS p, int jupdate)",
             "FLOW_STAGE_BOUNDARY"),
            ("double linear_solve(GRID *grid, SYS_MEM *smem, PARAMS p)", "flow_linear_solve")]:
        assert sig in src, sig
        body = src[src.index(sig):]
        body = body[:body.index("\n}\n")]
        assert target in body, sig


def test_shim_forwards_every_replaced_reference_function():
    src = open(SHIM).read()
    for sig, target in [("double solve(GRID *grid, SYS_MEM *smem, PARAMS p, int ts)", "flow_solve"),
                        ("void Compute_Body_Forces(GRID *grid, PARAMS p, double *Forces)",
                         "flow_body_forces"),
                        ("void write_surface_cp(GRID *grid, PARAMS p)", "flow_write_surface_cp")]:
        assert sig in src
        body = src[src.index(sig):]
        body = body[:body.index("\n}\n")]
        assert target + "(" in body, sig
