"""GPU parity of the precision form (flow_set_precision(ctx, 1)): FP32
off-diagonal blocks and LU factors, multicolour block Gauss-Seidel sweeps.

The oracle restates the same arithmetic (FP32 rounding of the FP64
assembly, the same fused multiply-add order, reciprocal pivots) on the CPU,
so the bar is bit-for-bit equality of the iterates step by step.  A second
test runs both forms to a 1e-10 drop and compares the converged forces, the
precision form's contract: the converged answer is that of the FP64 form."""
import numpy as np
import pytest

from cases import chunk_order, ndiff

pytestmark = pytest.mark.gpu


def _setup(nc, nr, curved, order, subits, mode=1):
    from dataclasses import replace
    from flowgpu import capi, workloads
    from flowgpu.prep import Mesh
    from oracle import port
    wl = workloads.Workload(f"mixed{nc}x{nr}", nc, nr, curved, order, 0.8 if order == 3 else 0.5,
                            subits=subits)
    mesh = Mesh.from_case(wl.write(), order=order)
    fp = wl.params()
    Q0 = mesh.initial_state(fp)
    og = port.OracleGrid(mesh.sizes, mesh.arrays())
    og.set("Q", Q0)
    gpu = capi.Solver.from_mesh(mesh, fp, device=0)
    gpu.set_precision(mode)
    gpu.set_state(Q0)
    return mesh, fp, og, port.params_from_flow(fp), gpu


@pytest.mark.parametrize("nc,nr,curved,order,subits,steps,mode", [
    (32, 8, False, 1, 2, 6, 1),
    (32, 8, True, 3, 2, 6, 1),
    (128, 32, True, 3, 4, 4, 1),
    (64, 16, False, 1, 3, 4, 1),
    (32, 8, True, 3, 2, 6, 2),
    (128, 32, True, 3, 2, 4, 2),
    (64, 16, False, 1, 3, 4, 2),
    (8, 3, False, 1, 2, 5, 1),  # 24 nodes
    (12, 4, True, 3, 2, 5, 2),  # 48 nodes
])
def test_mixed_steps_bitwise(nc, nr, curved, order, subits, steps, mode):
    """mode 1: multicolour sweeps; mode 2: sweeps in the reference's row order."""
    mesh, fp, og, p, gpu = _setup(nc, nr, curved, order, subits, mode)
    nn = mesh.sizes["nn"]
    for ts in range(1, steps + 1):
        og.solve_mixed(p, ts, ordered=(mode == 2))
        gpu.solve(ts)
        for name in ("Q", "nQ"):
            assert ndiff(og[name][4:], gpu.get(name)[4:]) == 0, (name, ts)
        for name in ("R", "dQ"):
            assert ndiff(og[name][4:4 * (nn + 1)], gpu.get(name)[4:]) == 0, (name, ts)
        assert gpu.body_forces() == og.body_forces(p)
    assert gpu.status() == 0
    gpu.close()


@pytest.mark.parametrize("nc,nr,curved,order,subits,steps,rows,levels,ring,df", [
    (32, 8, True, 3, 4, 6, 0, 0, 0, 0),
    (128, 32, True, 3, 4, 4, 0, 0, 0, 0),
    (128, 32, True, 3, 4, 4, 0, 0, 32, 0),
    (128, 32, True, 3, 4, 4, 0, 0, 16, 0),
    (64, 16, False, 1, 3, 4, 64, 0, 16, 0),
    (128, 32, True, 3, 2, 3, 200, 6, 32, 0),
    (32, 8, True, 3, 4, 6, 0, 0, 0, 1),
    (128, 32, True, 3, 4, 4, 0, 0, 0, 1),
    (64, 16, False, 1, 3, 4, 64, 0, 0, 1),
    (128, 32, True, 3, 2, 3, 200, 6, 0, 1),
    (8, 3, False, 1, 3, 5, 0, 0, 0, 0),  # 24 nodes: one chunk
    (12, 4, True, 3, 4, 5, 0, 0, 0, 1),
])
def test_chunked_steps_bitwise(nc, nr, curved, order, subits, steps, rows, levels, ring, df):
    """mode 3: coloured chunks of the reference order, against the oracle's
    sweep in the same row permutation, for each ring shape of the sweep and
    with the one-launch (dataflow) sweep."""
    mesh, fp, og, p, gpu = _setup(nc, nr, curved, order, subits, 3)
    gpu.set_chunk(rows, levels)
    gpu.set_sweep_ring(ring)
    gpu.set_sweep_dataflow(bool(df))
    starts, ncol = gpu.chunk_starts()
    nn = mesh.sizes["nn"]
    perm, ncol2 = chunk_order(og["ia"], og["ja"], starts)
    assert ncol2 == ncol and sorted(perm.tolist()) == list(range(1, nn + 1))
    if rows:
        assert np.diff(starts).max() <= rows
    for ts in range(1, steps + 1):
        og.solve_mixed_order(p, ts, perm)
        gpu.solve(ts)
        for name in ("Q", "nQ"):
            assert ndiff(og[name][4:], gpu.get(name)[4:]) == 0, (name, ts)
        for name in ("R", "dQ"):
            assert ndiff(og[name][4:4 * (nn + 1)], gpu.get(name)[4:]) == 0, (name, ts)
    assert gpu.status() == 0
    gpu.close()


def test_mixed_converges_to_the_fp64_answer():
    from flowgpu import capi, workloads
    from flowgpu.prep import Mesh
    wl = workloads.Workload("mixedconv", 64, 16, True, 3, 0.8, subits=4)
    mesh = Mesh.from_case(wl.write(), order=3)
    fp = wl.params()
    out = {}
    for mode in (0, 1, 2, 3):
        s = capi.Solver.from_mesh(mesh, fp, device=0)
        s.set_precision(mode)
        s.set_state(mesh.initial_state(fp))
        steps, r0, r1 = s.converge(1, 20000, 1e-10)
        assert r1 < 1e-10 * r0
        out[mode] = (steps, s.body_forces(), s.get("Q"))
        s.close()
    n0, f0, q0 = out[0]
    for mode in (1, 2, 3):
        n1, f1, q1 = out[mode]
        assert abs(f1[0] - f0[0]) <= 1e-8 * max(1.0, abs(f0[0]))
        assert abs(f1[1] - f0[1]) <= 1e-8 * max(1.0, abs(f0[1]))
        assert np.max(np.abs(q1 - q0)) < 1e-7


def test_sweep_schedule_bitwise():
    """mode 3 with 2 sweeps up to step 3 and 4 after, against the oracle run
    with those sweep counts step by step."""
    import ctypes
    from oracle import port
    mesh, fp, og, p, gpu = _setup(64, 16, True, 3, 4, 3)
    gpu.set_sweep_schedule(2, 3)
    starts, ncol = gpu.chunk_starts()
    nn = mesh.sizes["nn"]
    perm, _ = chunk_order(og["ia"], og["ja"], starts)
    for ts in range(1, 7):
        p.subits = 2 if ts <= 3 else 4
        og.solve_mixed_order(p, ts, perm)
        gpu.solve(ts)
        assert ndiff(og["Q"][4:], gpu.get("Q")[4:]) == 0, ts
        assert ndiff(og["dQ"][4:4 * (nn + 1)], gpu.get("dQ")[4:]) == 0, ts
    gpu.close()


@pytest.mark.parametrize("jmode", [1, 2])
@pytest.mark.parametrize("nc,nr,curved,order,subits,steps,mode", [
    (32, 8, True, 3, 4, 6, 1),
    (64, 16, False, 1, 3, 5, 1),
    (32, 8, True, 3, 4, 6, 3),
    (128, 32, True, 3, 4, 4, 3),
    (64, 16, False, 1, 3, 5, 3),
    (8, 3, False, 1, 3, 4, 3),  # 24 nodes: less than one CTA of the fused kernel
])
def test_approximate_jacobian_steps_bitwise(nc, nr, curved, order, subits, steps, mode, jmode):
    """flow_set_jacobian: the interior face Jacobians by the approximate Roe
    form, fused with the assembly (1) or in two kernels (2), against the
    oracle's restatement step by step (the residual is the FP64 one; only the
    FP32 blocks differ from mode 0's)."""
    mesh, fp, og, p, gpu = _setup(nc, nr, curved, order, subits, mode)
    gpu.set_jacobian(jmode)
    p.jac_approx = 1
    nn = mesh.sizes["nn"]
    perm = None
    if mode == 3:
        starts, _ = gpu.chunk_starts()
        perm, _ = chunk_order(og["ia"], og["ja"], starts)
    for ts in range(1, steps + 1):
        if mode == 3:
            og.solve_mixed_order(p, ts, perm)
        else:
            og.solve_mixed(p, ts)
        gpu.solve(ts)
        for name in ("Q", "nQ"):
            assert ndiff(og[name][4:], gpu.get(name)[4:]) == 0, (name, ts)
        for name in ("R", "dQ"):
            assert ndiff(og[name][4:4 * (nn + 1)], gpu.get(name)[4:]) == 0, (name, ts)
    assert gpu.status() == 0
    gpu.close()


@pytest.mark.parametrize("order", [1, 3])
def test_approximate_jacobian_converges_to_the_fp64_answer(order):
    """The approximate Jacobian changes the preconditioner, not the residual:
    the converged forces are the FP64 drop-in's within 1e-8."""
    from flowgpu import capi, workloads
    from flowgpu.prep import Mesh
    wl = workloads.Workload(f"approxconv{order}", 64, 16, order == 3, order,
                            0.8 if order == 3 else 0.5, subits=4, limit=2 if order == 3 else 0)
    mesh = Mesh.from_case(wl.write(), order=order)
    fp = wl.params()
    out = {}
    for mode, jac in ((0, 0), (3, 1)):
        s = capi.Solver.from_mesh(mesh, fp, device=0)
        s.set_precision(mode)
        s.set_jacobian(jac)
        s.set_state(mesh.initial_state(fp))
        steps, r0, r1 = s.converge(1, 20000, 1e-10)
        assert r1 < 1e-10 * r0
        out[mode] = (steps, s.body_forces())
        s.close()
    (n0, f0), (n1, f1) = out[0], out[3]
    assert abs(f1[0] - f0[0]) <= 1e-8 * max(1.0, abs(f0[0]))
    assert abs(f1[1] - f0[1]) <= 1e-8 * max(1.0, abs(f0[1]))


@pytest.mark.parametrize("subits,ring,order", [(4, 0, 3), (3, 0, 3), (2, 32, 3), (4, 16, 1),
                                               (5, 0, 1)])
def test_paired_colour_passes_bitwise(subits, ring, order):
    """Mode 3 with a colour's two passes in a row as one launch (the default)
    against one launch per pass: the same iterates, step by step, with graph
    chunks, for several sweep counts and ring shapes."""
    from flowgpu import capi, workloads
    from flowgpu.prep import Mesh
    wl = workloads.Workload("pairs", 128, 32, order == 3, order, 0.8 if order == 3 else 0.5,
                            subits=subits)
    mesh = Mesh.from_case(wl.write(), order=order)
    fp = wl.params()
    out = []
    for pairs in (False, True):
        s = capi.Solver.from_mesh(mesh, fp, device=0)
        s.set_precision(3)
        s.set_sweep_ring(ring)
        s.set_sweep_pairs(pairs)
        s.set_state(mesh.initial_state(fp))
        steps, r0, r1 = s.converge(1, 200, 1e-10, chunk=16, check=False)
        out.append((steps, r0, r1, s.get("Q"), s.get("dQ"), s.status()))
        s.close()
    (n0, a0, b0, q0, d0, st0), (n1, a1, b1, q1, d1, st1) = out
    assert st0 == st1 and n0 == n1 and a0 == a1 and b0 == b1
    assert np.array_equal(q0, q1) and np.array_equal(d0, d1)
