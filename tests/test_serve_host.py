"""Host-side pieces of the batching/serving forms (no GPU): the seeded
request stream, latency percentiles, the longest-first packing used for the
CPU reference arm, and the algorithmic-byte formulas of the roofline."""
import math

import numpy as np


def test_request_stream_is_seeded_per_index_and_in_range():
    from flowgpu import serve
    a = [serve.sample_request(i) for i in range(200)]
    b = [serve.sample_request(i) for i in range(200)]
    assert a == b
    assert serve.sample_request(5, seed=1) != serve.sample_request(5, seed=0)
    for r in a:
        assert r.nc % 2 == 0 and abs(r.nc - 4 * r.nr) <= 2
        assert 0.3 <= r.mach <= 0.85 and -4.0 <= r.alpha <= 6.0
        assert r.order in (1, 3)
        assert 1500 <= r.nodes <= 230000
    logs = np.log([r.nodes for r in a])
    assert math.log(2000) - 0.3 < logs.min() and logs.max() < math.log(200000) + 0.3
    assert {r.order for r in a} == {1, 3}


def test_percentiles_and_longest_first_packing():
    import bench
    from flowgpu import serve
    p = serve.percentiles(list(range(1, 101)))
    assert p["p50"] == 50.5 and p["p99"] > 99.0
    assert serve.percentiles([])["p50"] is None
    assert bench._lpt_makespan([5, 4, 3, 3, 3], 2) == 10  # 5+3 | 4+3+3
    assert bench._lpt_makespan([1, 1, 1], 8) == 1


def test_plain_fp64_takes_the_recorded_run_that_solves_soonest():
    from flowgpu import serve
    ms = {2: 1.0, 4: 1.7}
    # both converge: 4 sweeps take fewer steps but cost more a step
    assert serve.fastest_recorded_run([(2, 1000, 0), (4, 500, 0)], ms) == (4, 500, 0)
    assert serve.fastest_recorded_run([(2, 1000, 0), (4, 700, 0)], ms) == (2, 1000, 0)
    # a converged run beats a faster one that fails or stops at max_steps
    assert serve.fastest_recorded_run([(2, 3000, 0), (4, 64, 44)], ms) == (2, 3000, 0)
    assert serve.fastest_recorded_run([(2, 8000, 256), (4, 900, 0)], ms) == (4, 900, 0)
    # none converges: the cheapest of them
    assert serve.fastest_recorded_run([(2, 8000, 256), (4, 64, 44)], ms) == (4, 64, 44)


def test_roofline_approximate_jacobian_halves_the_face_blocks():
    from flowgpu import roofline, workloads
    from flowgpu.prep import Mesh
    wl = workloads.Workload("rl_a", 64, 16, True, 3, 0.8)
    m = Mesh.from_case(wl.write(), order=3)
    ns = m.sizes["ns"] if "ns" in m.sizes else m.sizes["nsubedges"]
    assert roofline.subedge_flux_bytes(m) - roofline.subedge_flux_bytes(m, approx=True) == 128 * ns
    assert roofline.assemble_bytes(m, 3, approx=True) < roofline.assemble_bytes(m, 3)


def test_roofline_bytes_scale_with_the_mesh():
    from flowgpu import roofline, workloads
    from flowgpu.prep import Mesh
    small = workloads.Workload("rl_s", 32, 8, True, 3, 0.8)
    big = workloads.Workload("rl_b", 64, 16, True, 3, 0.8)
    ms = Mesh.from_case(small.write(), order=3)
    mb = Mesh.from_case(big.write(), order=3)
    bs, bb = roofline.node_prepare_bytes(ms), roofline.node_prepare_bytes(mb)
    assert 1500 < bs / ms.sizes["nn"] < 3500
    assert 3.0 < bb / bs < 5.0
    assert roofline.colour_sweep_bytes(mb) > 0 and roofline.ordered_sweep_bytes(mb) > 0
