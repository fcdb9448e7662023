"""The serving engine (flow_server over a flow_arena): solves of different
meshes, orders, flow conditions and precisions admitted together give, each,
the result the same solve gives alone (bit for bit: same steps, state and
forces), and admission respects the arena's budget."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MIX = [  # nc, nr, curved, order, mach, alpha, precision, subits
    (64, 16, True, 3, 0.8, 1.25, 1, 4),
    (32, 8, False, 1, 0.5, 1.25, 0, 2),
    (48, 12, True, 3, 0.6, -2.0, 0, 2),
    (96, 24, True, 3, 0.75, 3.0, 1, 3),
    (40, 10, False, 1, 0.4, 4.0, 1, 3),
]


def _case(nc, nr, curved, order, mach, alpha, subits):
    from flowgpu import workloads
    from flowgpu.prep import Mesh
    wl = workloads.Workload(f"srv{nc}x{nr}", nc, nr, curved, order, mach, alpha=alpha,
                            subits=subits, max_steps=400)
    mesh = Mesh.from_case(wl.write(), order=order)
    return wl, mesh


def test_mixed_admission_matches_solves_run_alone():
    from flowgpu import capi
    cases = [(_case(nc, nr, cv, o, m, a, sub), prec)
             for (nc, nr, cv, o, m, a, prec, sub) in MIX]
    alone = []
    for (wl, mesh), prec in cases:
        fp = wl.params()
        s = capi.Solver.from_mesh(mesh, fp, device=0)
        s.set_precision(prec)
        s.set_state(mesh.initial_state(fp))
        steps, r0, r1 = s.converge(1, wl.max_steps, 1e-10, chunk=32, check=False)
        assert s.status() == 0
        alone.append((steps, s.get("Q"), s.body_forces(), r1 < 1e-10 * r0))
        s.close()
    arena = capi.Arena(2 << 30)
    # larger meshes on higher-priority streams: scheduling only, same results
    srv = capi.Server(arena, chunk=16, max_slots=8, priority_policy=1)
    for i, ((wl, mesh), prec) in enumerate(cases):
        fp = wl.params()
        slot = srv.submit(mesh, fp, mesh.initial_state(fp), precision=prec, drop=1e-10,
                          max_steps=wl.max_steps, tag=i)
        assert slot is not None
    got = {}
    while srv.running() > 0 or len(got) < len(cases):
        for c in srv.progress(wait_us=2000):
            q, f = srv.result(c["slot"])
            got[c["tag"]] = (c, q, f)
            srv.release(c["slot"])
    for i, (steps, q, f, converged) in enumerate(alone):
        c, q2, f2 = got[i]
        assert c["steps"] == steps, (i, c["steps"], steps)
        assert c["status"] == (0 if converged else capi.ERR_NOT_CONVERGED)
        assert np.array_equal(q[4:], q2[4:]), i
        assert f == f2, i
    srv.close()
    arena.close()


def test_admission_waits_for_arena_room():
    from flowgpu import capi
    (wl, mesh) = _case(64, 16, True, 3, 0.8, 1.25, 4)
    fp = wl.params()
    probe = capi.Solver.from_mesh(mesh, fp, device=0)
    probe.set_precision(1)
    need = probe.L.flow_ctx_device_bytes(probe.ctx)
    probe.close()
    arena = capi.Arena(int(need * 1.5))  # room for one context, not two
    srv = capi.Server(arena, chunk=16, max_slots=4)
    s0 = srv.submit(mesh, fp, mesh.initial_state(fp), precision=1, max_steps=64)
    assert s0 is not None
    assert srv.submit(mesh, fp, mesh.initial_state(fp), precision=1, max_steps=64) is None
    done = []
    while not done:
        done = srv.progress(wait_us=5000)
    srv.release(done[0]["slot"])
    s1 = srv.submit(mesh, fp, mesh.initial_state(fp), precision=1, max_steps=64)
    assert s1 is not None
    while srv.running():
        for c in srv.progress(wait_us=5000):
            srv.release(c["slot"])
    srv.close()
    arena.close()


@pytest.mark.parametrize("rule", [None, (2.0, 1.4)])
def test_stalled_solves_are_retired_and_converging_ones_are_not(rule):
    """A k=1 solve caught in the limiter's limit cycle is retired as stalled
    long before its step limit; a converging solve served next to it takes
    exactly the steps it takes alone: with the fixed window (a tenfold drop
    within 600 steps) and with the size-scaled rule (a halving within
    max(160, 1.4 sqrt(nodes)) steps)."""
    from flowgpu import capi
    (wl1, m1) = _case(64, 16, False, 1, 0.5, 1.25, 2)
    (wl2, m2) = _case(32, 8, True, 3, 0.8, 1.25, 4)
    fp2 = wl2.params()
    alone = capi.Solver.from_mesh(m2, fp2, device=0)
    alone.set_precision(3)
    alone.set_state(m2.initial_state(fp2))
    steps2, r0, r1 = alone.converge(1, 3000, 1e-10, check=False)
    alone.close()
    assert r1 < 1e-10 * r0
    arena = capi.Arena(1 << 30)
    if rule is None:
        srv = capi.Server(arena, chunk=16, max_slots=4, stall=600)
    else:
        srv = capi.Server(arena, chunk=16, max_slots=4, stall=160, stall_drop=rule[0],
                          stall_per_sqrt=rule[1])
    fp1 = wl1.params()
    srv.submit(m1, fp1, m1.initial_state(fp1), precision=3, max_steps=3000, tag=1)
    srv.submit(m2, fp2, m2.initial_state(fp2), precision=3, max_steps=3000, tag=2)
    got = {}
    while len(got) < 2:
        for c in srv.progress(wait_us=5000):
            got[c["tag"]] = c
            srv.release(c["slot"])
    assert got[1]["status"] == capi.ERR_STALLED and got[1]["steps"] < 2000
    assert got[2]["status"] == 0 and got[2]["steps"] == steps2
    srv.close()
    arena.close()


def test_staged_meshes_of_different_sizes_all_start():
    """Contexts staged first and started afterwards (the largest chunk
    window not the last one built) all run: kernel launch limits are not a
    per-context setting."""
    from flowgpu import capi
    cases = [_case(128, 32, True, 3, 0.8, 1.25, 4), _case(32, 8, True, 3, 0.8, 1.25, 4)]
    arena = capi.Arena(1 << 30)
    srv = capi.Server(arena, chunk=16, max_slots=4)
    slots = []
    for wl, m in cases:
        fp = wl.params()
        slots.append(srv.submit(m, fp, m.initial_state(fp), precision=3, max_steps=64,
                                hold=True))
    for sl in slots:
        srv.start(sl)
    done = []
    while len(done) < 2:
        done += srv.progress(wait_us=5000)
    for c in done:
        assert c["status"] in (0, capi.ERR_NOT_CONVERGED)
        srv.release(c["slot"])
    srv.close()
    arena.close()


def test_concurrent_staging_from_threads_matches_solves_run_alone():
    """Requests staged from several host threads at once (autotuning at
    admission included), started while the other threads still stage, give
    the results each solve gives alone; a bucket is tuned once."""
    import concurrent.futures as cf
    from flowgpu import capi
    cases = [(_case(nc, nr, cv, o, m, a, sub), prec)
             for (nc, nr, cv, o, m, a, prec, sub) in MIX] + \
            [(_case(64, 16, True, 3, 0.7, 0.5, 4), 3), (_case(48, 12, False, 1, 0.6, 2.0, 3), 3)]
    alone = []
    for (wl, mesh), prec in cases:
        fp = wl.params()
        s = capi.Solver.from_mesh(mesh, fp, device=0)
        s.set_precision(prec)
        s.set_state(mesh.initial_state(fp))
        steps, r0, r1 = s.converge(1, wl.max_steps, 1e-10, chunk=32, check=False)
        alone.append((steps, s.get("Q"), s.body_forces()))
        s.close()
    arena = capi.Arena(2 << 30)
    srv = capi.Server(arena, chunk=16, max_slots=len(cases), autotune=2)

    def stage(i):
        (wl, mesh), prec = cases[i]
        fp = wl.params()
        slot = srv.submit(mesh, fp, mesh.initial_state(fp), precision=prec, drop=1e-10,
                          max_steps=wl.max_steps, tag=i)
        assert slot is not None
        return slot

    got = {}
    with cf.ThreadPoolExecutor(max_workers=4) as ex:
        futs = [ex.submit(stage, i) for i in range(len(cases))]
        while len(got) < len(cases):
            done = srv.progress(wait_us=2000)
            for c in done:
                q, f = srv.result(c["slot"])
                got[c["tag"]] = (c, q, f)
                srv.release(c["slot"])
            if not done and all(f.done() for f in futs) and srv.running() == 0 \
                    and len(got) < len(cases):
                break  # a stage call failed: its future raises below
        for f in futs:
            f.result()
    for i, (steps, q, f) in enumerate(alone):
        c, q2, f2 = got[i]
        assert c["steps"] == steps, (i, c["steps"], steps)
        assert np.array_equal(q[4:], q2[4:]), i
        assert f == f2, i
    srv.close()
    arena.close()


def test_poisson_stream_admits_from_worker_threads_and_retires_every_request():
    """The serving driver: requests prepared and admitted by worker threads
    while the main thread keeps the running solves going; every request is
    retired once, with its arrival-to-retirement latency."""
    from flowgpu import capi, serve
    reqs = [serve.sample_request(i, seed=5, n_min=2000, n_max=6000) for i in range(4)]
    arena = capi.Arena(1 << 30)
    r = serve.run_poisson(reqs, 50.0, arena, subits=4, max_steps=120, drop=1e-8, precision=3,
                          chunk=16, max_slots=4, seed=5, prep_threads=3, autotune=2, stall=0)
    arena.close()
    assert len(r["records"]) == 4
    for x in r["records"]:
        # converged, at max_steps, or retired on a non-physical state
        assert isinstance(x["status"], int) and 0 < x["steps"] <= 120
        assert x["latency_s"] > 0. and x["admitted_s"] >= 0.
        assert x["latency_s"] <= r["span_s"] + 1e-6


def test_arena_without_room_refuses_before_building_the_context():
    """An arena with less room than the mesh's state buffers refuses the
    context at once (a budget refusal, no host re-layout or upload first)."""
    import ctypes as C
    from flowgpu import capi
    (wl, mesh) = _case(64, 16, True, 3, 0.8, 1.25, 4)
    fp = wl.params()
    arena = capi.Arena(1 << 20)
    L = capi.load()
    st = C.c_int(0)
    p = capi.params_struct(fp)
    ctx = L.flow_create_in(arena.h, C.byref(mesh.view), C.byref(p), C.byref(st))
    assert not ctx and st.value == 512  # FLOW_ERR_BUDGET: no room in the arena now
    assert b"no room" in L.flow_last_error()
    srv = capi.Server(arena, chunk=16, max_slots=2)
    assert srv.submit(mesh, fp, mesh.initial_state(fp), precision=3, max_steps=8) is None
    assert srv.running() == 0
    srv.close()
    arena.close()


def _request44():
    """Request 44 of the 64-solve batch stream (seed 0): an 81,796-node k=2
    O-grid at Mach 0.677 whose approximate-Jacobian Newton steps go
    non-physical near step 550 of the CFL ramp; the FP64 drop-in and the
    forward-difference Jacobians converge it."""
    from flowgpu import serve, workloads
    bw = workloads.BATCHES["batch64"]
    return serve.prepare(serve.sample_request(44, seed=0), bw.subits, bw.max_steps, bw.drop)


def test_failed_approximate_jacobian_solve_rolls_back_and_converges():
    """The served solve goes back to its failed chunk's first step with the
    forward-difference Jacobians: its state is bit for bit that of a context
    run alone on the approximate Jacobians up to that step and on the
    forward-difference ones after it, and its forces are within 1e-8 of the
    FP64 drop-in's.  With recovery off it retires in that chunk with
    non-physical error bits, as the context alone fails."""
    from flowgpu import capi
    pr = _request44()
    mesh, fp, q0 = pr.mesh, pr.params, pr.Q0
    arena = capi.Arena(4 << 30)
    got = {}
    for recovery in (True, False):
        srv = capi.Server(arena, chunk=32, max_slots=2, jacobian=2, recovery=recovery)
        srv.submit(mesh, fp, q0, precision=3, drop=1e-10, max_steps=6000, tag=int(recovery))
        while int(recovery) not in got:
            for c in srv.progress(wait_us=5000):
                q, f = srv.result(c["slot"]) if c["status"] == 0 else (None, None)
                got[c["tag"]] = (c, q, f)
                srv.release(c["slot"])
        srv.close()
    c, q, f = got[1]
    assert c["status"] == 0 and c["recovered_at"] > 1, c
    s = c["recovered_at"]
    assert (s - 1) % 32 == 0
    # alone: approximate Jacobians for steps 1 .. s-1, forward differences after
    alone = capi.Solver.from_mesh(mesh, fp, device=0)
    alone.set_precision(3)
    alone.set_jacobian(2)
    alone.set_state(q0)
    alone.run(1, s - 1)
    alone.set_jacobian(0)
    alone.run(s, c["steps"] - s + 1)
    assert np.array_equal(alone.get("Q")[4:], q[4:])
    alone.close()
    fp64 = capi.Solver.from_mesh(mesh, fp, device=0)
    fp64.set_state(q0)
    fp64.converge(1, 6000, 1e-10, check=False)
    assert fp64.status() == 0
    f64 = fp64.body_forces()
    fp64.close()
    assert max(abs(f[0] - f64[0]), abs(f[1] - f64[1])) < 1e-8
    # recovery off: the error bits of the context alone
    c0 = got[0][0]
    assert c0["recovered_at"] == 0
    assert c0["status"] & capi.ERR_NONPHYSICAL and not c0["status"] & ~capi.ERR_NONPHYSICAL
    assert c0["steps"] < s + 32
    alone = capi.Solver.from_mesh(mesh, fp, device=0)
    alone.set_precision(3)
    alone.set_jacobian(2)
    alone.set_state(q0)
    alone.converge(1, 6000, 1e-10, chunk=32, check=False)
    assert alone.status() & capi.ERR_NONPHYSICAL
    alone.close()
    arena.close()
