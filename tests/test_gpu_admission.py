"""Continuous admission under load, as the batching bench serves it: the
first 16 requests of the seeded request stream (meshes of 2k..124k nodes,
k=1 and k=2, precision mode 3, autotuning at admission, stream priority by
mesh size) admitted from 8 host threads, largest first, while the main
thread keeps the running solves' chunks in flight (graph captures) and reads
each state back as its solve retires.  Context creation, pinned allocations
and context teardown on some threads overlap graph captures on others; every
solve must still give the steps and state it gives alone, pass after pass."""
import concurrent.futures as cf

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N_REQ = 16
MAX_STEPS = 256
SUBITS = 4
THREADS = 8


def _prepared():
    from flowgpu import serve
    reqs = [serve.sample_request(i, seed=0) for i in range(N_REQ)]
    return serve.prepare_all(reqs, SUBITS, MAX_STEPS, 1e-10)


def _alone(pr):
    from flowgpu import capi
    s = capi.Solver.from_mesh(pr.mesh, pr.params, device=0)
    try:
        s.set_precision(3)
    except capi.FlowError:
        s.set_precision(1)  # what the server does for a mesh mode 3 cannot take
    s.set_state(pr.Q0)
    steps, r0, r1 = s.converge(1, MAX_STEPS, 1e-10, chunk=32, check=False)
    st = s.status() or (0 if r1 < 1e-10 * r0 else capi.ERR_NOT_CONVERGED)
    q = s.get("Q")
    s.close()
    return steps, st, q


def _stream_pass(prep, arena):
    from flowgpu import capi
    srv = capi.Server(arena, chunk=32, max_slots=N_REQ, autotune=4, priority_policy=1)
    got = {}

    def admit(i):
        while True:
            slot = srv.submit(prep[i].mesh, prep[i].params, prep[i].Q0, precision=3,
                              drop=1e-10, max_steps=MAX_STEPS, tag=i)
            if slot is not None:
                return slot

    with cf.ThreadPoolExecutor(max_workers=THREADS) as ex:
        order = sorted(range(len(prep)), key=lambda i: -prep[i].req.nodes)
        futs = [ex.submit(admit, i) for i in order]
        while len(got) < len(prep):
            for c in srv.progress(wait_us=500):
                q = None
                if c["status"] in (0, capi.ERR_NOT_CONVERGED):
                    q, _f = srv.result(c["slot"], want_q=True)
                srv.release(c["slot"])
                got[c["tag"]] = (c, q)
            for f in futs:
                if f.done() and f.exception() is not None:
                    raise f.exception()
        for f in futs:
            f.result()
    srv.close()
    return got


def test_threaded_admission_of_the_batch_matches_solves_run_alone():
    from flowgpu import capi
    prep = _prepared()
    assert max(p.req.nodes for p in prep) > 100_000
    alone = [_alone(pr) for pr in prep]
    arena = capi.Arena(16 << 30)
    for _ in range(3):
        got = _stream_pass(prep, arena)
        for i, (steps, st, q) in enumerate(alone):
            c, q2 = got[i]
            # a request that turns non-physical does so alone too, at the same step
            assert c["status"] == st, (i, c["status"], st)
            assert c["steps"] == steps, (i, c["steps"], steps)
            if q2 is not None:
                assert np.array_equal(q[4:], q2[4:]), i
    arena.close()
