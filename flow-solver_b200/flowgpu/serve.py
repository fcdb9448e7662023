"""Batching and serving of steady solves on one GPU (flow_server in an arena).

Request streams follow the batching / serving forms of the workload family:
mesh node counts log-uniform in [n_min, n_max] with a 4:1 circumferential to
radial ratio (same airfoil family and seeded diagonals/jitter as the single
meshes), free-stream Mach uniform in [0.3, 0.85], angle of attack uniform in
[-4, 6] degrees, reconstruction order k=1 (straight walls) or k=2 (curved
walls), all drawn from one numpy PCG64 seed per request index.

Host preprocessing (mesh generation, then flow_prep_build on the generated
arrays: ordering, stencils, SVD) runs in a thread pool (the C library
releases the GIL) and overlaps the GPU.
"""
from __future__ import annotations

import concurrent.futures as cf
import math
import threading
import time
from dataclasses import dataclass, replace

import numpy as np

from . import capi, workloads
from .prep import Mesh


@dataclass(frozen=True)
class Request:
    index: int
    nc: int
    nr: int
    order: int
    mach: float
    alpha: float

    @property
    def nodes(self) -> int:
        return self.nc * self.nr

    def workload(self, subits: int, max_steps: int, drop: float) -> workloads.Workload:
        return workloads.Workload(f"req{self.index}_{self.nc}x{self.nr}_k{1 if self.order == 1 else 2}",
                                  self.nc, self.nr, self.order == 3, self.order, self.mach,
                                  alpha=self.alpha, subits=subits, max_steps=max_steps,
                                  drop=drop, seed=1000 + self.index)


def sample_request(index: int, seed: int = 0, n_min: int = 2000, n_max: int = 200000,
                   orders=(1, 3)) -> Request:
    """Request `index` of stream `seed` (independent of every other index)."""
    rng = np.random.Generator(np.random.PCG64([seed, index]))
    n = math.exp(rng.uniform(math.log(n_min), math.log(n_max)))
    nr = max(8, int(round(math.sqrt(n / 4.0))))
    nc = max(32, 2 * int(round(2.0 * nr)))  # even, 4:1
    mach = float(rng.uniform(0.3, 0.85))
    alpha = float(rng.uniform(-4.0, 6.0))
    order = int(orders[rng.integers(len(orders))])
    return Request(index, nc, nr, order, round(mach, 6), round(alpha, 6))


@dataclass
class Prepared:
    req: Request
    wl: workloads.Workload
    mesh: Mesh
    params: object
    Q0: np.ndarray
    prep_s: float


def prepare(req: Request, subits: int, max_steps: int, drop: float) -> Prepared:
    """Generate the request's grid and preprocess it in memory (no mesh file:
    flow_prep_build gives the arrays flow_prep_read would give for it)."""
    t0 = time.perf_counter()
    wl = req.workload(subits, max_steps, drop)
    mesh = Mesh.from_grid(wl.grid(), order=wl.order)
    fp = wl.params()
    return Prepared(req, wl, mesh, fp, mesh.initial_state(fp), time.perf_counter() - t0)


def prepare_all(reqs, subits: int, max_steps: int, drop: float, threads: int = 8):
    capi.load()  # bind once before the worker threads use it
    with cf.ThreadPoolExecutor(max_workers=threads) as ex:
        return list(ex.map(lambda r: prepare(r, subits, max_steps, drop), reqs))


def fastest_recorded_run(runs, ms_per_step) -> tuple:
    """The FP64 drop-in's run of one request that solves it soonest.

    runs: (sweeps, steps, status) per recorded sweep count; ms_per_step:
    {sweeps: measured ms per step}.  Runs that converged (status 0) are
    preferred; among them (or among all, when none converged) the one with
    the least steps x ms/step.  Returns (sweeps, steps, status)."""
    pool = [r for r in runs if r[2] == 0] or list(runs)
    return min(pool, key=lambda r: r[1] * ms_per_step[r[0]])


def percentiles(xs, ps=(50, 95, 99)) -> dict:
    if not xs:
        return {f"p{p}": None for p in ps}
    a = np.asarray(xs, dtype=np.float64)
    return {f"p{p}": float(np.percentile(a, p)) for p in ps}


def run_batch(prepared, arena: capi.Arena, precision: int = 1, chunk: int = 32,
              max_slots: int = 64, want_q: bool = False, autotune: int = 0,
              stall: int = 0, ramp_sweeps: int = 0, priority_policy: int = 0) -> dict:
    """Admit every prepared solve (as the arena allows), run all to
    retirement.  Returns per-solve records and the makespan."""
    srv = capi.Server(arena, chunk=chunk, max_slots=max_slots, autotune=autotune, stall=stall,
                      ramp_sweeps=ramp_sweeps, priority_policy=priority_policy)
    pending = list(range(len(prepared)))
    recs = {}
    t0 = time.perf_counter()
    submit_t = {}
    while pending or srv.running() > 0:
        while pending:
            i = pending[0]
            pr = prepared[i]
            slot = srv.submit(pr.mesh, pr.params, pr.Q0, precision=precision, drop=pr.wl.drop,
                              max_steps=pr.wl.max_steps, tag=i)
            if slot is None:
                break
            submit_t[i] = time.perf_counter()
            pending.pop(0)
        for c in srv.progress(wait_us=500):
            i = c["tag"]
            q, f = (None, None)
            if c["status"] in (0, capi.ERR_NOT_CONVERGED, capi.ERR_STALLED):  # not of a failed one
                q, f = srv.result(c["slot"], want_q=want_q)
            srv.release(c["slot"])
            now = time.perf_counter()
            recs[i] = dict(c, latency_s=now - t0, service_s=now - submit_t[i], forces=f, Q=q)
    makespan = time.perf_counter() - t0
    srv.close()
    return {"records": [recs[i] for i in range(len(prepared))], "makespan_s": makespan}


def run_sequential(prepared, precision: int = 0, chunk: int = 64, device: int = 0) -> dict:
    """Each solve alone, one after the other (the plain drop-in usage)."""
    recs = []
    t0 = time.perf_counter()
    for pr in prepared:
        s = capi.Solver.from_mesh(pr.mesh, pr.params, device=device)
        s.set_precision(precision)
        s.set_state(pr.Q0)
        ts = time.perf_counter()
        steps, r0, r1 = s.converge(1, pr.wl.max_steps, pr.wl.drop, chunk=chunk, check=False)
        st = s.status()
        f = s.body_forces() if st == 0 else None
        recs.append({"steps": steps, "r_first": r0, "r_last": r1,
                     "status": st if st else (0 if r1 < pr.wl.drop * r0 else capi.ERR_NOT_CONVERGED),
                     "seconds": time.perf_counter() - ts, "device_ms": s.last_device_ms(),
                     "forces": f})
        s.close()
    return {"records": recs, "total_s": time.perf_counter() - t0}


def run_poisson(reqs, rate_per_s: float, arena: capi.Arena, subits: int, max_steps: int,
                drop: float, precision: int = 1, chunk: int = 32, max_slots: int = 64,
                seed: int = 0, prep_threads: int = 8, autotune: int = 0,
                stall: int = 0, ramp_sweeps: int = 0, jacobian: int = 0,
                stall_drop: float = 10., stall_per_sqrt: float = 0.) -> dict:
    """Open-loop Poisson arrivals at `rate_per_s`: each request is prepared
    on arrival by a worker thread, which then admits it (stages its context
    on the device and starts it) as soon as the arena has room; the main
    thread only keeps the running solves' chunks in flight and retires them.
    Latency = retirement - arrival."""
    rng = np.random.Generator(np.random.PCG64([seed, 7]))
    gaps = rng.exponential(1.0 / rate_per_s, size=len(reqs))
    arrivals = np.cumsum(gaps) - gaps[0]
    capi.load()
    srv = capi.Server(arena, chunk=chunk, max_slots=max_slots, autotune=autotune, stall=stall,
                      ramp_sweeps=ramp_sweeps, jacobian=jacobian, stall_drop=stall_drop,
                      stall_per_sqrt=stall_per_sqrt)
    recs = [dict() for _ in reqs]
    lock = threading.Lock()
    room = threading.Condition(lock)  # signalled whenever a solve is released
    t0 = time.perf_counter()

    def admit(i):
        pr = prepare(reqs[i], subits, max_steps, drop)
        while True:
            slot = srv.submit(pr.mesh, pr.params, pr.Q0, precision=precision, drop=drop,
                              max_steps=max_steps, tag=i)
            if slot is not None:
                break
            with room:  # the arena or the slot table is full: wait for a release
                room.wait(timeout=0.05)
        with lock:
            recs[i].update(admitted_s=time.perf_counter() - t0 - arrivals[i], prep_s=pr.prep_s,
                           nodes=reqs[i].nodes, order=reqs[i].order)

    ex = cf.ThreadPoolExecutor(max_workers=prep_threads)
    futures = []
    nxt = done = 0
    while done < len(reqs):
        now = time.perf_counter() - t0
        while nxt < len(reqs) and arrivals[nxt] <= now:
            futures.append(ex.submit(admit, nxt))
            nxt += 1
        for c in srv.progress(wait_us=500 if srv.running() else 0):
            i = c["tag"]
            f = None
            if c["status"] in (0, capi.ERR_NOT_CONVERGED, capi.ERR_STALLED):
                _, f = srv.result(c["slot"], want_q=False)
            srv.release(c["slot"])
            with room:
                recs[i].update(c, forces=f, latency_s=time.perf_counter() - t0 - arrivals[i])
                room.notify_all()
            done += 1
        for fut in futures:
            if fut.done() and fut.exception() is not None:
                raise fut.exception()  # a request could not be prepared or admitted
        if not srv.running():
            time.sleep(0.001)
    ex.shutdown()
    span = time.perf_counter() - t0
    srv.close()
    return {"records": recs, "span_s": span, "arrivals": arrivals.tolist()}
