#!/usr/bin/env python3
"""Converged steady solves per second of the flow solver's nonlinear iteration.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl flow|reference]
                    [--workload NAME]

Default workload: the batching form ``batch64`` -- 64 independent steady
solves per GPU from the seeded request stream (meshes of 2k..200k nodes,
log-uniform, 4:1 O-grids; Mach 0.3..0.85, angle of attack -4..6 degrees,
k=1 or k=2), admitted together to the serving engine (one device arena, one
stream per solve, CUDA-graph chunks of pseudo-time steps) in the precision
form (FP64 residual, FP32 blocks, Gauss-Seidel in coloured chunks of the
reference order; approximate Roe face Jacobians, with a one-chunk roll-back
to the forward-difference ones for a solve they drive non-physical), each
retired at a 1e-10 drop of ||R_rho||, at its step limit or when it stalls.
A "step" of this benchmark is one pass over the batch.

* value: converged solves / device time of the passes (CUDA events), with
  every mesh and initial state already on the device (staged).
* e2e: the same through the C ABI from host buffers, served continuously:
  requests admitted from host threads (mesh arrays and state copied to the
  device), started as they land, every state and the lift/drag forces read
  back as each solve retires, all inside the timed region.
* latency: p50/p95/p99 of the per-solve device time from start to retirement.
* plain_fp64: the same requests solved one at a time by the FP64 drop-in
  (bit-identical to the reference), modelled: the recorded FP64 step count
  of each request x its measured FP64 ms/step, at whichever recorded sweep
  count (2 or 4 per step) solves it soonest; two requests are also solved
  to convergence in the run and the model's error on them is printed.
* roofline: the kernel class with the largest share of a step (node
  preparation, face fluxes, assembly or the chunk sweeps) on the batch's
  largest mesh that the FP64 drop-in solves, compulsory bytes over its
  measured duration against the measured HBM copy bandwidth.
* cpu_baseline: the reference (oracle/_ref, built from its own sources) on
  one host core, timed on the smallest meshes of the batch and scaled by node
  count to every request's recorded step count.

Single-mesh workloads (``--workload ogrid512x128_k2_m080`` ...) time the
plain FP64 drop-in: one solve per step, value = solves/s.

Multi-GPU (torchrun, one process per GPU): each rank serves its own requests
(the batch's next 16 of the stream), value = all ranks' converged solves /
the slowest rank's time ("scaling": "weak"); no device collective.

--impl reference times the reference's own CPU solver on all host cores,
rank 0 only.
"""
from __future__ import annotations

import dataclasses
import argparse
import concurrent.futures as cf
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
# many solves share the GPU, one stream each: let their kernels overlap
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
PKG = os.path.join(ROOT, "flow-solver_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

METRIC = "converged solves/s (1e-10 drop) served vs plain FP64 GPU; p50/p99 latency"
UNIT = "solves/s"
REF_SAMPLE_STEPS = 2        # pseudo-time steps per reference-arm bench step
BENCH_BUDGET_S = 1500.      # wall-clock target of a whole batch run (warm-up and checks included)
SERVE_RATES = (0.5, 2.0)    # requests/s of the serving measurement in the batch run
SERVE_REQUESTS = 16
# stall retirement of the serving runs (as batch64's): no halving of the best
# residual within max(160, 1.4 sqrt(nodes)) steps
SERVE_STALL, SERVE_STALL_DROP, SERVE_STALL_PER_SQRT = 160, 2.0, 1.4
SERVE_MIN_LEFT_S = 200.     # run the serving measurement only with this much time left
REF_ARM_TIMEOUT_S = 900     # bound on the reference arm's whole sample
STAGE_THREADS = max(1, min(8, os.cpu_count() or 1))  # concurrent admissions per batch pass
CPU_BASELINE_STEPS = 6      # pseudo-time steps timed for cpu_baseline


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during a timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(prefix="clocks_", suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        rows = []
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) >= 9:
                    rows.append(f)
        except Exception:
            pass
        finally:
            if self.path and os.path.exists(self.path):
                os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = sorted(float(r[1]) for r in rows if r[1].replace(".", "").isdigit())
        mx = max((float(r[2]) for r in rows if r[2].replace(".", "").isdigit()), default=None)
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v == "Active"})
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(rows)}


def measured_peaks() -> tuple[dict, str]:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def ncu_traffic_per_sweep(workload: str):
    """DRAM bytes of one sweep launch from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as f:
            return json.load(f).get(workload, {}).get("sweep_dram_bytes_per_launch")
    except Exception:
        return None


# ---------------------------------------------------------------------------
def dist_setup(n_gpus: int):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("gloo", timeout=timedelta(seconds=600))
        pg = dist
    return world, rank, local, pg


def allreduce_max(pg, v: float) -> float:
    if pg is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def allreduce_sum(pg, v: float) -> float:
    if pg is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.SUM)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


# ---------------------------------------------------------------------------
def run_flow(args):
    import numpy as np
    import torch
    from flowgpu import capi, workloads
    from flowgpu.prep import Mesh

    world, rank, local, pg = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    wl = workloads.get(args.workload)
    params = wl.params()
    casedir = wl.write(tempfile.mkdtemp(prefix=f"bench_r{rank}_"))
    t0 = time.time()
    mesh = Mesh.from_case(casedir, order=wl.order)
    prep_s = time.time() - t0
    solver = capi.Solver.from_mesh(mesh, params, device=local)
    solver.set_sweep_mode(args.sweep_mode)
    sizes = mesh.sizes
    nnz = int(mesh.array("ia")[sizes["nn"] + 1])
    Q0 = mesh.initial_state(params)
    q_pin = torch.from_numpy(Q0.copy()).pin_memory()
    out_pin = torch.empty_like(q_pin).pin_memory()
    q_np, out_np = q_pin.numpy(), out_pin.numpy()
    stream = torch.cuda.ExternalStream(solver.stream(), device=torch.device("cuda", local))

    def solve_e2e(ev):
        """One end-to-end solve; ev = 4 events: before the H2D copy, after
        it, after convergence, after the D2H copies."""
        ev[0].record(stream)
        solver.set_state(q_np)                      # H2D from pinned memory
        ev[1].record(stream)
        n, r0, r1 = solver.converge(1, wl.max_steps, wl.drop)
        ev[2].record(stream)
        solver.get_into("Q", out_np)                # D2H of the converged state
        f = solver.body_forces()                    # D2H of lift/drag
        ev[3].record(stream)
        return n, f

    def events():
        return [torch.cuda.Event(enable_timing=True) for _ in range(4)]

    steps_conv = None
    for i in range(args.warmup):
        n, forces = solve_e2e(events())
        steps_conv = n if steps_conv is None else steps_conv
        if n != steps_conv:
            raise RuntimeError(f"non-deterministic step count {n} != {steps_conv}")
    log(f"[rank {rank}] {wl.name}: nn={sizes['nn']} steps_to_converge={steps_conv} prep={prep_s:.2f}s")

    # ---- timed region: K end-to-end solves.  value = the device span with
    # the inputs resident (after the H2D copy, before the D2H copies);
    # e2e = the whole span including the copies. ----
    launches0 = solver.launch_count()
    solver.set_timing(True)
    barrier(pg)
    torch.cuda.synchronize()
    evs = [events() for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        for k in range(args.steps):
            n, forces = solve_e2e(evs[k])
        torch.cuda.synchronize()
    dev_ms = sum(e[1].elapsed_time(e[2]) for e in evs)
    e2e_ms = sum(e[0].elapsed_time(e[3]) for e in evs)
    ktimes = solver.kernel_times()
    solver.set_timing(False)
    launches = solver.launch_count() - launches0
    barrier(pg)

    dev_ms_max = allreduce_max(pg, dev_ms)
    e2e_ms_max = allreduce_max(pg, e2e_ms)
    total_solves = args.steps * world
    value = total_solves / (dev_ms_max / 1e3)
    e2e = total_solves / (e2e_ms_max / 1e3)

    # ---- roofline of the ordered sweep (largest share of a step) ----
    peaks, peak_kind = measured_peaks()
    cnt, ms = ktimes["sweep"]
    sweep_ms = ms / max(cnt, 1)
    bytes_per_sweep = 132 * nnz + 96 * sizes["nn"]
    achieved = bytes_per_sweep / (sweep_ms * 1e-3) / 1e9
    share = ms / max(sum(v[1] for v in ktimes.values()), 1e-30)
    traffic = ncu_traffic_per_sweep(wl.name)
    roofline = {"bound": "hbm", "kernel": "k_sweep_ordered", "achieved": round(achieved, 2),
                "peak": peaks["hbm_gbs"], "peak_kind": peak_kind, "unit": "GB/s",
                "frac": round(achieved / peaks["hbm_gbs"], 5), "traffic": traffic,
                "algorithmic_bytes_per_launch": bytes_per_sweep,
                "avg_launch_ms": round(sweep_ms, 4), "share_of_step": round(share, 3),
                "note": "the sweep is latency-bound (one dependency level at a time)"}
    kernels = {k: {"launches": c, "avg_ms": round(t / max(c, 1), 4)} for k, (c, t) in ktimes.items()}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(casedir, steps_conv)

    if rank == 0:
        q_bytes = 8 * Q0.size
        line = {
            "metric": METRIC, "value": round(value, 5), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(dev_ms_max / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": wl.name, "mesh": f"O-grid {wl.nc}x{wl.nr}, NACA 0012, "
                       f"seeded jitter+diagonals (seed {wl.seed})", "nodes": sizes["nn"],
                       "order": "k=2 (SVD pseudo-inverse)", "mach": wl.mach, "alpha": wl.alpha,
                       "cfl": "ramp 1->10->1e4 (ramp=1111)", "gs_sweeps": wl.subits,
                       "drop": wl.drop, "pseudo_steps_per_solve": steps_conv,
                       "sweep_mode": "ordered (reference order, bit-exact)",
                       "l2": "working set larger than L2 (matrix 58 MB + face Jacobians 100 MB)",
                       "parallelism": f"replicas x{world}"},
            "e2e": {"value": round(e2e, 5), "unit": UNIT, "h2d_bytes_per_step": q_bytes,
                    "d2h_bytes_per_step": q_bytes + 16},
            "roofline": roofline, "kernels": kernels, "gpu_launches": int(launches),
            "clocks": clk.summary(), "cpu_baseline": cpu,
            "forces": {"lift": forces[0], "drag": forces[1]},
        }
        print(json.dumps(line), flush=True)
    solver.close()
    if pg is not None:
        pg.destroy_process_group()


def ncu_traffic(workload: str, key: str):
    """DRAM bytes per launch of a kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as f:
            return json.load(f).get(workload, {}).get(key)
    except Exception:
        return None


def _view_bytes(mesh) -> int:
    """Bytes of the grid arrays a caller passes through flow_grid_view."""
    return int(sum(a.nbytes for a in mesh.arrays().values() if a is not None))


def _lpt_makespan(times, workers: int) -> float:
    """Makespan of independent jobs on `workers` identical workers, longest
    job first to the least loaded worker."""
    loads = [0.0] * max(1, workers)
    for t in sorted(times, reverse=True):
        k = loads.index(min(loads))
        loads[k] += t
    return max(loads)


def run_batch(args, bw):
    import numpy as np
    import torch
    from flowgpu import capi, roofline, serve

    t_run0 = time.time()
    world, rank, local, pg = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    reqs = [serve.sample_request(rank * bw.n + i, seed=bw.seed) for i in range(bw.n)]
    t0 = time.time()
    prep = serve.prepare_all(reqs, bw.subits, bw.max_steps, bw.drop)
    prep_s = time.time() - t0
    free, _total = torch.cuda.mem_get_info(local)
    arena_bytes = int(min(free * 0.85, 150e9))
    arena = capi.Arena(arena_bytes, device=local)
    h2d = sum(_view_bytes(p.mesh) + p.Q0.nbytes for p in prep)
    d2h = sum(p.Q0.nbytes + 16 for p in prep)
    log(f"[rank {rank}] {bw.name}: {bw.n} requests, {sum(r.nodes for r in reqs)} nodes, "
        f"host preprocessing {prep_s:.1f}s")

    def one_pass():
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        srv = capi.Server(arena, chunk=bw.chunk, max_slots=bw.n, autotune=bw.autotune,
                          stall=bw.stall, priority_policy=bw.priority_policy,
                          jacobian=bw.jacobian, stall_drop=bw.stall_drop,
                          stall_per_sqrt=bw.stall_per_sqrt)
        torch.cuda.synchronize()
        ev[0].record()
        # context + mesh arrays + state to the device, several requests at a
        # time (the server stages concurrently from host threads)
        with cf.ThreadPoolExecutor(max_workers=STAGE_THREADS) as ex:
            futs = [ex.submit(srv.submit, pr.mesh, pr.params, pr.Q0, precision=bw.precision,
                              drop=bw.drop, max_steps=bw.max_steps, tag=i, hold=True)
                    for i, pr in enumerate(prep)]
            slots = [f.result() for f in futs]
        if any(sl is None for sl in slots):
            raise RuntimeError("the device arena cannot hold the whole batch")
        torch.cuda.synchronize()
        ev[1].record()
        for sl in slots:
            srv.start(sl)
        recs = {}
        while len(recs) < len(slots):
            for c in srv.progress(wait_us=500):
                recs[c["tag"]] = c
        torch.cuda.synchronize()
        ev[2].record()
        forces = {}
        for i, c in recs.items():  # converged states and forces back to the host
            if c["status"] in (0, capi.ERR_NOT_CONVERGED, capi.ERR_STALLED):
                _q, forces[i] = srv.result(c["slot"], want_q=True)
            srv.release(c["slot"])
        ev[3].record()
        torch.cuda.synchronize()
        srv.close()
        return ([recs[i] for i in range(len(slots))], forces,
                ev[1].elapsed_time(ev[2]), ev[0].elapsed_time(ev[3]))

    def stream_pass():
        # end to end as a user serves the batch: every request admitted from
        # a host thread and started as soon as its inputs are on the device,
        # each state and force read back as its solve retires
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        srv = capi.Server(arena, chunk=bw.chunk, max_slots=bw.n, autotune=bw.autotune,
                          stall=bw.stall, priority_policy=bw.priority_policy,
                          jacobian=bw.jacobian, stall_drop=bw.stall_drop,
                          stall_per_sqrt=bw.stall_per_sqrt)
        torch.cuda.synchronize()
        ev[0].record()
        recs = {}
        room = threading.Condition()  # signalled at every release

        def admit(i):
            # an admission the server refuses (no room or slot now) waits for
            # a release and tries again; its message is kept for the line
            deadline = time.perf_counter() + 120.
            while True:
                sl = srv.submit(prep[i].mesh, prep[i].params, prep[i].Q0,
                                precision=bw.precision, drop=bw.drop,
                                max_steps=bw.max_steps, tag=i)
                if sl is not None:
                    return sl
                msg = srv.L.flow_server_last_error().decode()
                refusals.append(msg)
                if time.perf_counter() > deadline:
                    raise RuntimeError("admission refused for 120 s: " + msg)
                with room:
                    room.wait(timeout=0.05)

        with cf.ThreadPoolExecutor(max_workers=STAGE_THREADS) as ex:
            # largest meshes first: the longest solves set the pass's span
            by_size = sorted(range(len(prep)), key=lambda i: -prep[i].req.nodes)
            futs = [ex.submit(admit, i) for i in by_size]
            while len(recs) < len(prep):
                done = srv.progress(wait_us=500)
                for c in done:
                    if c["status"] in (0, capi.ERR_NOT_CONVERGED, capi.ERR_STALLED):
                        srv.result(c["slot"], want_q=True)
                    srv.release(c["slot"])
                    recs[c["tag"]] = c
                if done:
                    with room:
                        room.notify_all()
                for f in futs:
                    if f.done() and f.exception() is not None:
                        raise f.exception()
                if not done and srv.running() == 0:
                    time.sleep(0.0005)
        torch.cuda.synchronize()
        ev[1].record()
        torch.cuda.synchronize()
        srv.close()
        return [recs[i] for i in range(len(prep))], ev[0].elapsed_time(ev[1])

    first = None
    pass_s = []
    for _ in range(args.warmup):
        tw = time.time()
        recs, _f, _a, _b = one_pass()
        pass_s.append(time.time() - tw)
        sig = [(r["status"], r["steps"]) for r in recs]
        if first is None:
            first = sig
        elif sig != first:
            raise RuntimeError("non-deterministic batch: step counts differ between passes")
    # the first pass also tunes the kernel variants of every size bucket
    t_pass = (sum(pass_s[1:]) / len(pass_s[1:])) if len(pass_s) > 1 else (pass_s[0] if pass_s
                                                                           else 0.)
    log(f"[rank {rank}] {bw.name}: warm-up passes {[round(x, 1) for x in pass_s]} s")
    barrier(pg)
    dev_ms = e2e_ms = 0.
    lat, launches, n_conv, n_fail, n_stall = [], 0, 0, 0, 0
    evals, node_evals = 0, 0  # residual(+Jacobian) evaluations: one per served step
    dforce = []
    with ClockSampler(local) as clk:
        for k in range(args.steps):
            recs, forces, v_ms, e_ms = one_pass()
            if bw.fp64_forces is not None and rank == 0:
                for i, r in enumerate(recs):  # converged in both forms
                    if r["status"] == 0 and bw.fp64_status[i] == 0 and i in forces:
                        f64 = bw.fp64_forces[i]
                        dforce.append(max(abs(forces[i][0] - f64[0]), abs(forces[i][1] - f64[1])))
            dev_ms += v_ms
            e2e_ms += e_ms
            lat += [r["device_ms"] / 1e3 for r in recs]
            launches += sum(r["launches"] for r in recs)
            evals += sum(r["steps"] for r in recs)
            node_evals += sum(r["steps"] * prep[i].req.nodes for i, r in enumerate(recs))
            n_conv += sum(1 for r in recs if r["status"] == 0)
            n_fail += sum(1 for r in recs
                          if r["status"] not in (0, capi.ERR_NOT_CONVERGED, capi.ERR_STALLED))
            n_stall += sum(1 for r in recs if r["status"] == capi.ERR_STALLED)
        stream_ms = 0.
        refusals = []
        # the streamed (end-to-end) passes repeat the value passes' work from
        # host buffers; as many as the run's time target leaves room for, at
        # least 3 and at most K (every rank runs the same number)
        # room kept for the FP64 model, the CPU baseline and the serving runs
        left = BENCH_BUDGET_S - (time.time() - t_run0) - 120. - SERVE_MIN_LEFT_S
        n_e2e = int(max(3, min(args.steps, left // max(1.1 * t_pass, 1e-3))))
        n_e2e = int(allreduce_max(pg, n_e2e)) if pg is not None else n_e2e
        log(f"[rank {rank}] {bw.name}: value passes done at {time.time() - t_run0:.0f} s; "
            f"{n_e2e} streamed passes")
        for k in range(n_e2e):
            recs, ms = stream_pass()
            if first is not None and [(r["status"], r["steps"]) for r in recs] != first:
                raise RuntimeError("non-deterministic batch: streamed pass differs")
            stream_ms += ms
    barrier(pg)
    dev_ms_max = allreduce_max(pg, dev_ms)
    e2e_ms_max = allreduce_max(pg, e2e_ms)
    stream_ms_max = allreduce_max(pg, stream_ms)
    n_conv_all = allreduce_sum(pg, n_conv)
    evals_all = allreduce_sum(pg, evals)
    node_evals_all = allreduce_sum(pg, node_evals)
    value = n_conv_all / (dev_ms_max / 1e3)
    # a streamed pass converges the same solves as a value pass (checked above)
    e2e = n_conv_all / max(args.steps, 1) * n_e2e / (stream_ms_max / 1e3)
    e2e_staged = n_conv_all / (e2e_ms_max / 1e3)

    # ---- roofline, on rank 0 only: its requests are the ones whose FP64
    # statuses are recorded (other ranks serve other requests of the stream) ----
    def roofline_lines():
        # the kernel class with the largest share of the step on the largest
        # mesh of the batch, served form
        # the served configuration of that mesh: its precision form and Jacobian,
        # the kernel variants the autotuner picks for it
        # (the largest one whose solve stays physical: some requests of the stream
        # reach a non-physical state within a few steps, in the reference too)
        ok = [i for i in range(len(prep)) if bw.fp64_status is None
              or bw.fp64_status[i] in (0, capi.ERR_NOT_CONVERGED)]
        big = max((prep[i] for i in ok), key=lambda p: p.req.nodes)
        s = capi.Solver.from_mesh(big.mesh, big.params, device=local)
        s.set_precision(bw.precision)
        s.set_jacobian(bw.jacobian)
        s.set_state(big.Q0)
        variants, _ = s.autotune(ts=2, steps=4)
        s.run(1, 8)
        s.set_timing(True)
        s.run(9, 24)
        kt = s.kernel_times()
        s.close()
        peaks, peak_kind = measured_peaks()
        fused = bw.jacobian == 1 and bw.precision != 0
        approx = bw.jacobian != 0 and bw.precision != 0
        # algorithmic bytes per launch of each kernel class (flowgpu/roofline.py)
        names = {"node_prepare": "k_node_stage" if variants[0] == 3 else "k_node_prepare4",
                 "subedge_flux": "k_faces_assemble" if fused else "k_subedge_flux",
                 "assemble": "k_assemble4"}
        per_launch = {"node_prepare": roofline.node_prepare_bytes(big.mesh),
                      "subedge_flux": (roofline.faces_assemble_bytes(big.mesh) if fused else
                                       roofline.subedge_flux_bytes(big.mesh, approx=approx)),
                      "assemble": roofline.assemble_bytes(big.mesh, bw.precision, approx=approx)}
        if bw.precision == 3:  # one sweep: its colour launches
            names["sweep"] = "k_sweep_chunk (one sweep)"
            per_launch["sweep"] = roofline.chunk_sweep_bytes(big.mesh)
        total_ms = max(sum(v[1] for v in kt.values()), 1e-30)
        top = max(per_launch, key=lambda k: kt[k][1])  # the class with the largest device time
        cnt, ms = kt[top]
        k_ms = ms / max(cnt, 1)
        achieved = per_launch[top] / (k_ms * 1e-3) / 1e9
        roof = {"bound": "hbm", "kernel": names[top], "mesh": f"{big.req.nc}x{big.req.nr}",
                "achieved": round(achieved, 1), "peak": peaks["hbm_gbs"], "peak_kind": peak_kind,
                "unit": "GB/s", "frac": round(achieved / peaks["hbm_gbs"], 4),
                "traffic": ncu_traffic(f"{bw.name}:{big.req.nc}x{big.req.nr}",
                                       f"{names[top]}_dram_bytes"),
                "algorithmic_bytes_per_launch": per_launch[top], "avg_launch_ms": round(k_ms, 4),
                "share_of_step": round(ms / total_ms, 3), "variants": list(variants),
                "others": {names[k]: {"avg_launch_ms": round(kt[k][1] / max(kt[k][0], 1), 4),
                                      "achieved_gbs": round(per_launch[k] / max(
                                          kt[k][1] / max(kt[k][0], 1), 1e-9) * 1e-6, 1),
                                      "share_of_step": round(kt[k][1] / total_ms, 3)}
                           for k in per_launch if k != top and kt[k][0]},
                "kernels_ms": {k: round(t / max(c, 1), 4) for k, (c, t) in kt.items() if c}}
        scnt, sms = kt["sweep"]
        if bw.precision == 3 and scnt:
            sw_bytes = roofline.chunk_sweep_bytes(big.mesh)
            sw_ms = sms / scnt
            sw_ach = sw_bytes / (sw_ms * 1e-3) / 1e9
            roof_sweep = {"bound": "latency (dependency levels inside a chunk)",
                          "kernel": "k_sweep_chunk (one sweep = one launch per chunk colour)",
                          "achieved": round(sw_ach, 1), "peak": peaks["hbm_gbs"], "unit": "GB/s",
                          "frac": round(sw_ach / peaks["hbm_gbs"], 4),
                          "algorithmic_bytes_per_sweep": sw_bytes, "avg_sweep_ms": round(sw_ms, 4),
                          "share_of_step": round(sms / max(sum(v[1] for v in kt.values()), 1e-30), 3)}
        else:
            roof_sweep = None
        return roof, roof_sweep

    roof, roof_sweep = roofline_lines() if rank == 0 else (None, None)

    # ---- plain FP64 drop-in on the same requests, one at a time ----
    plain = None
    if bw.fp64_steps is not None and rank == 0 and world == 1:
        # recorded runs of the drop-in: (sweeps, steps, status) per request
        recorded = [(2, bw.fp64_steps, bw.fp64_status)]
        if bw.fp64_steps4 is not None:
            recorded.append((4, bw.fp64_steps4, bw.fp64_status4))
        n = 96
        tot, per, chosen, conv64 = 0., [], [], 0
        for i, pr in enumerate(prep):
            ms = {}
            for sw, _steps, _status in recorded:
                s = capi.Solver.from_mesh(pr.mesh, dataclasses.replace(pr.params, subits=sw),
                                          device=local)
                s.set_state(pr.Q0)
                s.converge(1, n, 1e-300, chunk=32, check=False)
                ms[sw] = s.last_device_ms() / n
                s.close()
            # the sweep count that solves this request soonest (converged
            # runs first): a choice made with hindsight, so the baseline is
            # the drop-in at its best, not at one fixed setting
            runs = [(sw, steps[i], status[i]) for sw, steps, status in recorded]
            sw, steps_i, status_i = serve.fastest_recorded_run(runs, ms)
            per.append(round(ms[sw], 4))
            chosen.append((sw, steps_i, status_i))
            tot += steps_i * ms[sw] / 1e3
            conv64 += status_i == 0
        # the model checked on two requests solved to convergence here: the
        # converged ones whose modelled time is largest below 6 s
        est = {i: chosen[i][1] * per[i] / 1e3 for i in range(len(prep)) if chosen[i][2] == 0}
        pick = sorted((i for i in est if est[i] < 6.0), key=lambda i: -est[i])[:2]
        checks = []
        for i in pick:
            pr = prep[i]
            s = capi.Solver.from_mesh(pr.mesh, dataclasses.replace(pr.params,
                                                                    subits=chosen[i][0]),
                                      device=local)
            s.set_state(pr.Q0)
            steps_i, _r0, _r1 = s.converge(1, bw.max_steps, bw.drop, chunk=32, check=False)
            real = s.last_device_ms() / 1e3
            s.close()
            checks.append({"request": i, "nodes": pr.req.nodes, "sweeps": chosen[i][0],
                           "steps": steps_i, "recorded_steps": chosen[i][1],
                           "modelled_s": round(est[i], 3), "measured_s": round(real, 3),
                           "model_error": round(est[i] / real - 1.0, 4)})
        plain = {"value": round(conv64 / tot, 5), "unit": UNIT, "converged": conv64,
                 "seconds": round(tot, 2), "ms_per_step": per,
                 "sweeps": [c[0] for c in chosen], "modelled": True,
                 "how": "per request, the recorded FP64 step count (capped at max_steps; the "
                        "drop-in runs every solve to its drop or max_steps, as the reference's "
                        "driver does) x its FP64 drop-in ms/step measured over 96 steps (graph "
                        "chunks), at whichever of the recorded sweep counts ("
                        + ", ".join(str(r[0]) for r in recorded) + ") converges it soonest; "
                        "solved one after the other",
                 "model_checked_on": checks}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and bw.fp64_steps is not None:
        cpu = batch_cpu_baseline(prep, bw)

    # ---- the serving form (Poisson arrivals of 4k..500k-node requests at two
    # rates, the same requests at each), when the run's time target leaves room
    serving = None
    if rank == 0 and world == 1 and not args.no_serving:
        left = BENCH_BUDGET_S - (time.time() - t_run0)
        if left >= SERVE_MIN_LEFT_S:
            serving = [serving_run(rate, SERVE_REQUESTS, arena, arena_bytes, bw.jacobian)
                       for rate in SERVE_RATES]
        else:
            serving = {"skipped": f"the run's time target left {left:.0f} s"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 5), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(dev_ms_max / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64 residual / f32 Jacobian+sweeps",
            "data": "synthetic (seeded O-grids and flow conditions of the batching form)",
            "config": {"workload": bw.name, "form": "batching (served, all admitted together)",
                       "requests_per_gpu": bw.n, "stream_seed": bw.seed,
                       "nodes": [r.nodes for r in reqs], "orders": [r.order for r in reqs],
                       "precision": {1: "FP64 residual/geometry/update, FP32 blocks, "
                                        "multicolour GS",
                                     3: "FP64 residual/geometry/update, FP32 blocks, GS in "
                                        "coloured chunks of the reference order"}.get(
                                            bw.precision, f"mode {bw.precision}"),
                       "gs_sweeps": bw.subits, "drop": bw.drop, "max_steps": bw.max_steps,
                       "stall_retire": {"drop": bw.stall_drop, "min_steps": bw.stall,
                                        "steps_per_sqrt_node": bw.stall_per_sqrt},
                       "autotune_steps": bw.autotune,
                       "priority_policy": bw.priority_policy,
                       "converged_per_pass": n_conv // max(args.steps, 1),
                       "stalled_per_pass": n_stall // max(args.steps, 1),
                       "failed_per_pass": n_fail // max(args.steps, 1),
                       "l2": "working set larger than L2 (batch of meshes, 0.1-0.5 GB each)",
                       "parallelism": f"requests sharded over {world} GPU(s)"},
            "latency_s": serve.percentiles(lat),
            "forces_vs_fp64": {"max_abs_diff": max(dforce) if dforce else None,
                               "solves_compared": len(dforce) // max(args.steps, 1),
                               "what": "raw lift and drag of every request converged in both "
                                       "the served form and the FP64 drop-in (recorded)"},
            "plain_fp64": plain,
            "e2e": {"value": round(e2e, 5), "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "how": "requests admitted from host threads and started as their inputs "
                           "land (continuous batching), states and forces read back as they "
                           "retire; separate timed passes",
                    "passes": n_e2e,
                    "admission_retries": len(refusals),
                    "first_refusal": refusals[0] if refusals else None},
            "e2e_staged": {"value": round(e2e_staged, 5), "unit": UNIT,
                           "how": "every request staged from host buffers first, then all "
                                  "started, states and forces read back at the end (the "
                                  "value passes)"},
            "serving": serving,
            "roofline": roof, "roofline_sweep": roof_sweep, "gpu_launches": int(launches),
            "residual_evaluations": {
                "per_s": round(evals_all / (dev_ms_max / 1e3), 1),
                "node_evals_per_s": round(node_evals_all / (dev_ms_max / 1e3)),
                "what": "one residual + Jacobian evaluation per served pseudo-time step "
                        "(all requests, device time of the timed passes)"},
            "clocks": clk.summary(), "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    arena.close()
    if pg is not None:
        pg.destroy_process_group()


def batch_cpu_baseline(prep, bw) -> dict:
    """The reference on one host core: set-up and first step untimed, then
    CPU_BASELINE_STEPS steps timed on each of the 4 smallest meshes; the cost
    per node-step of each order scales every request to its recorded step
    count."""
    from oracle import ref
    if not ref.available():
        return {"value": None, "unit": UNIT, "cores": 1, "kind": "reference",
                "sample": "oracle/_ref/libflowref.so not built"}
    per_node = {}
    small = sorted(prep, key=lambda p: p.req.nodes)[:4]
    for pr in small:
        r = ref.RefSolver(pr.wl.write())
        r.solve(1)
        t0 = time.perf_counter()
        for ts in range(2, 2 + CPU_BASELINE_STEPS):
            r.solve(ts)
        dt = (time.perf_counter() - t0) / CPU_BASELINE_STEPS
        r.close()
        per_node.setdefault(pr.req.order, []).append(dt / pr.req.nodes)
    cost = {o: sum(v) / len(v) for o, v in per_node.items()}
    fallback = sum(cost.values()) / len(cost)
    total = sum(bw.fp64_steps[i] * pr.req.nodes * cost.get(pr.req.order, fallback)
                for i, pr in enumerate(prep))
    conv64 = sum(1 for st in bw.fp64_status if st == 0)
    return {"value": round(conv64 / total, 8), "unit": UNIT, "cores": 1, "kind": "reference",
            "modelled": True,
            "sample": f"{CPU_BASELINE_STEPS} timed steps on each of the {len(small)} smallest "
                      f"meshes ({', '.join(str(p.req.nodes) for p in small)} nodes); "
                      f"s per node-step by order {dict((o, f'{c:.3e}') for o, c in cost.items())}"
                      f" x recorded FP64 steps of all {len(prep)} requests"}


def measure_fp64(args, bw):
    """Record the FP64 drop-in's step count, status and forces on every
    request of the batch (the reference's own, since the drop-in is
    bit-identical) with `--subits` Gauss-Seidel sweeps per step (default 2).
    The solves run side by side in one server in precision mode 0; a served
    solve's iterates are those it has alone."""
    import torch
    from flowgpu import capi, serve
    torch.cuda.set_device(0)
    sweeps = args.subits or 2
    reqs = [serve.sample_request(i, seed=bw.seed) for i in range(bw.n)]
    prep = serve.prepare_all(reqs, sweeps, bw.max_steps, bw.drop)
    free, _ = torch.cuda.mem_get_info(0)
    arena = capi.Arena(int(min(free * 0.85, 150e9)))
    # 16 at a time: the FP64 drop-in's ordered sweeps poll across the GPU
    r = serve.run_batch(prep, arena, precision=0, chunk=64, max_slots=16)
    arena.close()
    recs = r["records"]
    steps = tuple(x["steps"] for x in recs)
    status = tuple(x["status"] for x in recs)
    forces = tuple(tuple(x["forces"]) if x["status"] == 0 else None for x in recs)
    print(json.dumps({"workload": bw.name, "subits": sweeps, "fp64_steps": steps,
                      "fp64_status": status,
                      "seconds": round(r["makespan_s"], 2), "fp64_forces": forces}),
          flush=True)


def cpu_baseline(casedir: str, steps_conv: int) -> dict:
    """The reference solver on this host: set-up and its first step (which
    grows the k=2 stencils and factors them), then CPU_BASELINE_STEPS timed
    pseudo-time steps; extrapolated to a converged solve."""
    from oracle import ref
    if not ref.available():
        return {"value": None, "unit": UNIT, "cores": 1, "kind": "reference",
                "sample": "oracle/_ref/libflowref.so not built"}
    r = ref.RefSolver(casedir)
    r.solve(1)
    t0 = time.perf_counter()
    for ts in range(2, 2 + CPU_BASELINE_STEPS):
        r.solve(ts)
    dt = (time.perf_counter() - t0) / CPU_BASELINE_STEPS
    r.close()
    return {"value": round(1.0 / (dt * steps_conv), 8), "unit": UNIT, "cores": 1,
            "kind": "reference",
            "sample": f"{CPU_BASELINE_STEPS} pseudo-time steps (2..{1 + CPU_BASELINE_STEPS}) of "
                      f"the same solve, {dt:.3f} s/step, x {steps_conv} steps per solve"}


def run_profile(args):
    """A few pseudo-time steps of one solve of the workload, nothing else:
    the command the ncu launch lists and kernel captures in profiles/ run."""
    from flowgpu import capi, workloads
    from flowgpu.prep import Mesh
    wl = workloads.get(args.workload)
    if args.subits:
        wl = dataclasses.replace(wl, subits=args.subits)
    mesh = Mesh.from_case(wl.write(), order=wl.order)
    solver = capi.Solver.from_mesh(mesh, wl.params(), device=0)
    solver.set_sweep_mode(args.sweep_mode)
    solver.set_precision(args.precision)
    if args.jacobian:
        solver.set_jacobian(args.jacobian)
    if args.node_variant >= 0:
        solver.set_variants(args.node_variant, 0)
    if args.sweep_rows:
        solver.set_sweep_ring(args.sweep_rows)
    if args.sweep_dataflow:
        solver.set_sweep_dataflow(True)
    solver.set_state(mesh.initial_state(wl.params()))
    rh, dh = solver.run(1, args.profile_steps)
    out = {"workload": wl.name, "steps": args.profile_steps,
           "ms_per_step": solver.last_device_ms() / args.profile_steps,
           "r_rho_last": rh[-1], "launches": solver.launch_count(),
           "status": solver.status()}
    if args.kernel_times:
        # the same steps again with per-kernel events (continues the solve)
        solver.set_timing(True)
        solver.run(1 + args.profile_steps, args.profile_steps)
        out["kernels_ms_per_launch"] = {
            k: (round(ms / cnt, 4) if cnt else 0.0) for k, (cnt, ms) in
            solver.kernel_times().items()}
        solver.set_timing(False)
    print(json.dumps(out), flush=True)
    solver.close()


# ---------------------------------------------------------------------------
def _ref_worker(args_tuple):
    casedir, warmup, steps = args_tuple
    sys.path.insert(0, ROOT)
    from oracle import ref
    r = ref.RefSolver(casedir)
    r.solve(1)
    ts = 2
    for _ in range(warmup):
        for _ in range(REF_SAMPLE_STEPS):
            r.solve(ts)
            ts += 1
    t0 = time.perf_counter()
    for _ in range(steps):
        for _ in range(REF_SAMPLE_STEPS):
            r.solve(ts)
            ts += 1
    dt = time.perf_counter() - t0
    r.close()
    return dt / (steps * REF_SAMPLE_STEPS)


def _ref_batch_worker(args_tuple):
    casedir, warmup, steps = args_tuple
    sys.path.insert(0, ROOT)
    from oracle import ref
    r = ref.RefSolver(casedir)
    r.solve(1)
    ts = 2
    for _ in range(warmup * REF_SAMPLE_STEPS):
        r.solve(ts)
        ts += 1
    t0 = time.perf_counter()
    for _ in range(steps * REF_SAMPLE_STEPS):
        r.solve(ts)
        ts += 1
    dt = time.perf_counter() - t0
    r.close()
    return dt / (steps * REF_SAMPLE_STEPS)


def run_reference_batch(args, bw):
    """The reference CPU solver on the batch's requests with all host cores:
    each request's time per pseudo-time step is measured (one process per
    core), times its recorded step count; the requests are packed on the
    cores longest first.  A request on which the FP64 drop-in (and so the
    reference) fails with a non-physical state is not run: the reference does
    not return from such states (request 9 of the batch hangs from step 3),
    so its recorded steps are charged at its order's measured cost per node
    and step."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from flowgpu import capi, serve
    from oracle import ref
    if not ref.available():
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref/libflowref.so (the reference built from "
                                         "its sources) is missing"}))
        return
    if bw.fp64_steps is None:
        print(json.dumps({"impl": "reference",
                          "unavailable": f"step counts of {bw.name} are not recorded"}))
        return
    import multiprocessing as mp
    cores = os.cpu_count() or 1
    reqs = [serve.sample_request(i, seed=bw.seed) for i in range(bw.n)]
    runnable = [i for i in range(bw.n) if bw.fp64_status[i] in (0, capi.ERR_NOT_CONVERGED)]
    dirs = {i: reqs[i].workload(2, bw.max_steps, bw.drop).write(
        tempfile.mkdtemp(prefix="bench_ref_")) for i in runnable}
    ctx = mp.get_context("spawn")
    per_step = {}
    with ctx.Pool(min(cores, len(runnable))) as pool:
        jobs = {i: pool.apply_async(_ref_batch_worker, ((dirs[i], args.warmup, args.steps),))
                for i in runnable}
        deadline = time.time() + REF_ARM_TIMEOUT_S
        for i, job in jobs.items():
            per_step[i] = job.get(timeout=max(1.0, deadline - time.time()))
    cost = {}
    for o in (1, 3):
        v = [per_step[i] / reqs[i].nodes for i in runnable if reqs[i].order == o]
        if v:
            cost[o] = sorted(v)[len(v) // 2]
    for i in range(bw.n):
        if i not in per_step:
            c = cost.get(reqs[i].order, next(iter(cost.values())))
            per_step[i] = c * reqs[i].nodes
    times = [bw.fp64_steps[i] * per_step[i] for i in range(bw.n)]
    makespan = _lpt_makespan(times, cores)
    conv64 = sum(1 for st in bw.fp64_status if st == 0)
    rate = conv64 / makespan
    sample = (f"{len(runnable)} of {bw.n} requests run, each timing {args.steps} x "
              f"{REF_SAMPLE_STEPS} pseudo-time steps after set-up and {args.warmup} x "
              f"{REF_SAMPLE_STEPS} warm-up steps ({min(cores, len(runnable))} processes); the "
              f"{bw.n - len(runnable)} that fail with a non-physical state charged at their "
              f"order's median s per node-step; recorded steps x s/step per request, packed "
              f"on {cores} cores longest first: makespan {makespan:.1f} s for {conv64} "
              f"converged solves")
    line = {"metric": METRIC, "value": round(rate, 8), "unit": UNIT, "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": bw.name, "nodes": [r.nodes for r in reqs],
                       "s_per_step": [round(per_step[i], 4) for i in range(bw.n)]},
            "cpu_baseline": {"value": round(rate, 8), "unit": UNIT, "cores": cores,
                             "kind": "reference", "modelled": True, "sample": sample},
            "e2e": {"value": round(rate, 8), "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from flowgpu import workloads
    from oracle import ref
    wl = workloads.get(args.workload)
    if not ref.available():
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref/libflowref.so (the reference built from "
                                         "its sources) is missing"}))
        return
    if not wl.steps_to_converge:
        print(json.dumps({"impl": "reference",
                          "unavailable": f"converged step count of {wl.name} not recorded"}))
        return
    import multiprocessing as mp
    cores = os.cpu_count() or 1
    casedir = wl.write(tempfile.mkdtemp(prefix="bench_ref_"))
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        per_step = pool.map(_ref_worker, [(casedir, args.warmup, args.steps)] * cores)
    rate = sum(1.0 / (s * wl.steps_to_converge) for s in per_step)
    sample = (f"{cores} concurrent reference processes, each timing {args.steps} x "
              f"{REF_SAMPLE_STEPS} pseudo-time steps after {args.warmup} x {REF_SAMPLE_STEPS} "
              f"warm-up steps (mean {sum(per_step) / cores:.3f} s/step), x "
              f"{wl.steps_to_converge} steps per converged solve")
    line = {"metric": METRIC, "value": round(rate, 8), "unit": UNIT, "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": wl.name, "nodes": wl.nc * wl.nr},
            "cpu_baseline": {"value": round(rate, 8), "unit": UNIT, "cores": cores,
                             "kind": "reference", "sample": sample},
            "e2e": {"value": round(rate, 8), "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_compare_precision(args):
    """The precision form against the all-FP64 drop-in on one mesh: each run
    to a 1e-10 drop of ||R_rho|| (or the workload's step limit) from the same
    initial state; steps, device time, and the lift/drag (and their
    coefficients, C = F / (0.5 M^2), chord 1) and state differences."""
    import numpy as np
    import torch
    from flowgpu import capi, workloads
    from flowgpu.prep import Mesh
    torch.cuda.set_device(0)
    wl = workloads.get(args.workload)
    t0 = time.time()
    mesh = Mesh.from_case(wl.write(), order=wl.order)
    prep_s = time.time() - t0
    Q0 = mesh.initial_state(wl.params())
    out = {}
    mode = args.precision or 3
    for prec, sub in ((0, 2), (mode, 4)):
        fp = dataclasses.replace(wl.params(), subits=sub)
        s = capi.Solver.from_mesh(mesh, fp, device=0)
        try:
            s.set_precision(prec)
        except capi.FlowError:
            prec = 1
            s.set_precision(1)
        s.set_state(Q0)
        steps, r0, r1 = s.converge(1, wl.max_steps, wl.drop, chunk=64, check=False)
        st = s.status()
        out[prec] = {"steps": steps, "device_s": round(s.last_device_ms() / 1e3, 3),
                     "r_drop": r1 / r0, "status": st,
                     "forces": s.body_forces() if st == 0 else None, "Q": s.get("Q")}
        s.close()
    a, b = out[0], out[[k for k in out if k != 0][0]]
    qn = 0.5 * wl.mach * wl.mach
    line = {"workload": wl.name, "nodes": mesh.sizes["nn"], "host_prep_s": round(prep_s, 1),
            "fp64": {k: v for k, v in a.items() if k != "Q"},
            "precision_form": dict({k: v for k, v in b.items() if k != "Q"},
                                   mode=[k for k in out if k != 0][0], gs_sweeps=4),
            "speedup": round(a["device_s"] / max(b["device_s"], 1e-9), 3)}
    if a["forces"] and b["forces"]:
        line["d_lift"] = abs(a["forces"][0] - b["forces"][0])
        line["d_drag"] = abs(a["forces"][1] - b["forces"][1])
        line["d_CL"] = line["d_lift"] / qn
        line["d_CD"] = line["d_drag"] / qn
        line["max_abs_dQ"] = float(np.max(np.abs(a["Q"][4:] - b["Q"][4:])))
    print(json.dumps(line), flush=True)


def serving_run(rate: float, n: int, arena, budget: int, jacobian: int = 0,
                index0: int = 0) -> dict:
    """The serving form: an open-loop Poisson stream of n requests (node
    counts log-uniform in [4k, 500k], the batching stream's flow conditions
    and orders, stream seed 1, request indices index0..), each prepared on
    arrival by a worker thread, admitted as the arena allows, retired at a
    1e-8 drop (or stalled / at max_steps).  Converged solves per second of
    the run's span and p50/p95/p99 latency from arrival to retirement."""
    from flowgpu import capi, serve
    reqs = [serve.sample_request(index0 + i, seed=1, n_min=4000, n_max=500000)
            for i in range(n)]
    r = serve.run_poisson(reqs, rate, arena, subits=4, max_steps=8000, drop=1e-8,
                          precision=3, chunk=32, max_slots=64, seed=1, autotune=4,
                          stall=SERVE_STALL, ramp_sweeps=2, jacobian=jacobian,
                          stall_drop=SERVE_STALL_DROP, stall_per_sqrt=SERVE_STALL_PER_SQRT)
    recs = r["records"]
    conv = [x for x in recs if x.get("status") == 0]
    return {"value": round(len(conv) / r["span_s"], 5), "unit": UNIT,
            "form": "serving (open-loop Poisson arrivals)", "requests": n,
            "rate_per_s": rate, "span_s": round(r["span_s"], 2), "converged": len(conv),
            "stalled": sum(1 for x in recs if x.get("status") == capi.ERR_STALLED),
            "not_converged": sum(1 for x in recs if x.get("status") == capi.ERR_NOT_CONVERGED),
            "failed": sum(1 for x in recs if x.get("status") not in
                          (0, capi.ERR_STALLED, capi.ERR_NOT_CONVERGED)),
            "latency_s_converged": serve.percentiles([x["latency_s"] for x in conv]),
            "latency_s_all": serve.percentiles([x["latency_s"] for x in recs]),
            "admission_wait_s": serve.percentiles([x.get("admitted_s", 0.) for x in recs]),
            "nodes": [x.get("nodes") for x in recs], "steps": [x.get("steps") for x in recs],
            "status": [x.get("status") for x in recs],
            "config": {"drop": 1e-8, "max_steps": 8000, "precision": 3, "gs_sweeps": 4,
                       "jacobian": jacobian, "ramp_sweeps_on_meshes_from_250k_nodes": 2,
                       "stall_retire": {"drop": SERVE_STALL_DROP, "min_steps": SERVE_STALL, "steps_per_sqrt_node": SERVE_STALL_PER_SQRT}, "arena_bytes": budget, "stream_seed": 1,
                       "first_request": index0, "nodes_range": [4000, 500000]}}


def run_serve(args):
    """The serving form alone (bench.py --serve-rate R): one line."""
    import torch
    from flowgpu import capi, serve, workloads
    torch.cuda.set_device(0)
    n, rate = args.serve_requests, args.serve_rate
    reqs = [serve.sample_request(i, seed=1, n_min=4000, n_max=500000) for i in range(n)]
    free, _ = torch.cuda.mem_get_info(0)
    budget = int(min(free * 0.85, 150e9))
    arena = capi.Arena(budget, device=0)
    with ClockSampler(0) as clk:
        r = serve.run_poisson(reqs, rate, arena, subits=4, max_steps=8000, drop=1e-8,
                              precision=3, chunk=32, max_slots=64, seed=1, autotune=4,
                              stall=SERVE_STALL, ramp_sweeps=2,
                              jacobian=workloads.BATCHES[workloads.DEFAULT_BENCH].jacobian,
                              stall_drop=SERVE_STALL_DROP, stall_per_sqrt=SERVE_STALL_PER_SQRT)
    arena.close()
    recs = r["records"]
    conv = [x for x in recs if x.get("status") == 0]
    line = {"metric": METRIC, "value": round(len(conv) / r["span_s"], 5), "unit": UNIT,
            "form": "serving (open-loop Poisson arrivals)", "requests": n,
            "rate_per_s": rate, "span_s": round(r["span_s"], 2), "converged": len(conv),
            "stalled": sum(1 for x in recs if x.get("status") == capi.ERR_STALLED),
            "not_converged": sum(1 for x in recs if x.get("status") == capi.ERR_NOT_CONVERGED),
            "failed": sum(1 for x in recs if x.get("status") not in
                          (0, capi.ERR_STALLED, capi.ERR_NOT_CONVERGED)),
            "latency_s_converged": serve.percentiles([x["latency_s"] for x in conv]),
            "latency_s_all": serve.percentiles([x["latency_s"] for x in recs]),
            "admission_wait_s": serve.percentiles([x.get("admitted_s", 0.) for x in recs]),
            "prep_s": serve.percentiles([x.get("prep_s", 0.) for x in recs]),
            "nodes": [x.get("nodes") for x in recs], "steps": [x.get("steps") for x in recs],
            "status": [x.get("status") for x in recs],
            "config": {"drop": 1e-8, "max_steps": 8000, "precision": 3, "gs_sweeps": 4,
                       "ramp_sweeps_on_meshes_from_250k_nodes": 2,
                       "stall_retire": {"drop": SERVE_STALL_DROP, "min_steps": SERVE_STALL, "steps_per_sqrt_node": SERVE_STALL_PER_SQRT}, "arena_bytes": budget, "stream_seed": 1,
                       "nodes_range": [4000, 500000]},
            "clocks": clk.summary()}
    print(json.dumps(line), flush=True)


def torchrun_argv(argv, gpus: int, port: int) -> list:
    """The command that runs this script as `gpus` ranks, one per GPU, the
    way a multi-GPU launch does: torchrun on this node over 127.0.0.1."""
    return [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
            f"--nproc-per-node={gpus}", "--master-addr=127.0.0.1", f"--master-port={port}",
            os.path.abspath(__file__), *argv]


def relaunch_as_ranks(argv, gpus: int) -> int:
    """`--gpus N` (N > 1) outside torchrun: start the N ranks here instead of
    silently running one.  Returns torchrun's exit code."""
    import socket
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    log(f"--gpus {gpus} without torchrun: launching {gpus} ranks")
    return subprocess.call(torchrun_argv(argv, gpus, port))


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="flow", choices=("flow", "reference"))
    ap.add_argument("--workload", default=None)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serving", action="store_true",
                    help="batch workloads: leave out the serving-form measurement")
    ap.add_argument("--kernel-times", action="store_true",
                    help="with --profile-steps: also print per-kernel device times")
    ap.add_argument("--profile-steps", type=int, default=0,
                    help="only run this many pseudo-time steps of one solve (for ncu captures)")
    ap.add_argument("--sweep-mode", type=int, default=0, help="0 grid-wide, 1 one-CTA ordered sweep")
    ap.add_argument("--measure-fp64", action="store_true",
                    help="batch workloads: record the FP64 drop-in's step counts per request")
    ap.add_argument("--precision", type=int, default=0,
                    help="with --profile-steps: 0 FP64 drop-in, 1 FP32 multicolour sweeps")
    ap.add_argument("--sweep-dataflow", action="store_true",
                    help="with --profile-steps: one launch per mode 3 sweep (dataflow chunks)")
    ap.add_argument("--sweep-rows", type=int, default=0,
                    help="with --profile-steps: sub-level rows of the mode 3 sweep ring (64, 32, 16)")
    ap.add_argument("--jacobian", type=int, default=0,
                    help="with --profile-steps: precision-form face Jacobians (flow_set_jacobian)")
    ap.add_argument("--node-variant", type=int, default=-1,
                    help="with --profile-steps: node kernel variant (3: staged in shared memory)")
    ap.add_argument("--subits", type=int, default=0,
                    help="with --profile-steps: Gauss-Seidel sweeps per step (0: the workload's); "
                         "with --measure-fp64: the FP64 drop-in's sweeps (0: 2)")
    ap.add_argument("--serve-rate", type=float, default=0.,
                    help="run the serving form: Poisson arrivals at this rate (requests/s)")
    ap.add_argument("--serve-requests", type=int, default=16)
    ap.add_argument("--compare-precision", action="store_true",
                    help="one mesh (--workload): the precision form (--precision, default 3) "
                         "against the FP64 drop-in, each to a 1e-10 drop")
    args = ap.parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(relaunch_as_ranks(sys.argv[1:], args.gpus))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world != args.gpus:
        log(f"--gpus {args.gpus} but WORLD_SIZE={world}: running {world} rank(s)")
    if args.serve_rate > 0:
        run_serve(args)
        return
    if args.compare_precision:
        run_compare_precision(args)
        return
    from flowgpu import workloads
    args.workload = args.workload or workloads.DEFAULT_BENCH
    bw = workloads.BATCHES.get(args.workload)
    if args.profile_steps > 0:
        if bw is not None:
            args.workload = workloads.DEFAULT
        run_profile(args)
    elif bw is not None:
        if args.impl == "reference":
            run_reference_batch(args, bw)
        elif args.measure_fp64:
            measure_fp64(args, bw)
        else:
            run_batch(args, bw)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_flow(args)


if __name__ == "__main__":
    main()
