#!/usr/bin/env python3
"""Converged steady solves per second of the flow solver's nonlinear iteration.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl flow|reference]
                    [--workload NAME]

A "step" is one complete steady solve of the workload: pseudo-time steps of
the reference's solve() (residual, Jacobian, two ordered block Gauss-Seidel
sweeps, update) until the density residual norm has dropped by 1e-10.

* value: solves/s with the initial state already on the device (restored
  from a device snapshot), timed with CUDA events on the library's stream.
* e2e: the same through the C ABI with host buffers: the initial state is
  copied from pinned host memory, the converged solution and the lift/drag
  forces are copied back, inside the timed region.
* roofline: the ordered sweep kernel (the largest share of a step) against
  the measured HBM copy bandwidth, with the compulsory bytes of one sweep
  (132 B per matrix block + 96 B per node).
* cpu_baseline: the reference solver (oracle/_ref, built from its own
  sources) on this host, a bounded sample of pseudo-time steps extrapolated
  with the workload's converged step count.

Multi-GPU (torchrun, one process per GPU): every rank runs its own replica of
the solve (the path does not shard), value = all ranks' solves / the slowest
rank's time ("scaling": "weak").

--impl reference times the reference's own CPU solver on all host cores
(one process per core, each timing a bounded sample of the workload's
pseudo-time steps), rank 0 only.
"""
from __future__ import annotations

import dataclasses
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "flow-solver_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

METRIC = "converged solves/s (1e-10 drop of ||R_rho||), steady k=2 Euler, FP64"
UNIT = "solves/s"
REF_SAMPLE_STEPS = 2        # pseudo-time steps per reference-arm bench step
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


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="flow", choices=("flow", "reference"))
    ap.add_argument("--workload", default=None)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--kernel-times", action="store_true",
                    help="with --profile-steps: also print per-kernel device times")
    ap.add_argument("--profile-steps", type=int, default=0,
                    help="only run this many pseudo-time steps of one solve (for ncu captures)")
    ap.add_argument("--sweep-mode", type=int, default=0, help="0 grid-wide, 1 one-CTA ordered sweep")
    ap.add_argument("--precision", type=int, default=0,
                    help="with --profile-steps: 0 FP64 drop-in, 1 FP32 multicolour sweeps")
    ap.add_argument("--subits", type=int, default=0,
                    help="with --profile-steps: Gauss-Seidel sweeps per step (0: the workload's)")
    args = ap.parse_args()
    from flowgpu import workloads
    args.workload = args.workload or workloads.DEFAULT
    if args.impl == "reference":
        run_reference(args)
    elif args.profile_steps > 0:
        run_profile(args)
    else:
        run_flow(args)


if __name__ == "__main__":
    main()
