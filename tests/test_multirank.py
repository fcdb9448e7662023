"""The multi-GPU host logic of bench.py with world-size-2 gloo ranks on the
CPU: each rank serves its own slice of the request stream (no request on two
ranks), and the timings/counts combine as max over ranks / sum over ranks."""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "flow-solver_b200")]
    import bench
    from flowgpu import serve, workloads
    w, r, local, pg = bench.dist_setup(world)
    bw = workloads.BATCHES["batch16"]
    idx = [rank * bw.n + i for i in range(bw.n)]
    reqs = [serve.sample_request(i, seed=bw.seed) for i in idx]
    t_max = bench.allreduce_max(pg, 10.0 + rank)
    n_sum = bench.allreduce_sum(pg, 3.0 + rank)
    bench.barrier(pg)
    out.put((rank, w, r, idx, [q.nodes for q in reqs], t_max, n_sum))
    pg.destroy_process_group()


def test_two_gloo_ranks_shard_requests_and_combine():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, w0, rr0, idx0, n0, t0, s0), (r1, w1, rr1, idx1, n1, t1, s1) = res
    assert (w0, w1, rr0, rr1) == (2, 2, 0, 1)
    assert not set(idx0) & set(idx1)
    assert t0 == t1 == 11.0
    assert s0 == s1 == 7.0


def test_reference_arm_other_ranks_exit_without_work(monkeypatch, capsys):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "flow-solver_b200")]
    import bench
    from flowgpu import workloads
    monkeypatch.setenv("RANK", "1")

    class A:
        gpus, steps, warmup = 2, 1, 1
    bench.run_reference_batch(A(), workloads.BATCHES["batch16"])
    assert capsys.readouterr().out == ""


def test_gpus_without_torchrun_relaunches_as_ranks(monkeypatch):
    """bench.py --gpus N outside torchrun starts N ranks (torchrun on this
    node over 127.0.0.1) instead of silently running one."""
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "flow-solver_b200")]
    import bench
    argv = bench.torchrun_argv(["--gpus", "4", "--steps", "2"], 4, 29512)
    assert argv[1:4] == ["-m", "torch.distributed.run", "--nnodes=1"]
    assert "--nproc-per-node=4" in argv and "--master-addr=127.0.0.1" in argv
    assert "--master-port=29512" in argv
    assert argv[-4:] == ["--gpus", "4", "--steps", "2"]
    assert argv[-5].endswith("bench.py")
    calls = []
    monkeypatch.delenv("WORLD_SIZE", raising=False)
    monkeypatch.setattr(bench.subprocess, "call", lambda cmd: calls.append(cmd) or 0)
    monkeypatch.setattr(sys, "argv", ["bench.py", "--gpus", "2"])
    import pytest as _pt
    with _pt.raises(SystemExit) as ex:
        bench.main()
    assert ex.value.code == 0 and len(calls) == 1
    assert "--nproc-per-node=2" in calls[0]
