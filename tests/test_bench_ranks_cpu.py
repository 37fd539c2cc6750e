"""The multi-rank bench path on CPU: two gloo ranks (one process each, as
torchrun launches them) run the same collective steps; timings reduce to the
maximum over ranks and the whole-job rate counts every rank's replica; the
reference arm does its work on rank 0 only."""
import os
import socket
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        got_ws, got_rank, got_local = bench.dist_env()
        step_ms = 10.0 + 5.0 * rank          # the slower rank decides the step time
        ms = bench.max_over_ranks(step_ms, got_ws)
        e2e = bench.max_over_ranks(0.02 * (rank + 1), got_ws)
        q.put((got_rank, got_ws, got_local, ms, bench.whole_job_rate(ms, got_ws),
               bench.whole_job_rate(1e3 * e2e, got_ws)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_to_the_slowest():
    ws = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(ws))
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    for rank, (r, w, local, ms, rate, e2e_rate) in enumerate(res):
        assert (r, w, local) == (rank, ws, rank)
        assert ms == 15.0                       # max over ranks
        assert rate == pytest.approx(ws * 1e3 / 15.0)  # two replicas per step
        assert e2e_rate == pytest.approx(ws / 0.04)


def test_single_rank_needs_no_process_group():
    import bench
    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.whole_job_rate(100.0, 1) == pytest.approx(10.0)


def _ref_rank(rank, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank))
    import bench

    class A:
        workload = "small"
        warmup = 0
        steps = 1
        gpus = 2

    if rank == 0:
        q.put(("rank0", bench.dist_env()))
    else:
        bench.run_reference(A())  # returns at once: the reference arm runs on rank 0 only
        q.put(("rank1-returned", bench.dist_env()))


def test_reference_arm_runs_on_rank_zero_only():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_ref_rank, args=(1, q))
    p.start()
    tag, env = q.get(timeout=120)
    p.join(60)
    assert tag == "rank1-returned" and env[1] == 1 and p.exitcode == 0
