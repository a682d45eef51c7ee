"""The multi-GPU path of bench.py on CPU: two replica ranks over gloo share a
barrier and a max over ranks, and the whole-job throughput counts every
replica's targets over the slowest rank's time.  The GPU runs use the same
helpers over NCCL (one process per GPU, no data-path collective).
"""
import os
import socket

import pytest
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        barrier, max_over_ranks = bench.rank_tools(world, "cpu")
        barrier()
        step_ms = 100.0 + 50.0 * rank          # the second replica is the slower one
        ms = max_over_ranks(step_ms)
        barrier()
        out.put((rank, ms, bench.job_throughput(world, 4_000_000, ms)))
    finally:
        dist.destroy_process_group()


def test_two_replicas_share_the_slowest_time():
    world = 2
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    codes = [p.exitcode for p in procs]
    for p in procs:
        if p.is_alive():
            p.kill()
    assert codes == [0, 0], codes
    res = sorted(out.get(timeout=5) for _ in range(world))
    for rank, ms, tput in res:
        assert ms == 150.0
        assert tput == pytest.approx(2 * 4_000_000 / 0.150)


def test_single_rank_tools_need_no_process_group():
    barrier, max_over_ranks = bench.rank_tools(1, "cpu")
    barrier()
    assert max_over_ranks(3.5) == 3.5
    assert bench.job_throughput(1, 1000, 500.0) == 2000.0


def test_reference_arm_runs_on_rank_zero_only(capsys):
    class Args:
        ref_sample, n, warmup, steps, workload = 10, 100, 0, 1, "gaussian4m"
    assert bench.run_reference(Args, 2, 1) is None      # rank 1: no work, no output
    assert capsys.readouterr().out == ""
