"""The N > 1 bench path: replicas with no data-path collective; the timing is the max over ranks and
the work is the sum over ranks. Run as two gloo ranks on the CPU."""
import os
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.join(os.path.dirname(__file__), "..")


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        assert bench.dist_env() == (world, rank, rank)
        seconds, units = bench.aggregate(1.0 + rank, 10.0 * (rank + 1))
        bench.barrier()
        out[rank] = (seconds, units)
    finally:
        dist.destroy_process_group()


def test_two_rank_aggregate_is_max_time_and_summed_work():
    port = 29500 + (os.getpid() % 1000)
    ctx = mp.get_context("spawn")
    with ctx.Manager() as manager:
        out = manager.dict()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
        assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
        assert out[0] == out[1] == (2.0, 30.0)


def test_single_process_aggregate_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert not dist.is_initialized()
    assert bench.aggregate(3.5, 7.0) == (3.5, 7.0)


def test_clock_summary_parses_nvidia_smi_csv():
    sys.path.insert(0, ROOT)
    import bench
    text = ("0, 1965, 1965, 500.1, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active\n"
            "0, 1800, 1965, 900.0, 0x0000000000000004, Not Active, Not Active, Not Active, Active\n"
            "0, 1900, 1965, 700.0, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active\n")
    s = bench.summarize_clocks(text)
    assert s["sm_mhz"] == 1900 and s["sm_max_mhz"] == 1965
    assert s["reasons"] == ["sw_power_cap"] and s["samples"] == 3
