"""The multi-GPU path of bench.py (one independent replica per rank, no data
collective, the slowest rank's time) exercised with 2 gloo ranks on the CPU."""
import os
import socket
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, REPO)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms_local = [7.5, 9.25][rank]  # rank 1 is the slower one
        ms_max = bench.max_over_ranks(ms_local, dist, device="cpu")
        rate = bench.whole_job_rate(world, 4_194_304, 32, ms_max)
        dist.barrier()
        out[rank] = (ms_max, rate)
    finally:
        dist.destroy_process_group()


def test_two_ranks_take_the_slowest_time_and_sum_the_work():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0] == res[1]
    ms_max, rate = res[0]
    assert ms_max == 9.25
    assert rate == pytest.approx(2 * 4_194_304 * 32 / 9.25e-3)


def test_reference_arm_runs_on_rank_zero_only(capsys):
    """Under torchrun every rank starts the reference arm; ranks other than 0
    exit at once without output (the CPU baseline is one host's cores)."""
    sys.path.insert(0, REPO)
    import argparse

    import bench
    args = argparse.Namespace(gpus=2, steps=1, warmup=3, impl="reference")
    bench.run_reference(args, rank=1)
    assert capsys.readouterr().out == ""
