"""Replicas-only multi-GPU mode of bench.py, exercised on CPU with gloo.

The (T) problem fits one GPU, so `bench.py --gpus N` runs N independent
problems, one per rank, with no collective on the data path; the only
communication is the max over ranks of the timed region.  Two gloo ranks
check that reduction and the whole-job throughput built from it, and that
the reference arm does its work on rank 0 only.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist

    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        local = 2.0 + rank          # rank 1 is the slow replica
        t = bench.max_over_ranks(local)
        out[rank] = (t, bench.job_throughput(world, 3, 1e12, t))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_job_throughput_two_gloo_ranks():
    world = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    for rank in range(world):
        t, val = res[rank]
        assert t == pytest.approx(3.0)
        # 2 replicas x 3 steps x 1 TFLOP in the slowest replica's 3 s
        assert val == pytest.approx(2.0)


def test_single_process_needs_no_process_group():
    import bench
    assert bench.max_over_ranks(1.25) == 1.25


def test_reference_arm_is_rank0_only(capsys):
    import argparse

    import bench
    args = argparse.Namespace(steps=1, warmup=3, cpu_target=1.0, workload="water_ccpvdz_o5v19")
    bench.run_reference(args, 5, 19, rank=1)
    assert capsys.readouterr().out == ""
