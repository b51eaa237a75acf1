"""Multi-GPU path of the bench on CPU: world_size-2 gloo ranks (replicas only,
no data-path collective) agree on the max-over-ranks time and the whole-job
throughput, and the reference arm leaves non-zero ranks without work."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, init_method=f"tcp://127.0.0.1:{port}")
    try:
        # rank r "measured" 10 + r ms per step and 3 + 2r ms end to end
        ts = bench.max_over_ranks([10.0 + rank, 3.0 + 2 * rank], dist)
        out[rank] = (ts[0], ts[1], bench.replica_throughput(world, 1000, ts[0]))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_throughput_two_ranks():
    world, port = 2, free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
    assert out[0] == out[1] == (11.0, 5.0, 2 * 1000 / 11e-3)


def test_single_rank_needs_no_process_group():
    assert bench.max_over_ranks([4.0, 2.0]) == [4.0, 2.0]
    assert bench.replica_throughput(1, 500, 2.0) == pytest.approx(2.5e5)


def test_reference_arm_other_ranks_do_no_work(capsys):
    class Args:
        gpus, steps, warmup = 2, 1, 1
    bench.run_reference(Args(), rank=1, world=2)
    assert capsys.readouterr().out == ""
