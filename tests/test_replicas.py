"""The multi-GPU form of the benchmark is independent replicas (one mesh per GPU, no data-path
collective): the only cross-rank steps are the max over ranks of the timed totals and the whole-job
value. Checked here with two gloo ranks on the CPU: both ranks see the slowest rank's time and the
same aggregate.
"""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = [10.0 + 5.0 * rank, 40.0 - 7.0 * rank]  # (kernel ms, end-to-end ms) of this rank
        mx = bench.max_over_ranks(mine, dist, "cpu")
        out[rank] = (mx, bench.replica_value(world, 1000, 4, mx[0]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_max_and_value():
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    assert res[0] == res[1]
    mx, value = res[0]
    assert mx == [15.0, 40.0]
    assert value == pytest.approx(2 * 1000 * 4 / 15e-3 / 1e9)


def test_single_process_is_identity():
    assert bench.max_over_ranks([3.0, 4.0]) == [3.0, 4.0]
    assert bench.replica_value(1, 10, 2, 1.0) == pytest.approx(10 * 2 / 1e-3 / 1e9)
