"""The multi-GPU layout of bench.py on CPU: two gloo ranks, each with its own pair shard
(no data-path collective), timing reduced as the max over ranks."""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        times = [10.0 + rank, 20.0 - rank]          # per-rank device ms (dev, e2e)
        red = bench.reduce_max(times, dist, "cpu")
        _, basis, pairs, _ = bench.workload("config2", 1000, rank)
        digest = int(np.bitwise_xor.reduce(pairs.astype(np.uint64).ravel()))
        out[rank] = (red, digest, bench.aggregate_rate(1000, world, 5, red[0]))
    finally:
        dist.destroy_process_group()


def test_two_rank_reduction_and_shards():
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(2, _free_port(), out), nprocs=2, join=True)
    r0, r1 = out[0], out[1]
    assert r0[0] == r1[0] == [11.0, 20.0]           # max over ranks, same on every rank
    assert r0[1] != r1[1]                            # distinct shards
    assert abs(r0[2] - 1000 * 2 * 5 / 0.011) < 1e-6  # whole-job rate over the slowest rank
    # shards are deterministic
    _, _, p0, _ = bench.workload("config2", 1000, 0)
    _, _, p0b, _ = bench.workload("config2", 1000, 0)
    assert np.array_equal(p0, p0b)
