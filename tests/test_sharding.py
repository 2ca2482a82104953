"""CPU, two ranks over gloo: frequency sharding of a block (blade_b200.sharding).

Each rank runs the chain (the FP64 oracle stands in for the GPU kernels here) on
its own channel range with no data exchange; the products gathered in rank
order equal the unsharded result, for an uneven channel split too, and the
timing reduction takes the slowest rank."""

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from blade_b200 import sharding
from oracle import formulas as O

A, F, T, P, B, R, I = 4, 5, 64, 2, 3, 2, 2


def _block():
    rng = np.random.default_rng(2024)
    x = np.clip(np.rint(rng.standard_normal((A, F, T, P, 2)) * 8), -127, 127).astype(np.int8)
    w = np.exp(2j * np.pi * rng.random((B, A, F, 1, P))).astype(np.complex64)
    return x, w


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        x, w = _block()
        xs, ws = sharding.shard_block(torch.from_numpy(x), torch.from_numpy(w), world, rank)
        local = O.beamform_channelize_detect(xs.numpy(), ws.numpy(), R, I, 1)
        got = sharding.gather_channels(torch.from_numpy(np.ascontiguousarray(local)), F, rate=R, axis=1)
        slowest = sharding.max_over_ranks(1.0 + rank, device="cpu")
        if rank == 0:
            np.save(os.path.join(out_dir, "gathered.npy"), got.numpy())
            np.save(os.path.join(out_dir, "slowest.npy"), np.array([slowest]))
    finally:
        dist.destroy_process_group()


def test_channel_ranges_cover_the_band():
    for F_, world in [(192, 1), (192, 8), (5, 2), (7, 3), (3, 4)]:
        ranges = [sharding.channel_range(F_, world, r) for r in range(world)]
        assert ranges[0][0] == 0 and ranges[-1][1] == F_
        assert all(a[1] == b[0] for a, b in zip(ranges, ranges[1:]))
        sizes = [b - a for a, b in ranges]
        assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        sharding.channel_range(8, 2, 2)


def test_two_rank_sharded_chain_equals_unsharded(tmp_path):
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    x, w = _block()
    ref = O.beamform_channelize_detect(x, w, R, I, 1)
    got = np.load(tmp_path / "gathered.npy")
    assert got.shape == ref.shape
    np.testing.assert_array_equal(got, ref)  # same FP64 arithmetic per channel
    assert float(np.load(tmp_path / "slowest.npy")[0]) == 2.0
