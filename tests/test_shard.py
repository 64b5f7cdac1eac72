"""Host logic of the multi-GPU mode: frame partitioning and metadata gather,
run as two gloo ranks on CPU (frames are independent, so the data path needs
no collective)."""

import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from cusmic_b200 import shard


def test_partition_balances_and_covers():
    sizes = [4096 * 300, 256 * 256, 2048 * 2048, 1000 * 900, 512 * 512, 4000 * 4000, 300 * 300]
    for world in (1, 2, 3, 4, 8):
        parts = shard.partition(sizes, world)
        assert len(parts) == world
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(sizes)))
        loads = [sum(sizes[i] for i in p) for p in parts]
        # greedy largest-first: no rank exceeds the ideal by more than one frame
        assert max(loads) <= sum(sizes) / world + max(sizes)


def test_partition_rejects_empty_world():
    with pytest.raises(ValueError):
        shard.partition([1, 2], 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, sizes, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = shard.partition(sizes, world)[rank]
        # stand-in for the per-frame flagged counts a GPU rank would report
        values = [sizes[i] % 97 for i in mine]
        out[rank] = shard.gather_metadata(mine, values, len(sizes))
    finally:
        dist.destroy_process_group()


def test_gather_metadata_two_ranks():
    sizes = [262144, 4194304, 65536, 1048576, 16384]
    manager = mp.get_context("spawn").Manager()  # no fork of this (threaded) process
    out = manager.dict()
    mp.spawn(_worker, args=(2, _free_port(), sizes, out), nprocs=2, join=True)
    want = [s % 97 for s in sizes]
    assert out[0] == want and out[1] == want
