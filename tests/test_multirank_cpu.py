"""Multi-rank host logic on CPU with the gloo backend (world size 2): ensemble
scene sharding and the max-over-ranks timing reduction bench.py uses."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import wcsph


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, counts, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        shard = wcsph.shard_scenes(counts, world)[rank]
        load = sum(counts[k] for k in shard)
        gathered = [None] * world
        dist.all_gather_object(gathered, shard)
        t = torch.tensor([float(load)], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        out[rank] = (gathered, float(t.item()), load)
    finally:
        dist.destroy_process_group()


def test_ensemble_sharding_two_ranks():
    counts = [wcsph.preset_ensemble(1, k).info.fluid_n for k in range(256)]
    port = _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(2, port, counts, out), nprocs=2, join=True)
    gathered, max_load, _ = out[0]
    assert out[1][0] == gathered
    allk = sorted(k for s in gathered for k in s)
    assert allk == list(range(256))                        # complete, disjoint
    loads = [sum(counts[k] for k in s) for s in gathered]
    assert max_load == max(loads)                           # max over ranks
    assert max(loads) <= 1.01 * (sum(counts) / 2)           # balanced
