"""Ensemble sharding across ranks: deterministic bin packing and a 2-rank gloo gather of
per-instance observables (no GPU; processes started with spawn)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from cdd.ensemble import shard_instances, shard_loads, gather_observables

# config-4 ensemble: 16 each of 2-D 256^2, 512^2 and 3-D 48^3, 64^3, 96^3, 128^3
CELLS = [256 ** 2] * 16 + [512 ** 2] * 16 + [48 ** 3] * 16 + [64 ** 3] * 16 + [96 ** 3] * 16 + [128 ** 3] * 16


def test_shards_cover_every_instance_once_and_balance():
    for w in (1, 2, 4, 8):
        shards = shard_instances(CELLS, w)
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(len(CELLS)))
        loads = shard_loads(CELLS, shards)
        assert max(loads) - min(loads) <= max(CELLS)
        assert shards == shard_instances(CELLS, w)   # deterministic


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        shards = shard_instances(CELLS, world)
        mine = shards[rank]
        vals = [[float(i), 10.0 * i + rank] for i in mine]
        table = gather_observables(mine, vals, len(CELLS))
        if rank == 0:
            np.save(out, table)
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_gather(tmp_path):
    out = str(tmp_path / "table.npy")
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, start_method="spawn", join=True)
    table = np.load(out)
    shards = shard_instances(CELLS, 2)
    assert table.shape == (len(CELLS), 2)
    for r, s in enumerate(shards):
        for i in s:
            assert table[i, 0] == i and table[i, 1] == 10.0 * i + r
