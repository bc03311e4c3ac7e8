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


class _HostPlan:
    """Host stand-in for cdd.Plan with the calls ShardedEnsemble makes (no GPU): each instance
    advances its clock by 0.01 (instance index + 1) per step; its 'energy' is the sum of its field."""

    def __init__(self, instances, precision, tuning):
        import torch
        self.instances = list(instances)
        self.cells = [inst.cells for inst in self.instances]
        self.offsets = list(np.cumsum([0] + [9 * c for c in self.cells])[:-1])
        self.total_cells = int(sum(self.cells))
        self.t = np.zeros(len(self.instances))
        self.rate = np.array([inst.cfl for inst in self.instances])
        self._torch = torch

    def empty_field(self):
        return self._torch.zeros(9 * self.total_cells, dtype=self._torch.float64)

    def field_view(self, buf, k):
        o = int(self.offsets[k])
        return buf[o:o + 9 * self.cells[k]].view((9,) + tuple(self.instances[k].shape))

    def set_time(self, t, t_end):
        self.t[:] = t

    def run(self, beta, n, graph=True):
        self.t += n * self.rate

    def get_time(self):
        return self.t.copy(), None, None

    def observables(self, beta):
        e = np.array([float(self.field_view(beta, k).sum()) for k in range(len(self.instances))])
        m = np.array([float(self.field_view(beta, k)[8].mean()) for k in range(len(self.instances))])
        return e, m

    def check_status(self):
        pass


def _ensemble_worker(rank, world, port, out):
    import torch.distributed as dist
    from cdd.engine import Instance
    from cdd.ensemble import ShardedEnsemble
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        shapes = [(8, 8, 8), (16, 16), (4, 4, 4), (12, 12), (6, 6, 6)]
        insts = [Instance(sh, cfl=0.01 * (i + 1)) for i, sh in enumerate(shapes)]
        ens = ShardedEnsemble(insts, "f64", plan_factory=_HostPlan)
        assert ens.local_ids == shard_instances([i.cells for i in insts], world)[rank]
        ens.load(lambda i: np.full((9,) + shapes[i], float(i + 1)))
        for i in range(len(insts)):
            assert (ens.field(i) is not None) == ens.is_local(i)
        ens.set_time(0.0)
        ens.run(3)
        table = ens.observables()
        if rank == 0:
            np.save(out, table)
    finally:
        dist.destroy_process_group()


def test_sharded_ensemble_bookkeeping_two_ranks(tmp_path):
    """ShardedEnsemble on 2 gloo ranks: each rank builds a plan of its shard only, loads only its
    instances, and observables() returns every instance's row on every rank."""
    out = str(tmp_path / "ens.npy")
    mp.start_processes(_ensemble_worker, args=(2, _free_port(), out), nprocs=2, start_method="spawn", join=True)
    table = np.load(out)
    shapes = [(8, 8, 8), (16, 16), (4, 4, 4), (12, 12), (6, 6, 6)]
    for i, sh in enumerate(shapes):
        cells = int(np.prod(sh))
        assert table[i, 0] == pytest.approx(3 * 0.01 * (i + 1))
        assert table[i, 1] == pytest.approx(9 * cells * (i + 1))
        assert table[i, 2] == pytest.approx(i + 1)
