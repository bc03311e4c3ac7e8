"""The sharded ensemble path on the GPU (cdd.ensemble.ShardedEnsemble): with a world-size-1 NCCL
process group it equals the unsharded batched plan bitwise, its observables come back through the
NCCL all-reduce, and the per-rank plans of a 2-way shard step every instance bitwise like the
batched plan (instances never interact, so the split changes nothing)."""
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import cdd
from cdd.ensemble import ShardedEnsemble, shard_instances


def _instances():
    shapes = [(32, 32, 32), (64, 64), (16, 24, 32), (48, 48), (24, 24, 24)]
    insts = [cdd.Instance(sh, mu=1.0, nu=0.3, cfl=0.25, load_rate=(-0.01 * i, -0.01 * i, 0.02 * i))
             for i, sh in enumerate(shapes)]
    fields = [cdd.gaussian_random_field(sh, 0.06, 0.05, 70 + i) for i, sh in enumerate(shapes)]
    return insts, fields


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_sharded_ensemble_world1_nccl_equals_batched_plan():
    import torch.distributed as dist
    insts, fields = _instances()
    full = cdd.Plan(insts, "f32")
    fb = full.pack(fields)
    full.set_time(0.0, 1e30)
    full.run(fb, 3, graph=True)
    e_full, m_full = full.observables(fb)
    t_full, _, _ = full.get_time()
    dist.init_process_group("nccl", init_method="tcp://127.0.0.1:%d" % _free_port(), rank=0, world_size=1,
                            device_id=torch.device("cuda", torch.cuda.current_device()))
    try:
        ens = ShardedEnsemble(insts, "f32")
        assert ens.local_ids == list(range(len(insts)))
        ens.load(lambda i: fields[i])
        ens.set_time(0.0)
        ens.run(3)
        table = ens.observables()
        for i in range(len(insts)):
            assert torch.equal(ens.field(i), full.field_view(fb, i))
        np.testing.assert_array_equal(table[:, 0], t_full)
        np.testing.assert_array_equal(table[:, 1], e_full)
        np.testing.assert_array_equal(table[:, 2], m_full)
    finally:
        dist.destroy_process_group()


def test_two_way_shard_plans_equal_batched_plan_bitwise():
    insts, fields = _instances()
    full = cdd.Plan(insts, "f32")
    fb = full.pack(fields)
    full.set_time(0.0, 1e30)
    full.run(fb, 2, graph=True)
    shards = shard_instances([i.cells for i in insts], 2)
    assert all(shards)
    for ids in shards:
        p = cdd.Plan([insts[g] for g in ids], "f32")
        b = p.pack([fields[g] for g in ids])
        p.set_time(0.0, 1e30)
        p.run(b, 2, graph=True)
        for k, g in enumerate(ids):
            assert torch.equal(p.field_view(b, k), full.field_view(fb, g))
