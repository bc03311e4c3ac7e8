"""Ensembles of independent CDD instances across GPUs: one process per GPU, no data-path collective.

The reference runs independent simulations as separate processes, one per device
(Plasticity/exec_batch.py L26-61). Here an ensemble is split across ranks by a greedy
longest-processing-time bin packing on cell counts; every rank builds one batched ``cdd.Plan``
for its share and steps it without communication. Per-instance observables (time, energy, mean
strain) are gathered to all ranks at output times with ``torch.distributed`` (NCCL on GPUs,
gloo on CPU).
"""
import numpy as np


def shard_instances(cells, world_size):
    """Assign instances (given their cell counts) to ranks; returns one index list per rank.

    Largest first, each to the currently lightest rank (ties: lowest rank); deterministic.
    """
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    order = sorted(range(len(cells)), key=lambda i: (-int(cells[i]), i))
    load = [0] * world_size
    shards = [[] for _ in range(world_size)]
    for i in order:
        r = min(range(world_size), key=lambda k: (load[k], k))
        shards[r].append(i)
        load[r] += int(cells[i])
    return [sorted(s) for s in shards]


def shard_loads(cells, shards):
    return [int(sum(int(cells[i]) for i in s)) for s in shards]


def gather_observables(local_ids, values, n_total, group=None):
    """All-gather per-instance rows (e.g. [t, energy, mean_zz]) into a (n_total, k) array.

    local_ids: global instance indices of this rank; values: (len(local_ids), k) array.
    Works with any initialised torch.distributed backend; a single process returns its rows.
    """
    import torch.distributed as dist
    values = np.asarray(values, dtype=np.float64).reshape(len(local_ids), -1)
    k = values.shape[1] if values.size else 0
    if not (dist.is_available() and dist.is_initialized()):
        out = np.full((n_total, k), np.nan)
        out[list(local_ids)] = values
        return out
    parts = [None] * dist.get_world_size(group)
    dist.all_gather_object(parts, (list(local_ids), values.tolist()), group=group)
    k = max((len(v[0]) for _, v in parts if v), default=k)
    out = np.full((n_total, k), np.nan)
    for ids, vals in parts:
        for i, row in zip(ids, vals):
            out[i] = row
    return out
