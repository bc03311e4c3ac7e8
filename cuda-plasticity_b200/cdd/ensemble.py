"""Ensembles of independent CDD instances across GPUs: one process per GPU, no data-path collective.

The reference runs independent simulations as separate processes, one per device
(Plasticity/exec_batch.py L26-61). Here an ensemble is split across ranks by a greedy
longest-processing-time bin packing on cell counts; every rank builds one batched ``cdd.Plan``
for its share and steps it without communication (``ShardedEnsemble``). Per-instance observables
(time, energy, mean strain) are gathered to all ranks at output times with ``torch.distributed``
(one all-reduce: NCCL on GPUs, gloo on CPU).
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


def _dist():
    import torch.distributed as dist
    return dist if (dist.is_available() and dist.is_initialized()) else None


def gather_rows(local_ids, values, n_total, group=None, device=None):
    """Per-instance rows of every rank in one (n_total, k) float64 array on every rank.

    Each instance belongs to exactly one rank, so the rows are placed in a zero table and summed
    over ranks with one all-reduce (on ``device``: the rank's GPU for NCCL, the CPU for gloo).
    Without an initialised process group the table holds this process's rows (others NaN).
    """
    import torch
    values = np.asarray(values, dtype=np.float64).reshape(len(local_ids), -1)
    dist = _dist()
    k = values.shape[1]
    if dist is None:
        out = np.full((n_total, k), np.nan)
        out[list(local_ids)] = values
        return out
    t = torch.zeros((n_total, k), dtype=torch.float64, device=device or "cpu")
    if len(local_ids):
        t[torch.as_tensor(list(local_ids), dtype=torch.long, device=t.device)] = \
            torch.as_tensor(values, dtype=torch.float64, device=t.device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy()


class ShardedEnsemble:
    """Independent instances spread over the ranks of the current process group (one GPU each).

    Every rank owns the instances ``shard_instances`` gives it and steps them as one batched
    ``cdd.Plan`` on its own GPU: no communication inside a step. ``observables()`` gathers
    (t, energy, mean beta_zz) of all instances to every rank with one all-reduce; ``field(i)``
    is the device view of a local instance. All ranks must call ``observables`` together (it is
    a collective). With one process (no process group) it is a plain batched plan.
    """

    def __init__(self, instances, precision="f32", tuning=None, group=None, plan_factory=None):
        """plan_factory(instances, precision, tuning) builds the rank's plan (default: cdd.Plan on
        the current CUDA device; tests of the bookkeeping pass a host stand-in)."""
        import torch
        self.instances = list(instances)
        self.group = group
        dist = _dist()
        self.world = dist.get_world_size(group) if dist else 1
        self.rank = dist.get_rank(group) if dist else 0
        self.shards = shard_instances([inst.cells for inst in self.instances], self.world)
        self.local_ids = list(self.shards[self.rank])
        self._local_index = {g: k for k, g in enumerate(self.local_ids)}
        backend = dist.get_backend(group) if dist else None
        self._reduce_device = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" \
            else torch.device("cpu")
        if plan_factory is None:
            from .engine import Plan

            def plan_factory(insts, prec, tun):
                return Plan(insts, prec, tuning=tun)
        self.plan = None
        self.beta = None
        if self.local_ids:
            tun = tuning
            if isinstance(tuning, (list, tuple)):
                tun = [tuning[g] for g in self.local_ids]
            self.plan = plan_factory([self.instances[g] for g in self.local_ids], precision, tun)
            self.beta = self.plan.empty_field()

    @property
    def local_cells(self):
        return self.plan.total_cells if self.plan else 0

    @property
    def total_cells(self):
        return int(sum(inst.cells for inst in self.instances))

    def is_local(self, i):
        return i in self._local_index

    def field(self, i):
        """Device view (9,) + shape of global instance i; None when another rank owns it."""
        k = self._local_index.get(i)
        return None if k is None else self.plan.field_view(self.beta, k)

    def load(self, make_field):
        """Fill every local instance from make_field(i) (a numpy array or tensor of its shape)."""
        for g in self.local_ids:
            self.field(g).copy_(_as_tensor(make_field(g), self.field(g)))

    def set_time(self, t=0.0, t_end=1e30):
        if self.plan:
            self.plan.set_time(t, t_end)

    def run(self, n_steps, graph=True):
        """n_steps adaptive steps of every local instance (stream-ordered; no communication)."""
        if self.plan:
            self.plan.run(self.beta, n_steps, graph=graph)

    def check_status(self):
        if self.plan:
            self.plan.check_status()

    def observables(self):
        """(n_instances, 3) array of (t, energy, mean beta_zz) on every rank (a collective)."""
        rows = np.zeros((len(self.local_ids), 3))
        if self.plan:
            t, _, _ = self.plan.get_time()
            e, m = self.plan.observables(self.beta)
            rows[:, 0], rows[:, 1], rows[:, 2] = t, e, m
        return gather_rows(self.local_ids, rows, len(self.instances), self.group, self._reduce_device)


def _as_tensor(a, like):
    import torch
    t = torch.as_tensor(np.ascontiguousarray(a) if isinstance(a, np.ndarray) else a)
    return t.to(device=like.device, dtype=like.dtype)
