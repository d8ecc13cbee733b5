"""Multi-GPU sharding of the batched form: one process per GPU, the
independent instances partitioned across ranks, no data-path collective.

Each rank advances its own share with a ``WignerBatch`` (its own persistent
CUDA graph); the only exchange is the gather of the per-step observables to
rank 0 at the end of a run.  Work is balanced greedily (longest processing
time first) on the per-step device cost of an instance: its grid points times
the measured device time per point of its size class and damping
(``MEASURED_NS``, from ``python bench.py --workload shardcost``); sizes outside
the table fall back to N_x N_p log2(N_x N_p), times four when damped (the
transform count of a damped p-pass).
"""
import math

# device time per grid point per step (ns) of the mixed-precision batched form on one B200,
# by square size class; 'd': damped (Caldeira-Leggett).  Measured with
#   python bench.py --workload shardcost --steps 20 --warmup 3
# (SM clock 1965 MHz, default register caps).  The cost per point is nearly flat in the size:
# the passes are bound by latency and issue, not by the transform's log factor.
MEASURED_NS = {
    '128': 0.01832, '128d': 0.02487,
    '256': 0.01807, '256d': 0.02531,
    '512': 0.01957, '512d': 0.02508,
    '1024': 0.02102, '1024d': 0.02808,
}


def instance_cost(d, table=None):
    """Relative per-step device cost of one batched instance descriptor."""
    t = MEASURED_NS if table is None else table
    n_x, n_p = int(d['n_x']), int(d['n_p'])
    damped = float(d.get('gamma', 0.)) != 0.
    key = '%d%s' % (max(n_x, n_p), 'd' if damped else '')
    if key in t:
        return n_x * n_p * float(t[key])
    n = n_x * n_p
    return n * math.log2(n) * (4. if damped else 1.) * 1e-3


def partition(instances, world):
    """Indices of the instances each of ``world`` ranks runs: greedy LPT on
    ``instance_cost``; every index appears once, each rank's list ascending."""
    if world < 1:
        raise ValueError('world must be >= 1')
    order = sorted(range(len(instances)), key=lambda i: (-instance_cost(instances[i]), i))
    load = [0.] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += instance_cost(instances[i])
    return [sorted(p) for p in parts]


def imbalance(instances, parts):
    """max rank cost / mean rank cost of a partition."""
    loads = [sum(instance_cost(instances[i]) for i in p) for p in parts]
    mean = sum(loads) / len(loads)
    return max(loads) / mean if mean > 0 else 1.


def gather_observables(obs_local, parts, rank, group=None):
    """Reassemble per-instance observables on rank 0: ``obs_local`` is this
    rank's array [len(parts[rank]), n + 1, 11]; rank 0 returns the array over
    all instances in their original order, the other ranks None.  Uses
    ``torch.distributed.gather_object`` (any backend)."""
    import numpy as np
    import torch.distributed as dist
    world = len(parts)
    if world == 1:
        return obs_local
    got = [None] * world if rank == 0 else None
    dist.gather_object(obs_local, got, dst=0, group=group)
    if rank != 0:
        return None
    n_inst = sum(len(p) for p in parts)
    out = np.empty((n_inst,) + tuple(got[0].shape[1:]), dtype=got[0].dtype)
    for r, p in enumerate(parts):
        out[p] = got[r]
    return out
