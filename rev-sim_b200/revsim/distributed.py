"""One process per GPU: replica sharding and the gradient exchange of a parameter update.

The reversible-simulation gradient does not shard within a replica; independent replicas
(batched water boxes, diamond replicas) spread across ranks with no collective on the data
path.  The one exchange is the parameter update of a batch: the per-replica gradients of
every rank are averaged into one parameter update, one all-reduce of P + 1 doubles over the
process group (NCCL over NVLink on GPUs, gloo on CPU).
"""

import numpy as np


def partition_replicas(n_atoms, world):
    """Greedy atom-count balance: replicas in decreasing size (ties: lower index first) go to
    the rank with the fewest atoms so far (ties: lower rank).  Returns, per rank, the
    ascending list of its replica indices; every rank computes the same partition."""
    if world < 1:
        raise ValueError("world must be >= 1")
    n_atoms = [int(n) for n in n_atoms]
    order = sorted(range(len(n_atoms)), key=lambda r: (-n_atoms[r], r))
    load = [0] * world
    parts = [[] for _ in range(world)]
    for r in order:
        k = min(range(world), key=lambda q: (load[q], q))
        parts[k].append(r)
        load[k] += n_atoms[r]
    return [sorted(p) for p in parts]


def rank_share(n_atoms, world, rank):
    """The replicas rank `rank` of `world` runs: its part of partition_replicas (ascending
    replica indices).  Per-replica inputs (start states, temperatures, noise seed columns)
    are selected with it, so each replica gets the same inputs at every world size."""
    if not 0 <= rank < world:
        raise ValueError("rank out of range")
    return partition_replicas(n_atoms, world)[rank]


def allreduce_sum(values, group=None):
    """Element-wise sum over the ranks of a float64 array (the local array when no process
    group is initialised); used for set-up sums such as a replica-mean target."""
    import torch
    import torch.distributed as dist
    v = np.asarray(values, dtype=np.float64)
    if not (dist.is_available() and dist.is_initialized()):
        return v.copy()
    device = torch.device("cuda", torch.cuda.current_device()) \
        if dist.get_backend(group) == "nccl" else torch.device("cpu")
    t = torch.from_numpy(v.copy()).to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy()


def allreduce_mean(grads, group=None):
    """Mean over every replica of every rank of the per-replica gradients.

    grads: [n_local, P] this rank's per-replica gradients (n_local may be 0).  One
    all-reduce of the local sums and the local count; every rank returns the same mean
    [P].  Without an initialised process group the local mean is returned."""
    import torch
    import torch.distributed as dist
    g = np.asarray(grads, dtype=np.float64).reshape(len(grads), -1) if len(grads) else None
    if not (dist.is_available() and dist.is_initialized()):
        if g is None:
            raise ValueError("no replicas")
        return g.mean(axis=0)
    P = g.shape[1] if g is not None else None
    sizes = [None] * dist.get_world_size(group)
    dist.all_gather_object(sizes, P, group=group)
    P = next(s for s in sizes if s is not None)
    buf = np.zeros(P + 1)
    if g is not None:
        buf[:P] = g.sum(axis=0)
        buf[P] = len(g)
    device = torch.device("cuda", torch.cuda.current_device()) \
        if dist.get_backend(group) == "nccl" else torch.device("cpu")
    t = torch.from_numpy(buf).to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    out = t.cpu().numpy()
    return out[:P] / out[P]
