"""The multi-rank path on CPU (gloo, world size 2): replica sharding by atom-count balance
and the gradient exchange of a parameter update (one all-reduce), as the GPU ranks run it
with NCCL."""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from revsim.distributed import allreduce_mean, allreduce_sum, partition_replicas, rank_share


def test_partition_balances_atoms_and_is_deterministic():
    rng = np.random.default_rng(2)
    sizes = (3 * np.exp(rng.uniform(np.log(300), np.log(3000), size=64))).astype(int)
    for world in (1, 2, 3, 8):
        parts = partition_replicas(sizes, world)
        assert sorted(i for p in parts for i in p) == list(range(64))
        loads = [sum(sizes[i] for i in p) for p in parts]
        # greedy largest-first: every rank within the largest replica of the mean
        assert max(loads) - min(loads) <= sizes.max()
        assert parts == partition_replicas(list(sizes), world)
    assert partition_replicas([5, 5, 5], 2) == [[0, 2], [1]]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, grads, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        parts = partition_replicas([len(g) for g in grads], world)
        mine = [grads[i] for i in parts[rank]]
        mean = allreduce_mean(np.array(mine) if mine else np.zeros((0, 3)))
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), mean)
    finally:
        dist.destroy_process_group()


def test_two_rank_gradient_mean_equals_the_mean_of_all_replicas(tmp_path):
    rng = np.random.default_rng(5)
    grads = [rng.normal(size=3) * (i + 1) for i in range(5)]
    # spawned ranks (no fork of this multi-threaded process); results through files
    mp.spawn(_worker, args=(2, _free_port(), grads, str(tmp_path)), nprocs=2, join=True)
    res = [np.load(tmp_path / f"rank{r}.npy") for r in range(2)]
    ref = np.mean(grads, axis=0)
    assert np.allclose(res[0], ref, rtol=1e-14, atol=0) and np.array_equal(res[0], res[1])


def test_local_mean_without_a_process_group():
    g = np.arange(6.0).reshape(2, 3)
    assert np.array_equal(allreduce_mean(g), g.mean(axis=0))
    with pytest.raises(ValueError):
        allreduce_mean(np.zeros((0, 3)))


def _replica_rdf(r):
    return np.random.default_rng(100 + r).uniform(0, 2, 200)


def _replica_grad(r, target):
    return np.random.default_rng(200 + r).normal(size=7) * (1 + target[:7])


def _share_worker(rank, world, port, n_atoms, out_dir):
    """The replicas workload's set-up and update on one rank, as bench.py runs it: this rank's
    share, the replica-mean target (sum over ranks), the per-replica gradients of its share
    and their mean over all ranks."""
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = rank_share(n_atoms, world, rank)
        target = allreduce_sum(np.sum([_replica_rdf(r) for r in mine], axis=0)) / len(n_atoms)
        g = np.array([_replica_grad(r, target) for r in mine])
        np.save(os.path.join(out_dir, f"share{rank}.npy"), np.array(mine))
        np.save(os.path.join(out_dir, f"mean{rank}.npy"), allreduce_mean(g))
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas_workload_matches_one_rank(tmp_path):
    rng = np.random.default_rng(2)
    n_atoms = 3 * np.round(np.exp(rng.uniform(np.log(300), np.log(3000), 64))).astype(int)
    mp.spawn(_share_worker, args=(2, _free_port(), n_atoms, str(tmp_path)), nprocs=2, join=True)
    shares = [np.load(tmp_path / f"share{r}.npy") for r in range(2)]
    assert sorted(np.concatenate(shares).tolist()) == list(range(64))
    loads = [int(n_atoms[sh].sum()) for sh in shares]
    assert abs(loads[0] - loads[1]) <= n_atoms.max()
    target = np.mean([_replica_rdf(r) for r in range(64)], axis=0)
    ref = np.mean([_replica_grad(r, target) for r in range(64)], axis=0)
    means = [np.load(tmp_path / f"mean{r}.npy") for r in range(2)]
    assert np.allclose(means[0], ref, rtol=1e-12, atol=1e-14) and np.array_equal(means[0], means[1])
    assert rank_share(n_atoms, 1, 0) == list(range(64))
    with pytest.raises(ValueError):
        rank_share(n_atoms, 2, 2)
