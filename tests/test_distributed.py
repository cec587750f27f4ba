"""The multi-rank path on CPU (gloo, world size 2): replica sharding by atom-count balance
and the gradient exchange of a parameter update (one all-reduce), as the GPU ranks run it
with NCCL."""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from revsim.distributed import allreduce_mean, partition_replicas


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
