"""Multi-rank paths on CPU (gloo, world size 2): query batches split across
replicas and batched instances dealt across ranks reproduce the single-rank
results exactly; no rank's data depends on another's."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import oracle as O
from tree_layouts import data, shard


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_query_slices_cover_the_batch():
    for q in (0, 1, 7, 1000, 12345):
        for world in (1, 2, 3, 8):
            cuts = [shard.query_slice(q, r, world) for r in range(world)]
            assert cuts[0][0] == 0 and cuts[-1][1] == q
            assert all(a[1] == b[0] for a, b in zip(cuts, cuts[1:]))
            assert max(h - l for l, h in cuts) - min(h - l for l, h in cuts) <= 1


def test_instances_balance_by_keys():
    sizes = np.floor(2.0 ** np.random.default_rng(7).uniform(10, 22, 4096)).astype(np.int64)
    for world in (2, 4, 8):
        owner = shard.assign_instances(sizes, world)
        loads = np.bincount(owner, weights=sizes, minlength=world)
        assert loads.max() / loads.mean() < 1.01
        assert sorted(np.unique(owner)) == list(range(world))


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # replicated layout, sharded queries
        keys = data.sorted_keys_np(100_003, 1, 16, 3)
        tree = O.permute("btree", keys, 16)
        Q = data.queries_np(keys, 10_001, 0.5, 4)
        lo, hi = shard.query_slice(len(Q), rank, world)
        local = torch.from_numpy(O.search("btree", tree, Q[lo:hi], 16).view(np.int64))
        allans = shard.gather_answers(local, len(Q), world)
        # dealt instances, each rank permuting only its own
        sizes = np.floor(2.0 ** np.random.default_rng(1).uniform(4, 12, 64)).astype(np.int64)
        owner = shard.assign_instances(sizes, world)
        mine, offs = shard.local_batch(sizes, owner, rank)
        perms = {int(j): O.permutation("btree", int(sizes[j]), 8).tolist() for j in mine}
        gathered = [None] * world
        dist.all_gather_object(gathered, perms)
        if rank == 0:
            merged = {}
            for g in gathered:
                merged.update(g)
            out.put((allans.numpy(), merged, [int(x) for x in offs]))
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_paths_match_single_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = mp.spawn(_worker, args=(2, port, q), nprocs=2, join=False)
    answers, perms, _ = q.get(timeout=120)  # read before joining: a child holding queued data cannot exit
    while not procs.join(timeout=60):
        pass
    keys = data.sorted_keys_np(100_003, 1, 16, 3)
    tree = O.permute("btree", keys, 16)
    Q = data.queries_np(keys, 10_001, 0.5, 4)
    assert np.array_equal(answers.view(np.uint64), O.search("btree", tree, Q, 16))
    sizes = np.floor(2.0 ** np.random.default_rng(1).uniform(4, 12, 64)).astype(np.int64)
    assert sorted(perms) == list(range(len(sizes)))
    for j, p in perms.items():
        assert p == O.permutation("btree", int(sizes[j]), 8).tolist()
