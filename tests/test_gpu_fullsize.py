"""Bit-exact parity at the benchmark workloads' full sizes.

Every permuted array is compared word for word with the reference's own CPU
permutation of the same keys (B-tree, BST, standard vEB; compiled from its
sources) or, for the mvEB, which the reference builds only on the GPU, with the
oracle's restatement pinned to that GPU code.  Query answers are compared with
the reference's CPU search (B-tree, BST) or the oracle's search (vEB layouts)
on a seeded sample of each full-size batch; the batched mode checks all 4096
instances and every answer.  Workloads:

  B-tree b = 16, n = 5e8 uint64 (gaps [1,16], seed 3; 2^27 queries, seed 4)
  B-tree b = 16, n = 2^30 skewed uint64 (seed 8; 2^28 Zipf queries, seed 9),
      plain and learned-start queries
  BST n = 2^30 - 1 uint64 (gaps [1,16], seed 1; 2^27 queries, seed 2)
  mvEB and standard vEB, n = 2^30 - 1 and 3e8 uint32 (gaps [1,3], seed 5;
      2^27 queries, seed 6)
  batched: 4096 uint64 arrays, sizes log-uniform in [2^10, 2^22] (seed 7),
      gaps [1,64], b = 8; 2^26 queries, 70 % hits (seed 8)
"""
import numpy as np
import pytest

import parity as P
import tree_layouts as T
from tree_layouts import data

pytestmark = pytest.mark.gpu

SAMPLE = 1 << 22  # answers compared with the CPU checker per full-size batch


def _layout_and_queries(layout, b, n, kb, gap, kseed, q, qseed):
    import torch
    keys = data.sorted_keys_torch(n, 1, gap, kseed, kb)
    Q = data.queries_torch(keys, q, 0.5, qseed)
    tree = keys.clone()
    T.permute(layout, tree, b)
    rep, host = P.check_layout(layout, b, keys, tree, keep_host=True)
    assert rep["bit_exact"], f"{layout} n={n}: layout differs from {rep['checker']}"
    del keys
    ans = torch.empty(q, dtype=torch.int64, device="cuda")
    T.query(layout, tree, Q, ans, b)
    rep = P.check_answers(layout, b, host, Q, ans, SAMPLE, qseed)
    assert rep["exact"], rep
    del tree, Q, ans
    torch.cuda.empty_cache()


def test_btree_b16_500M_u64():
    _layout_and_queries("btree", 16, 500_000_000, 8, 16, 3, 2**27, 4)


def test_bst_2e30m1_u64():
    _layout_and_queries("bst", 1, 2**30 - 1, 8, 16, 1, 2**27, 2)


@pytest.mark.parametrize("layout", ["mveb", "veb"])
@pytest.mark.parametrize("n", [2**30 - 1, 300_000_000])
def test_veb_layouts_u32(layout, n):
    _layout_and_queries(layout, 0, n, 4, 3, 5, 2**27, 6)


def test_btree_b16_2e30_skewed_plain_and_learned():
    import torch

    import tree_layouts.learned as LL
    n, b, q = 2**30, 16, 2**28
    keys = data.skewed_keys_torch(n, 8)
    model, leaves = LL.train(keys, num_leaves=65536, steps=600, batch=65536, lr=3e-3, seed=1)
    Q = data.zipf_queries_torch(keys, q, 9)
    tree = keys.clone()
    T.permute("btree", tree, b)
    rep, host = P.check_layout("btree", b, keys, tree, keep_host=True)
    assert rep["bit_exact"], f"layout differs from {rep['checker']}"
    del keys
    plain = torch.empty(q, dtype=torch.int64, device="cuda")
    learned = torch.empty_like(plain)
    T.query("btree", tree, Q, plain, b)
    LL.query(tree, model, leaves, Q, learned, b)
    assert torch.equal(plain, learned)  # every one of the 2^28 answers
    rep = P.check_answers("btree", b, host, Q, plain, SAMPLE, 9)
    assert rep["exact"], rep
    del tree, Q, plain, learned
    torch.cuda.empty_cache()


def test_batched_4096_arrays_b8():
    import torch

    import tree_layouts.batched as TB
    b = 8
    sizes = TB.batch_sizes_np(4096, 10, 22, 7)
    keys, off = data.batch_keys_torch(sizes, 64, 7)
    Q, inst = data.batch_queries_torch(keys, off, 2**26, 0.7, 8)
    tree = keys.clone()
    plan = TB.BatchPlan(off, b=b)
    plan.permute(tree)
    ans = torch.empty(Q.numel(), dtype=torch.int64, device="cuda")
    plan.query(tree, Q, inst, ans)
    rep = P.check_batched(b, sizes, keys, tree, off, Q, inst, ans)
    assert rep["bit_exact"], f"an instance differs from {rep['checker']}"
    assert rep["answers_exact"], "a batched answer is wrong"
    del keys
    # a seeded sample against the reference's CPU search, instance by instance
    offs = off.cpu().numpy()
    host = P.host_u64(tree)
    rng = np.random.default_rng(8)
    idx = np.sort(rng.choice(Q.numel(), size=1 << 18, replace=False))
    it = torch.from_numpy(idx).cuda()
    qs, js, got = P.host_u64(Q[it]), inst[it].cpu().numpy(), ans[it].cpu().numpy().view(np.uint64)
    for j in np.unique(js):
        sel = js == j
        e, _ = P.answers("btree", host[offs[j]:offs[j + 1]], qs[sel], b)
        assert np.array_equal(got[sel], e), f"instance {j}"
    del tree, Q, inst, ans
    torch.cuda.empty_cache()
