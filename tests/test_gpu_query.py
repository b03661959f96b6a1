"""Parity of the sm_100a query kernels with the oracle (and, through the golden
fixtures, with the reference's own query code), through the C ABI."""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle as O
import tree_layouts as T
from gpu_util import from_dev, to_dev
from tree_layouts import data

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.uint64).tobytes()).hexdigest()[:24]


def gpu_answers(layout, tree, Q, b=16):
    import torch
    ans = torch.empty(len(Q), dtype=torch.int64, device="cuda")
    T.query(layout, to_dev(tree), to_dev(Q), ans, b)
    return ans.cpu().numpy().view(np.uint64)


@pytest.mark.parametrize("layout,b", [("bst", 1), ("btree", 16), ("btree", 8), ("btree", 3), ("btree", 32),
                                      ("btree", 1), ("btree", 64), ("mveb", 0), ("veb", 0)])
@pytest.mark.parametrize("dtype", [np.uint64, np.uint32])
def test_queries_match_oracle(layout, b, dtype):
    for n in [1, 2, 3, 5, 16, 17, 100, 255, 1000, 4097, 65535, 70001, 1048575, 3000017]:
        keys = data.sorted_keys_np(n, 1, 16 if dtype == np.uint64 else 3, n, dtype)
        tree = O.permute(layout, keys, b or 16)
        Q = data.queries_np(keys, 5000, 0.5, n + 1)
        Q = np.concatenate([Q, keys[:1] - 1 if keys[0] > 0 else keys[:1], keys[-1:] + 1]).astype(dtype)
        exp = O.search(layout, tree, Q, b or 16)
        got = gpu_answers(layout, tree, Q, b or 16)
        assert np.array_equal(got, exp), (layout, b, n)


@pytest.mark.parametrize("dtype", [np.uint64, np.uint32])
def test_sorted_binary_search_matches_oracle(dtype):
    for n in [1, 2, 3, 4, 5, 7, 8, 100, 4095, 4096, 8191, 8192, 8193, 65537, 1048575, 3000017]:
        keys = data.sorted_keys_np(n, 1, 16 if dtype == np.uint64 else 3, n + 7, dtype)
        Q = data.queries_np(keys, 5000, 0.5, n + 8)
        edge = [keys[0] - 1 if keys[0] > 0 else keys[0], keys[0], keys[-1], keys[-1] + 1]
        Q = np.concatenate([Q, np.array(edge, dtype=dtype)]).astype(dtype)
        exp = O.search_sorted(keys, Q)
        got = gpu_answers("sorted", keys, Q)
        assert np.array_equal(got, exp), (n, dtype)


def test_queries_match_reference_golden():
    with open(os.path.join(GOLD, "golden_cpu.json")) as f:
        g = json.load(f)
    for e in g["query_btree"]:
        keys = data.sorted_keys_np(e["n"], 1, 16, e["seed"])
        Q = data.queries_np(keys, e["q"], 0.5, e["seed"] + 1)
        assert sha(gpu_answers("btree", O.permute("btree", keys, e["b"]), Q, e["b"])) == e["sha"]
    for e in g["query_bst"]:
        keys = data.sorted_keys_np(e["n"], 1, 16, e["seed"])
        Q = data.queries_np(keys, e["q"], 0.5, e["seed"] + 1)
        assert sha(gpu_answers("bst", O.permute("bst", keys), Q)) == e["sha"]


def test_standard_veb_queries_match_reference_golden():
    with open(os.path.join(GOLD, "golden_cpu.json")) as f:
        g = json.load(f)
    for e in g["query_veb_std"]:
        keys = data.sorted_keys_np(e["n"], 1, 16, e["seed"])
        Q = data.queries_np(keys, e["q"], 1.0, e["seed"] + 1)
        assert sha(gpu_answers("veb", O.permute("veb", keys), Q)) == e["sha"], e["n"]


def test_benchmark_query_shapes_small():
    # config shapes at reduced n: BST 2^20-1 u64 with q=2^20, mvEB non-perfect u32 tables
    keys = data.sorted_keys_np(2**20 - 1, 1, 16, 1)
    Q = data.queries_np(keys, 2**20, 0.5, 2)
    tree = O.permute("bst", keys)
    assert np.array_equal(gpu_answers("bst", tree, Q), O.search("bst", tree, Q))
    keys = data.sorted_keys_np(3_000_000, 1, 3, 5, np.uint32)
    Q = data.queries_np(keys, 200_000, 0.5, 6)
    tree = O.permute("mveb", keys)
    assert np.array_equal(gpu_answers("mveb", tree, Q), O.search("mveb", tree, Q))


@pytest.mark.parametrize("layout,b", [("btree", 16), ("btree", 8), ("btree", 2), ("btree", 32), ("btree", 5),
                                      ("bst", 1), ("mveb", 0)])
@pytest.mark.parametrize("dtype", [np.uint64, np.uint32])
def test_queries_on_an_unaligned_layout(layout, b, dtype):
    """A layout that starts one key past a 16-byte boundary takes the kernels'
    scalar node reads; answers are unchanged."""
    import torch
    for n in [17, 1000, 70001, 1_048_575]:
        keys = data.sorted_keys_np(n, 1, 16 if dtype == np.uint64 else 3, n + 3, dtype)
        tree = O.permute(layout, keys, b or 16)
        Q = data.queries_np(keys, 20_000, 0.5, n + 4)
        buf = to_dev(np.concatenate([np.zeros(1, dtype), tree]))
        view = buf[1:]
        assert view.data_ptr() % 16 != 0
        ans = torch.empty(len(Q), dtype=torch.int64, device="cuda")
        T.query(layout, view, to_dev(Q), ans, b or 16)
        assert np.array_equal(ans.cpu().numpy().view(np.uint64), O.search(layout, tree, Q, b or 16)), (layout, b, n)


@pytest.mark.parametrize("b", [1, 2, 3, 4, 5, 7, 8, 9, 15, 16, 17, 31, 32, 33, 64, 100])
def test_btree_queries_every_node_width(b):
    """Every node width: 16-byte rows, one key per lane (b <= 32), and the
    scalar group kernel (b > 32 without 16-byte rows)."""
    for dtype in (np.uint64, np.uint32):
        for n in [b, b + 1, 5 * b + 3, 100_003]:
            keys = data.sorted_keys_np(n, 1, 16 if dtype == np.uint64 else 3, n + b, dtype)
            tree = O.permute("btree", keys, b)
            Q = data.queries_np(keys, 10_000, 0.5, b)
            Q = np.concatenate([Q, keys[:1] - 1 if keys[0] > 0 else keys[:1], keys[-1:] + 1]).astype(dtype)
            assert np.array_equal(gpu_answers("btree", tree, Q, b), O.search("btree", tree, Q, b)), (b, n, dtype)


@pytest.mark.parametrize("variant", [0, 2, 5, 6])
def test_btree_query_kernel_forms(variant):
    """Each B-tree node-read form gives the oracle's answers: a group of
    b*w/32 lanes with one 32-byte load each (the default for 64-, 128- and
    256-byte nodes), a thread per query with 32-byte loads (variant 6, and with
    the top levels in shared memory, 5) and with 16-byte loads (2); the partial
    last leaf and queries past both ends included."""
    import ctypes as C
    L = T.lib()
    L.tl_debug_set_query_variant.argtypes = [C.c_int]
    L.tl_debug_set_query_variant(variant)
    try:
        for b, dtype in [(4, np.uint64), (8, np.uint64), (16, np.uint64), (32, np.uint64), (8, np.uint32),
                         (16, np.uint32), (32, np.uint32), (64, np.uint32)]:
            for n in [1, b - 1, b, b + 1, 7 * b + 5, 65_537, 1_000_003]:
                if n < 1:
                    continue
                keys = data.sorted_keys_np(n, 1, 16 if dtype == np.uint64 else 3, n + b, dtype)
                tree = O.permute("btree", keys, b)
                Q = data.queries_np(keys, 20_000, 0.5, n + 2)
                Q = np.concatenate([Q, keys[:1] - 1 if keys[0] > 0 else keys[:1], keys[-1:] + 1]).astype(dtype)
                assert np.array_equal(gpu_answers("btree", tree, Q, b), O.search("btree", tree, Q, b)), \
                    (variant, b, n, dtype)
    finally:
        L.tl_debug_set_query_variant(0)


@pytest.mark.parametrize("variant", [0, 3, 4])
@pytest.mark.parametrize("layout", ["mveb", "veb"])
def test_veb_query_kernel_forms(variant, layout):
    """Each vEB descent form gives the oracle's answers, perfect and
    non-perfect trees, u32 and u64: one descent per thread (default), two or
    four in lock-step (3, 4)."""
    import ctypes as C
    L = T.lib()
    L.tl_debug_set_query_variant.argtypes = [C.c_int]
    L.tl_debug_set_query_variant(variant)
    try:
        for dtype in (np.uint32, np.uint64):
            for n in [1, 2, 3, 7, 100, 4095, 65536, 1_000_003, 2**21 - 1]:
                keys = data.sorted_keys_np(n, 1, 3, n + 11, dtype)
                tree = O.permute(layout, keys, 16)
                Q = data.queries_np(keys, 20_000, 0.5, n + 12)
                Q = np.concatenate([Q, keys[:1] - 1 if keys[0] > 0 else keys[:1], keys[-1:] + 1]).astype(dtype)
                assert np.array_equal(gpu_answers(layout, tree, Q), O.search(layout, tree, Q, 16)), \
                    (variant, layout, n, dtype)
    finally:
        L.tl_debug_set_query_variant(0)


@pytest.mark.parametrize("layout,n,kb,q", [("mveb", 2**24 - 1, 4, 2**23), ("bst", 2**23 - 1, 8, 2**23),
                                           ("bst", 2**25 - 1, 8, 2**23), ("mveb", 2**24 - 1, 4, 2**27)])
def test_grouped_queries_at_16_and_20_bucket_bits(layout, n, kb, q):
    """Batches large enough for 16 bucket bits (2^23 queries: four passes) and
    for 20 (2^27: five passes), grouped by default, equal the same batches
    searched as given (variant 19); the 256 MB BST takes the grouped shape
    with the smaller pinned prefix."""
    import ctypes as C

    import torch
    L = T.lib()
    L.tl_debug_set_query_variant.argtypes = [C.c_int]
    keys = data.sorted_keys_torch(n, 1, 3 if kb == 4 else 16, n % 1000 + 3, kb)
    tree = keys.clone()
    T.permute(layout, tree, 16)
    tabs = T.VebTablesDevice(n, "cuda", standard=layout == "veb") if layout != "bst" else None
    Q = data.queries_torch(keys, q, 0.5, 11)
    got = torch.empty(q, dtype=torch.int64, device="cuda")
    exp = torch.empty_like(got)
    T.query(layout, tree, Q, got, 16, tables=tabs)  # default: grouped at these sizes
    try:
        L.tl_debug_set_query_variant(19)
        T.query(layout, tree, Q, exp, 16, tables=tabs)
    finally:
        L.tl_debug_set_query_variant(0)
    assert torch.equal(got, exp), (layout, n, q)
    hit = got != n
    assert torch.equal(tree[got[hit]], Q[hit])


@pytest.mark.parametrize("layout,n,kb", [("mveb", 2**24 - 1, 4), ("mveb", 20_000_003, 4), ("veb", 2**22 - 1, 8),
                                         ("bst", 2**23 - 1, 8), ("bst", 9_000_001, 4)])
def test_partitioned_queries_match_unpartitioned(layout, n, kb):
    """A batch searched grouped by value (a partition of the batch's value
    range into up to 2^20 buckets, 4 bits a pass, answers written back through the carried
    index, vEB descents in 256-thread blocks; variant 20 forces it at any
    size) equals the batch searched as
    given (variant 19) for batch lengths around the partition's 4096-entry
    tiles, with duplicates and a batch of one value; every hit names its key's
    slot and every miss is a key absent from the sorted keys."""
    import ctypes as C

    import torch
    L = T.lib()
    L.tl_debug_set_query_variant.argtypes = [C.c_int]
    keys = data.sorted_keys_torch(n, 1, 3 if kb == 4 else 16, n % 1000 + 1, kb)
    tree = keys.clone()
    T.permute(layout, tree, 16)
    tabs = T.VebTablesDevice(n, "cuda", standard=layout == "veb") if layout != "bst" else None
    Qall = data.queries_torch(keys, 2**21, 0.5, 7)
    Qall[:3] = keys[0]  # duplicates and the smallest key
    for q in [1, 2, 4095, 4096, 4097, 100_003, 2**21]:
        Q = Qall[:q].clone()
        got = torch.empty(q, dtype=torch.int64, device="cuda")
        exp = torch.empty_like(got)
        try:
            L.tl_debug_set_query_variant(20)
            T.query(layout, tree, Q, got, 16, tables=tabs)
            L.tl_debug_set_query_variant(19)
            T.query(layout, tree, Q, exp, 16, tables=tabs)
        finally:
            L.tl_debug_set_query_variant(0)
        assert torch.equal(got, exp), (layout, n, q)
        hit = got != n
        assert torch.equal(tree[got[hit]], Q[hit])
        pos = torch.searchsorted(keys, Q).clamp_max(n - 1)
        assert torch.equal(keys[pos] == Q, hit)
    Q = torch.full((5000,), int(keys[n // 2].item()), dtype=keys.dtype, device="cuda")  # one value
    got = torch.empty(5000, dtype=torch.int64, device="cuda")
    try:
        L.tl_debug_set_query_variant(20)
        T.query(layout, tree, Q, got, 16, tables=tabs)
    finally:
        L.tl_debug_set_query_variant(0)
    assert torch.equal(tree[got], Q)
