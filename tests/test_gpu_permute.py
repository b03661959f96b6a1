"""Parity of the sm_100a permutations with the oracle, through the C ABI.

Bit-exact on seeded inputs at sizes the oracle finishes in seconds (every size
1..300, tile and unit boundaries, perfect and non-perfect trees, both key
widths, unaligned base pointers, caller-supplied workspace); at the benchmark's
full sizes through size-independent properties: the result is a permutation of
the input, sampled positions equal the layout formula, and a query for every
key finds it.
"""
import numpy as np
import pytest

import oracle as O
import tree_layouts as T
from gpu_util import from_dev, to_dev
from tree_layouts import data

pytestmark = pytest.mark.gpu

SMALL = list(range(1, 301))
EDGE = [511, 512, 1023, 1024, 4095, 4096, 4097, 8191, 8192, 8193, 16383, 16385, 65535, 65536, 65537,
        83520, 83521, 100003, 131071, 262143, 300001, 1048575, 1048576, 2097151, 3000017]
CASES = [("bst", 1), ("btree", 2), ("btree", 3), ("btree", 8), ("btree", 16), ("btree", 17), ("btree", 32),
         ("mveb", 0), ("veb", 0)]


def run(layout, keys, b, **kw):
    t = to_dev(keys)
    T.permute(layout, t, b or 16, **kw)
    return from_dev(t)


@pytest.mark.parametrize("layout,b", CASES)
@pytest.mark.parametrize("dtype", [np.uint64, np.uint32])
def test_small_sizes_bit_exact(layout, b, dtype):
    for n in SMALL:
        keys = data.sorted_keys_np(n, 1, 4, n, dtype)
        assert np.array_equal(run(layout, keys, b), O.permute(layout, keys, b or 16)), (layout, b, n)


@pytest.mark.parametrize("layout,b", CASES)
@pytest.mark.parametrize("dtype", [np.uint64, np.uint32])
def test_edge_sizes_bit_exact(layout, b, dtype):
    for n in EDGE:
        keys = data.sorted_keys_np(n, 1, 3, 7 + n, dtype)
        assert np.array_equal(run(layout, keys, b), O.permute(layout, keys, b or 16)), (layout, b, n)


@pytest.mark.parametrize("layout,b", [("bst", 1), ("btree", 16), ("mveb", 0), ("veb", 0)])
@pytest.mark.parametrize("dtype", [np.uint64, np.uint32])
def test_unaligned_base_pointer(layout, b, dtype):
    import torch
    for n, off in [(100003, 1), (70001, 3), (8193, 1)]:
        keys = data.sorted_keys_np(n, 1, 5, n, dtype)
        buf = to_dev(np.concatenate([np.zeros(off, dtype), keys, np.zeros(5, dtype)]))
        view = buf[off:off + n]
        T.permute(layout, view, b or 16)
        out = from_dev(buf)
        assert np.array_equal(out[off:off + n], O.permute(layout, keys, b or 16))
        assert (out[:off] == 0).all() and (out[off + n:] == 0).all()  # nothing outside [0, n) touched
        torch.cuda.synchronize()


def test_caller_supplied_workspace_and_timing():
    import torch
    n = 1_000_003
    keys = data.sorted_keys_np(n, 1, 16, 3)
    t = to_dev(keys)
    ws = torch.empty(T.workspace_bytes("btree", n, 16, 8), dtype=torch.uint8, device="cuda")
    ms = T.permute("btree", t, 16, workspace=ws, timed=True)
    assert ms > 0
    assert np.array_equal(from_dev(t), O.permute("btree", keys, 16))


@pytest.mark.parametrize("layout,b,n,dtype", [
    ("btree", 16, 20_000_000, np.uint64),
    ("bst", 1, 2**23 - 1, np.uint64),
    ("mveb", 0, 2**24 - 1, np.uint32),
    ("mveb", 0, 30_000_001, np.uint32),
    ("btree", 8, 9_999_991, np.uint64),
    ("veb", 0, 2**23 - 1, np.uint64),
    ("veb", 0, 2**24 + 12_345, np.uint32),
])
def test_medium_sizes_bit_exact(layout, b, n, dtype):
    keys = data.sorted_keys_np(n, 1, 3 if dtype == np.uint32 else 16, n % 1000, dtype)
    assert np.array_equal(run(layout, keys, b), O.permute(layout, keys, b or 16))


def _full_size_properties(layout, b, n, key_bytes, gap):
    """Permute n keys generated in HBM; check permutation, sampled positions and
    that a query for every key returns its position."""
    import torch
    keys = data.sorted_keys_torch(n, 1, gap, 11, key_bytes)
    tree = keys.clone()
    T.permute(layout, tree, b)
    # multiset preserved: sorting the layout gives back the keys (unsigned order)
    srt = torch.sort(tree.view(torch.int64) if key_bytes == 8 else tree.to(torch.int64) & 0xFFFFFFFF)[0]
    ref = keys.view(torch.int64) if key_bytes == 8 else keys.to(torch.int64) & 0xFFFFFFFF
    if key_bytes == 8:
        assert torch.equal(srt, ref)  # keys < 2^63 here: signed order == unsigned order
    else:
        assert torch.equal(srt, ref)
    del srt
    rng = np.random.default_rng(5)
    ranks = np.concatenate([rng.integers(0, n, 2000), [0, n - 1, n // 2]])
    pos = torch.tensor([T.layout_position(layout, n, int(s), b) for s in ranks], device="cuda")
    assert torch.equal(tree[pos], keys[torch.from_numpy(ranks).cuda()])
    ans = torch.empty(n, dtype=torch.int64, device="cuda")
    T.query(layout, tree, keys, ans, b)
    assert torch.equal(tree[ans], keys)
    assert int(ans.max()) < n


@pytest.mark.parametrize("layout,b,n,kb,gap", [
    ("btree", 16, 500_000_000, 8, 16),
    ("mveb", 0, 2**30 - 1, 4, 3),
    ("mveb", 0, 300_000_000, 4, 3),
    ("bst", 1, 2**28 - 1, 8, 16),
    ("btree", 16, 2**28, 8, 16),
    ("veb", 0, 2**30 - 1, 4, 3),
    ("veb", 0, 300_000_000, 4, 3),
])
def test_full_size_properties(layout, b, n, kb, gap):
    _full_size_properties(layout, b, n, kb, gap)


@pytest.mark.parametrize("layout,b,n,kb", [("btree", 16, 500_000_000, 8), ("btree", 16, 2**30, 8),
                                           ("btree", 8, 60_000_000, 8), ("btree", 3, 20_000_000, 8),
                                           ("btree", 2, 9_999_991, 4), ("btree", 17, 123_456_789, 8),
                                           ("btree", 32, 2**27, 4), ("bst", 1, 2**30 - 1, 8),
                                           ("bst", 1, 2**26 + 12345, 4), ("btree", 16, 2**20 + 7, 8)])
def test_ordered_tables_gpu_build_equals_host_build(layout, b, n, kb):
    """A permutation of a geometry not seen before computes its ordered-tile
    tables with two kernels (each tile's predecessor, each tile's scratch count
    under both tie orders) and the chain walk on the host; the result is the
    host build's, entry by entry (tickets, scratch slots, bulk ranges, fix
    segments)."""
    import ctypes as C
    L = T.lib()
    L.tl_debug_order_tables_match.argtypes = [C.c_int, C.c_uint64, C.c_uint64, C.c_uint32, C.c_void_p]
    assert L.tl_debug_order_tables_match(T.LAYOUTS[layout], n, b, kb, None) == 1, (layout, b, n, kb)
