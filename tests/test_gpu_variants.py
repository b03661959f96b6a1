"""The reference's involutions and cycle-leader families (BST, B-tree, mvEB)
and its hybrid BST as variants of the permutation (tl_permute_algorithm),
through the C ABI: bit-exact against the oracle at sizes it finishes in
seconds (perfect and non-perfect trees, both key widths, leaves with and
without full nodes) and equal to the library's own stream permutation at
larger sizes."""
import numpy as np
import pytest

import oracle as O
import tree_layouts as T
from gpu_util import from_dev, to_dev
from tree_layouts import data

pytestmark = pytest.mark.gpu

SIZES = list(range(1, 260)) + [511, 512, 1023, 1025, 4095, 4097, 65535, 65537, 100003, 1048575, 3000017]


@pytest.mark.parametrize("dtype", [np.uint64, np.uint32])
def test_bst_involutions_bit_exact(dtype):
    for n in SIZES:
        keys = data.sorted_keys_np(n, 1, 3, 29 + n, dtype)
        t = to_dev(keys)
        T.permute_algorithm("bst", "involutions", t, 1)
        assert np.array_equal(from_dev(t), O.permute("bst", keys, 1)), n


@pytest.mark.parametrize("n", [2**26 - 1, 50_000_017])
def test_bst_involutions_equal_stream(n):
    import torch
    keys = data.sorted_keys_torch(n, 1, 16, 31, 8)
    a, s = keys.clone(), keys.clone()
    assert T.permute_algorithm("bst", "involutions", a, 1, timed=True) > 0
    T.permute_algorithm("bst", "stream", s, 1)
    assert torch.equal(a, s)


BTREE_SIZES = {
    2: list(range(1, 120)) + [3**9 - 1, 3**9, 3**9 + 5, 100003],
    3: list(range(1, 90)) + [4**7 - 1, 4**7 + 2, 70001],
    8: list(range(1, 100)) + [9**4 - 1, 9**4, 9**5 - 1, 9**5 + 9, 654321],
    16: [1, 15, 16, 17, 33, 288, 289, 290, 17**3 - 1, 17**3 + 16, 17**4 - 1, 17**4 + 100, 1000003],
    1: [1, 2, 3, 7, 8, 100, 4095, 4097],
    33: [5, 33, 34, 100, 1155, 34**3 - 1, 50000],
}


@pytest.mark.parametrize("b", sorted(BTREE_SIZES))
@pytest.mark.parametrize("dtype", [np.uint64, np.uint32])
def test_btree_involutions_bit_exact(b, dtype):
    for n in BTREE_SIZES[b]:
        keys = data.sorted_keys_np(n, 1, 3, 17 + n, dtype)
        t = to_dev(keys)
        T.permute_algorithm("btree", "involutions", t, b)
        assert np.array_equal(from_dev(t), O.permute("btree", keys, b)), (b, n)


@pytest.mark.parametrize("n,b", [(17**6 - 1, 16), (50_000_017, 16), (9**8 - 1, 8), (30_000_001, 8)])
def test_btree_involutions_equal_stream(n, b):
    import torch
    keys = data.sorted_keys_torch(n, 1, 16, 37, 8)
    a, s = keys.clone(), keys.clone()
    assert T.permute_algorithm("btree", "involutions", a, b, timed=True) > 0
    T.permute_algorithm("btree", "stream", s, b)
    assert torch.equal(a, s)


MVEB_SIZES = list(range(1, 300)) + [511, 1023, 1024, 2047, 4095, 4097, 32767, 65535, 65536, 70001, 2**20 - 1,
                                    1_000_003]


@pytest.mark.parametrize("dtype", [np.uint32, np.uint64])
def test_mveb_involutions_bit_exact(dtype):
    for n in MVEB_SIZES:
        keys = data.sorted_keys_np(n, 1, 3, 23 + n, dtype)
        t = to_dev(keys)
        T.permute_algorithm("mveb", "involutions", t, 1)
        assert np.array_equal(from_dev(t), O.permute("mveb", keys, 1)), n


@pytest.mark.parametrize("n,kb", [(2**24 - 1, 4), (2**16 * 300 + 7, 4), (30_000_001, 8)])
def test_mveb_involutions_equal_stream(n, kb):
    import torch
    keys = data.sorted_keys_torch(n, 1, 3, 41, kb)
    a, s = keys.clone(), keys.clone()
    assert T.permute_algorithm("mveb", "involutions", a, 1, timed=True) > 0
    T.permute_algorithm("mveb", "stream", s, 1)
    assert torch.equal(a, s)


CYCLE_CASES = [("btree", b) for b in sorted(BTREE_SIZES)] + [("bst", 1), ("mveb", 0)]


def _cycle_sizes(layout, b):
    if layout == "btree":
        return BTREE_SIZES[b]
    if layout == "bst":
        return SIZES
    return MVEB_SIZES


@pytest.mark.parametrize("layout,b", CYCLE_CASES)
@pytest.mark.parametrize("dtype", [np.uint64, np.uint32])
def test_cycles_bit_exact(layout, b, dtype):
    for n in _cycle_sizes(layout, b):
        keys = data.sorted_keys_np(n, 1, 3, 19 + n, dtype)
        t = to_dev(keys)
        T.permute_algorithm(layout, "cycles", t, b or 1)
        assert np.array_equal(from_dev(t), O.permute(layout, keys, b or 16)), (layout, b, n)


@pytest.mark.parametrize("dtype", [np.uint64, np.uint32])
def test_hybrid_bst_bit_exact(dtype):
    for n in SIZES:
        keys = data.sorted_keys_np(n, 1, 3, 43 + n, dtype)
        t = to_dev(keys)
        T.permute_algorithm("bst", "hybrid", t, 1)
        assert np.array_equal(from_dev(t), O.permute("bst", keys, 1)), n


@pytest.mark.parametrize("layout,algo,n,b,kb", [
    ("btree", "cycles", 17**6 - 1, 16, 8), ("btree", "cycles", 30_000_001, 16, 8), ("btree", "cycles", 9**7 + 3, 8, 4),
    ("bst", "cycles", 2**24 - 1, 1, 8), ("bst", "cycles", 20_000_003, 1, 4), ("bst", "hybrid", 2**24 - 1, 1, 8),
    ("bst", "hybrid", 20_000_003, 1, 8), ("mveb", "cycles", 2**24 - 1, 0, 4), ("mveb", "cycles", 30_000_001, 0, 4),
])
def test_cycles_equal_stream(layout, algo, n, b, kb):
    import torch
    keys = data.sorted_keys_torch(n, 1, 3, 47, kb)
    a, s = keys.clone(), keys.clone()
    assert T.permute_algorithm(layout, algo, a, b or 1, timed=True) > 0
    T.permute_algorithm(layout, "stream", s, b or 16)
    assert torch.equal(a, s)


def test_variants_refuse_what_they_do_not_build():
    import torch
    t = torch.zeros(100, dtype=torch.int64, device="cuda")
    for layout, algo in [("veb", "cycles"), ("btree", "hybrid"), ("mveb", "hybrid"), ("veb", "involutions")]:
        with pytest.raises(T.TreeLayoutError) as e:
            T.permute_algorithm(layout, algo, t, 4)
        assert e.value.status == T.ERROR_UNSUPPORTED
