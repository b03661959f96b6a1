"""The full-size parity checkers (oracle/parity.py) agree with the oracle at
sizes both finish quickly: the reference's CPU permutations and searches they
call, the widening of 4-byte keys, the padding the reference's B-tree search
needs, the per-instance batched path, and the sizes where the reference's own
level count fails and the oracle stands in."""
import numpy as np
import pytest

import oracle as O
import parity as P
from tree_layouts import data


@pytest.mark.parametrize("layout,b", [("btree", 16), ("btree", 8), ("btree", 4), ("bst", 1), ("mveb", 0),
                                      ("veb", 0)])
@pytest.mark.parametrize("dtype", [np.uint64, np.uint32])
def test_layout_checker_matches_oracle(layout, b, dtype):
    for n in [1, 2, 3, 17, 124, 125, 126, 4096, 65535, 100_003, 1_048_575]:
        keys = data.sorted_keys_np(n, 1, 3, n, dtype)
        got = keys.copy()
        P.layout_inplace(layout, got, b or 16)
        assert np.array_equal(got, O.permute(layout, keys, b or 16)), (layout, b, n)


def test_level_count_guard():
    assert not P.ref_level_count_ok(125, 4)  # log10(125)/log10(5) rounds below 3
    assert P.ref_level_count_ok(124, 4)
    assert not P.ref_level_count_ok(5, 16)  # n < b
    assert P.ref_level_count_ok(500_000_000, 16) and P.ref_level_count_ok(2**30, 16)


def test_batched_checker_matches_oracle():
    sizes = np.array([1024, 1, 0, 5000, 9**4, 70001, 2], dtype=np.int64)
    off = np.zeros(len(sizes) + 1, dtype=np.int64)
    np.cumsum(sizes, out=off[1:])
    keys = np.concatenate([data.sorted_keys_np(int(n), 1, 64, i) for i, n in enumerate(sizes)])
    got = keys.copy()
    P.batched_layout_inplace(got, off, 8)
    for j in range(len(sizes)):
        s, e = off[j], off[j + 1]
        assert np.array_equal(got[s:e], O.permute("btree", keys[s:e], 8)), j


@pytest.mark.parametrize("layout,b", [("btree", 16), ("btree", 3), ("bst", 1), ("mveb", 0), ("veb", 0)])
def test_answer_checker_matches_oracle(layout, b):
    for n, dtype in [(1_000_003, np.uint64), (65535, np.uint32), (2**20 - 1, np.uint64)]:
        keys = data.sorted_keys_np(n, 1, 3, n, dtype)
        tree = O.permute(layout, keys, b or 16)
        Q = data.queries_np(keys, 20_000, 0.5, 1)
        exp = O.search(layout, tree, Q, b or 16)
        got, _ = P.answers(layout, tree, Q, b or 16)
        assert np.array_equal(got, exp), (layout, n)
        if layout == "btree" and dtype == np.uint64:
            buf, view = P.padded(n, b)
            view[:] = tree
            got, _ = P.answers(layout, view, Q, b, tree_padded=True)
            assert np.array_equal(got, exp)
