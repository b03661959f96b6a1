"""The query roofline model bench.py reports (bytes per query: the key, the
answer, and one node fetch per level below the L2-resident depth) at the
workloads' shapes."""
import os
import sys

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), ".."))
import bench  # noqa: E402


def test_btree_headline_shape():
    # b = 16 over 5e8 u64: 8 levels, levels 0..4 (11.4 MB) fit in half of L2,
    # levels 5, 6, 7 cost a 128-byte node each
    assert bench.query_bytes_model("btree", 500_000_000, 16, 8) == (8 + 8 + 3 * 128, 5, 8)


def test_veb_and_bst_shapes():
    # mvEB 2^30 - 1 u32: 30 levels, 23 in half of L2, 7 sectors of 32 bytes
    assert bench.query_bytes_model("mveb", 2**30 - 1, 1, 4) == (4 + 8 + 7 * 32, 23, 30)
    # the reference's CPU case: all 20 levels of a 2^20 - 1 BST sit in L2
    assert bench.query_bytes_model("bst", 2**20 - 1, 1, 8) == (16, 20, 20)


def test_partial_last_level_counts_as_a_level():
    # 17^3 - 1 + 5 keys, b = 16: a perfect 3-level top tree and a last level of 5 keys
    nbytes, l2, levels = bench.query_bytes_model("btree", 17**3 - 1 + 5, 16, 8)
    assert levels == 4 and l2 == 4 and nbytes == 16
