"""The cycle-leader family's step lists (tl_permute_algorithm "cycles" and
"hybrid"), replayed on the host with the kernels' step semantics
(tl_debug_emulate_algorithm), reproduce the oracle's layouts: every size up
to 400, node widths 1 .. 100, perfect, power-of-power and ragged sizes."""
import numpy as np
import pytest

import oracle as O
import tree_layouts as T

RNG_SIZES = [int(x) for x in np.random.default_rng(1).integers(300, 2_000_000, 4)]


@pytest.mark.parametrize("layout,b", [("btree", 1), ("btree", 2), ("btree", 3), ("btree", 4), ("btree", 5),
                                      ("btree", 8), ("btree", 16), ("btree", 32), ("btree", 100), ("bst", 1),
                                      ("mveb", 0)])
def test_cycles_replay_matches_oracle(layout, b):
    sizes = list(range(1, 401)) + RNG_SIZES + [17**5 - 1, 17**5, 2**21 - 1, 2**20 + 5, 9**6, 5**8 - 1, 125]
    for n in sizes:
        got, _ = T.emulate_algorithm(layout, "cycles", np.arange(n, dtype=np.uint64), b or 1)
        assert np.array_equal(got, O.permutation(layout, n, b or 16)), (layout, b, n)


def test_hybrid_replay_matches_oracle():
    for n in list(range(1, 401)) + RNG_SIZES + [2**21 - 1, 2**20 + 5]:
        got, _ = T.emulate_algorithm("bst", "hybrid", np.arange(n, dtype=np.uint64), 1)
        assert np.array_equal(got, O.permutation("bst", n)), n


def test_cycles_step_counts_grow_with_depth():
    # the B-tree rounds: one gather per round and level, two extra steps for
    # the last level of a non-perfect tree
    _, perfect = T.emulate_algorithm("btree", "cycles", np.arange(17**4 - 1, dtype=np.uint64), 16)
    _, ragged = T.emulate_algorithm("btree", "cycles", np.arange(17**4 + 1000, dtype=np.uint64), 16)
    assert 0 < perfect < ragged < 64
