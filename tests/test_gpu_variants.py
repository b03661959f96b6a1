"""The reference's BST-by-involutions family as a variant of the permutation
(tl_permute_algorithm), through the C ABI: bit-exact against the oracle at
sizes it finishes in seconds (perfect and non-perfect trees, both key widths)
and equal to the library's own stream permutation at larger sizes."""
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
