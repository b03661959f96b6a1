"""The reverse permutation (layout -> sorted order) through the C ABI.

The reference has no reverse permutation; its forward layouts, as the oracle
restates them, are the inputs: bit-exact on seeded keys at sizes the oracle
finishes in seconds (every size 1..300, tile and unit boundaries, both key
widths), and at the benchmark's sizes a round trip permute -> unpermute that
must give back the input exactly.
"""
import numpy as np
import pytest

import oracle as O
import tree_layouts as T
from gpu_util import from_dev, to_dev
from tree_layouts import data

pytestmark = pytest.mark.gpu

CASES = [("bst", 1), ("btree", 2), ("btree", 3), ("btree", 8), ("btree", 16), ("btree", 32), ("mveb", 0), ("veb", 0)]
EDGE = [511, 4095, 4096, 4097, 8191, 8192, 8193, 65535, 65537, 83521, 262143, 300001, 1048575, 3000017]


@pytest.mark.parametrize("layout,b", CASES)
@pytest.mark.parametrize("dtype", [np.uint64, np.uint32])
def test_oracle_layouts_back_to_sorted(layout, b, dtype):
    for n in list(range(1, 301, 7)) + EDGE:
        keys = data.sorted_keys_np(n, 1, 3, 13 + n, dtype)
        t = to_dev(O.permute(layout, keys, b or 16))
        T.unpermute(layout, t, b or 16)
        assert np.array_equal(from_dev(t), keys), (layout, b, n)


def test_caller_workspace_timing_and_too_small():
    import torch
    n = 1_000_003
    keys = data.sorted_keys_np(n, 1, 16, 3)
    t = to_dev(O.permute("btree", keys, 16))
    need = T.lib().tl_unpermute_workspace_bytes
    import ctypes as C
    out = C.c_uint64()
    assert need(1, n, 16, 8, C.byref(out)) == 0
    ws = torch.empty(out.value, dtype=torch.uint8, device="cuda")
    assert T.unpermute("btree", t, 16, workspace=ws, timed=True) > 0
    assert np.array_equal(from_dev(t), keys)
    small = torch.empty(out.value - 256, dtype=torch.uint8, device="cuda")
    with pytest.raises(T.TreeLayoutError) as e:
        T.unpermute("btree", t, 16, workspace=small)
    assert e.value.status == T.ERROR_WORKSPACE_TOO_SMALL
    assert np.array_equal(from_dev(t), keys)  # rejected before any device work


@pytest.mark.parametrize("layout,b,n,kb,gap", [
    ("btree", 16, 500_000_000, 8, 16),
    ("bst", 1, 2**28 - 1, 8, 16),
    ("btree", 8, 60_000_000, 8, 16),
    ("mveb", 0, 2**30 - 1, 4, 3),
    ("veb", 0, 300_000_000, 4, 3),
])
def test_full_size_round_trip(layout, b, n, kb, gap):
    import torch
    keys = data.sorted_keys_torch(n, 1, gap, 17, kb)
    t = keys.clone()
    T.permute(layout, t, b)
    assert not torch.equal(t, keys)
    T.unpermute(layout, t, b)
    assert torch.equal(t, keys)
