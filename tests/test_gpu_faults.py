"""Failure detection on the GPU without faulting it: every device wait in the
stream kernel is bounded.  Here the waits are made to expect a flag value that
no tile ever publishes, with a short bound; the call must come back with
TL_ERROR_TIMEOUT (no hang, no trap) and the context must stay usable."""
import numpy as np
import pytest

import oracle as O
import tree_layouts as T
from gpu_util import from_dev, to_dev
from tree_layouts import data

pytestmark = pytest.mark.gpu


def test_expired_wait_reports_timeout_and_context_survives():
    n = 2_000_003
    keys = data.sorted_keys_np(n, 1, 16, 1)
    t = to_dev(keys)
    T.set_wait(spin_limit=64, force_timeout=True)
    try:
        with pytest.raises(T.TreeLayoutError) as ei:
            T.permute("btree", t, 16)
        assert ei.value.status == T.ERROR_TIMEOUT
    finally:
        T.set_wait(0, False)
    t = to_dev(keys)
    T.permute("btree", t, 16)
    assert np.array_equal(from_dev(t), O.permute("btree", keys, 16))


def test_invalid_width_and_null_query_buffers():
    import torch
    with pytest.raises(T.TreeLayoutError) as ei:
        T.query("btree", torch.zeros(10, dtype=torch.int64, device="cuda"),
                torch.zeros(4, dtype=torch.int64, device="cuda"), torch.zeros(0, dtype=torch.int64, device="cuda"),
                b=0)
    assert ei.value.status == T.ERROR_INVALID_VALUE
