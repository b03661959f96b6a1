"""tl_permute_static_ws: the permutation entry point for callers that cannot
allocate device memory (a plugin whose host engine owns every allocation, a
latency-bound service that must not call cudaMalloc mid-request).  Its
workspace is a fixed array inside the library, so its output must equal the
allocating entry point's (tl_permute) bit for bit, on consecutive calls that
reuse that array, and sizes whose workspace does not fit must be refused.

Collected last (file name) so that a run stopping at the first failure has
run every other test first; it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

import oracle as O
import tree_layouts as T
from tree_layouts import data

pytestmark = pytest.mark.gpu

STATIC_BYTES = 32 << 20


def _lib():
    L = T.lib()
    L.tl_permute_static_ws.argtypes = [C.c_int, C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint32, C.c_void_p]
    return L


def _dev(keys):
    import torch
    view = np.int64 if keys.dtype == np.uint64 else np.int32
    return torch.from_numpy(keys.view(view).copy()).cuda()


def _static(layout, t, b):
    import torch
    rc = _lib().tl_permute_static_ws(T.LAYOUTS[layout], t.data_ptr(), t.numel(), b, t.element_size(),
                                     torch.cuda.current_stream().cuda_stream)
    return rc


@pytest.mark.parametrize("layout,b,sizes,dtype", [
    ("btree", 16, (1_419_856, 2_000_003), np.uint64),
    ("mveb", 0, (2**24 - 1, 3_000_017), np.uint32),
    ("bst", 1, (2**20 - 1, 777_777), np.uint64),
])
def test_static_workspace_matches_allocating_entry_point_twice(layout, b, sizes, dtype):
    import torch
    for i, n in enumerate(sizes):  # two calls in a row on the shared array
        # tl_permute_workspace_bytes covers the fixed-direction schedules this
        # entry point keeps to, so these sizes fit the static array
        assert T.workspace_bytes(layout, n, b or 16, np.dtype(dtype).itemsize) <= STATIC_BYTES
        keys = data.sorted_keys_np(n, 1, 3 if dtype == np.uint32 else 16, 100 + i, dtype)
        a = _dev(keys)
        ref = _dev(keys)
        assert _static(layout, a, b or 16) == T.SUCCESS
        T.permute(layout, ref, b or 16)
        torch.cuda.synchronize()
        assert torch.equal(a, ref), (layout, n)
        got = a.cpu().numpy().view(dtype)
        assert np.array_equal(got, O.permute(layout, keys, b or 16)), (layout, n)


def test_static_workspace_refuses_what_does_not_fit():
    import torch
    n = 100_000_000  # B-tree whose top tree holds 24.1M keys: ~190 MB of scratch
    assert T.workspace_bytes("btree", n, 16, 8) > STATIC_BYTES
    t = torch.empty(1, dtype=torch.int64, device="cuda")
    rc = _lib().tl_permute_static_ws(T.LAYOUT_BTREE, t.data_ptr(), n, 16, 8, None)
    assert rc == T.ERROR_UNSUPPORTED
