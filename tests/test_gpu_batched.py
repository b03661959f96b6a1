"""Batched mode: every instance's layout bit-exact to the oracle's, one
persistent launch replayed from a CUDA graph, batched queries exact against
the oracle, and the autotuner keeps results exact."""
import numpy as np
import pytest

import oracle as O
import tree_layouts.batched as TB
from tree_layouts import data

pytestmark = pytest.mark.gpu


def _batch(num, lo, hi, seed, extra=()):
    sizes = np.concatenate([TB.batch_sizes_np(num, lo, hi, seed), np.asarray(extra, dtype=np.int64)])
    keys, off = data.batch_keys_torch(sizes, 64, seed)
    return keys, off, sizes


def _expected(keys_np, sizes, b):
    out = keys_np.copy()
    o = 0
    for n in sizes:
        if n:
            out[o:o + n] = O.permute("btree", keys_np[o:o + n], b)
        o += n
    return out


@pytest.mark.parametrize("b", [8, 16, 3, 1])
def test_batched_layouts_match_oracle(b):
    keys, off, sizes = _batch(300, 4, 15, b, extra=[0, 1, 2, b, b + 1, 5000, 70001])
    ref = _expected(keys.cpu().numpy().view(np.uint64), sizes, b)
    plan = TB.BatchPlan(off, b=b)
    plan.permute(keys)
    assert np.array_equal(keys.cpu().numpy().view(np.uint64), ref)


def test_batched_permute_replays_from_a_cuda_graph():
    import torch
    keys, off, sizes = _batch(200, 6, 14, 5)
    pristine = keys.clone()
    ref = _expected(keys.cpu().numpy().view(np.uint64), sizes, 8)
    plan = TB.BatchPlan(off, b=8)
    ws = plan.workspace()
    s = torch.cuda.Stream()
    plan.permute(keys, ws, stream=s)  # warm-up outside the capture
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        plan.permute(keys, ws, stream=s, check=False)
    for _ in range(3):
        keys.copy_(pristine)
        g.replay()
        torch.cuda.synchronize()
        plan.status(ws)
        assert np.array_equal(keys.cpu().numpy().view(np.uint64), ref)
    del g


def test_batched_queries_match_oracle():
    import torch
    keys, off, sizes = _batch(150, 5, 14, 9, extra=[1, 3, 9])
    plan = TB.BatchPlan(off, b=8)
    sorted_np = keys.cpu().numpy().view(np.uint64).copy()
    Q, inst = data.batch_queries_torch(keys, off, 200_000, 0.7, 11)
    plan.permute(keys)
    ans = torch.empty(Q.numel(), dtype=torch.int64, device="cuda")
    plan.query(keys, Q, inst, ans)
    lay = keys.cpu().numpy().view(np.uint64)
    offs = off.cpu().numpy()
    qn, ins, got = Q.cpu().numpy().view(np.uint64), inst.cpu().numpy(), ans.cpu().numpy().view(np.uint64)
    for j in range(len(sizes)):
        sel = ins == j
        if not sel.any():
            continue
        exp = O.search("btree", lay[offs[j]:offs[j + 1]], qn[sel], 8)
        assert np.array_equal(got[sel], exp), j
    assert (got[ins < len(sizes)] <= sizes.max()).all()


def test_autotune_keeps_results_exact():
    import torch
    keys, off, sizes = _batch(400, 8, 16, 13)
    ref = _expected(keys.cpu().numpy().view(np.uint64), sizes, 8)
    Q, inst = data.batch_queries_torch(keys, off, 100_000, 0.7, 3)
    plan = TB.BatchPlan(off, b=8)
    report = plan.autotune(keys, Q, inst)
    assert "classes" in report and report["permute_ms"] > 0
    assert np.array_equal(keys.cpu().numpy(), np.asarray(data.batch_keys_torch(sizes, 64, 13)[0].cpu().numpy()))
    plan.permute(keys)
    assert np.array_equal(keys.cpu().numpy().view(np.uint64), ref)
    t = plan.tuning()
    assert t["threads"] in (256, 512)
