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


def _small_tiles(plan, tile_keys=256):
    plan.set_tuning(tile_keys=[tile_keys] * TB.NCLASS)


def _ordered_plan(off, b, tile_keys=256, key_bytes=8):
    """A plan whose instances of 64 tiles or more all take the ordered schedule
    (debug schedule mode 2 while the plan is built)."""
    import tree_layouts as T
    T.lib().tl_debug_set_schedule(2)
    try:
        plan = TB.BatchPlan(off, b=b, key_bytes=key_bytes)
        _small_tiles(plan, tile_keys)
    finally:
        T.lib().tl_debug_set_schedule(0)
    return plan


@pytest.mark.parametrize("b", [8, 16, 3, 1])
def test_batched_ordered_schedule_matches_oracle(b):
    # 256-key tiles: every instance of 2^14 keys or more has 64 tiles or more
    # and takes the ordered schedule; the rest keep the fixed directions
    keys, off, sizes = _batch(120, 4, 17, 40 + b, extra=[16384, 16383, 70001, 1 << 17])
    ref = _expected(keys.cpu().numpy().view(np.uint64), sizes, b)
    plan = _ordered_plan(off, b)
    n_ord, k_ord = plan.ordered()
    assert n_ord >= 4 and k_ord >= 16384 + 70001 + (1 << 17)
    assert n_ord < len(sizes)
    plan.permute(keys)
    assert np.array_equal(keys.cpu().numpy().view(np.uint64), ref)


def test_batched_ordered_schedule_u32_keys():
    import torch
    keys, off, sizes = _batch(60, 8, 17, 77, extra=[1 << 16])
    k32 = keys.to(torch.int32)
    assert int(keys.max()) < 2**31
    ref = _expected(k32.cpu().numpy().view(np.uint32), sizes, 8)
    plan = _ordered_plan(off, 8, key_bytes=4)
    assert plan.ordered()[0] >= 1
    plan.permute(k32)
    assert np.array_equal(k32.cpu().numpy().view(np.uint32), ref)


def test_batched_ordered_schedule_replays_from_a_cuda_graph():
    import torch
    keys, off, sizes = _batch(80, 6, 17, 21, extra=[1 << 17])
    pristine = keys.clone()
    ref = _expected(keys.cpu().numpy().view(np.uint64), sizes, 8)
    plan = _ordered_plan(off, 8, 512)
    assert plan.ordered()[0] >= 1
    ws = plan.workspace()
    s = torch.cuda.Stream()
    plan.permute(keys, ws, stream=s)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        plan.permute(keys, ws, stream=s, check=False)
    for _ in range(2):
        keys.copy_(pristine)
        g.replay()
        torch.cuda.synchronize()
        plan.status(ws)
        assert np.array_equal(keys.cpu().numpy().view(np.uint64), ref)
    del g


def test_batched_fixed_schedule_switch_keeps_results():
    import tree_layouts as T
    keys, off, sizes = _batch(60, 6, 17, 33, extra=[1 << 17])
    ref = _expected(keys.cpu().numpy().view(np.uint64), sizes, 8)
    T.lib().tl_debug_set_schedule(1)
    try:
        plan = TB.BatchPlan(off, b=8)
        _small_tiles(plan)
        assert plan.ordered() == (0, 0)
    finally:
        T.lib().tl_debug_set_schedule(0)
    plan.permute(keys)
    assert np.array_equal(keys.cpu().numpy().view(np.uint64), ref)


def test_batched_default_orders_only_where_it_pays():
    # by default an instance takes the ordered schedule only where that cuts its
    # scratch keys to 30 %; results are exact either way
    keys, off, sizes = _batch(60, 12, 17, 5, extra=[1 << 17, 1 << 16])
    ref = _expected(keys.cpu().numpy().view(np.uint64), sizes, 1)
    forced = _ordered_plan(off, 1)
    plan = TB.BatchPlan(off, b=1)
    _small_tiles(plan)
    assert plan.ordered()[0] <= forced.ordered()[0]
    plan.permute(keys)
    assert np.array_equal(keys.cpu().numpy().view(np.uint64), ref)
