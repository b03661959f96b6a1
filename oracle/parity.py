"""Full-size parity checkers: the expected layout and the expected query answers
for a host copy of a workload, taken from the reference's own CPU code where
the reference has CPU code for the path (compiled from its sources into
_ref/libref_cpu.so by this directory's Makefile) and from the oracle's C
restatement otherwise.

TEST INFRASTRUCTURE ONLY: used by tests/ and by the benchmark's parity check,
outside any timed region, always as the checker.

Which checker serves which path:
  B-tree layout   timePermuteBtree, cpu/src/btree-cycles.h:71-96 (OpenMP)
  BST layout      timePermuteBST, cpu/src/bst-involutions.h:119-144 (OpenMP)
  standard vEB    timePermutevEB, cpu/src/veb-cycles.h:380-395 (OpenMP)
  mvEB layout     the oracle's restatement of gpu/src/mveb-cycles.cuh:233-440
                  (the reference has no CPU mvEB; the restatement is pinned to
                  the reference's GPU code by tests/golden/golden_mveb_gpu.json)
  B-tree queries  searchAll, cpu/src/query-btree.h:58-64, on the layout padded
                  with b words of all-ones (its node scan reads past n)
  BST queries     searchAll, cpu/src/query-bst.h:45-51
  vEB queries     the oracle's searchvEB[_nonperfect] restatement
                  (cpu/src/query-veb.h:43-64 / :128-170) over the reference's
                  table builders: the reference's own CPU search writes past
                  its pos array on a miss, so it only serves hit-only batches.
Without _ref/libref_cpu.so every path falls back to the oracle.
"""
from __future__ import annotations

import math
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np

import oracle as O

THREADS = os.cpu_count() or 1


def ref_level_count_ok(n: int, b: int) -> bool:
    """False where the reference's double-precision level count
    (log10(n)/log10(b+1), cpu/src/btree-cycles.h:74) is off by one; its own
    arithmetic underflows at those n and it crashes, so the oracle checks them."""
    if n <= b:
        return False  # cpu/src/btree-cycles.h:54-59 recurses without end for n < b
    hf = int(math.log10(n) / math.log10(b + 1))
    h, p = 0, 1
    while p * (b + 1) <= n:
        p *= b + 1
        h += 1
    return hf == h


def _widen(a: np.ndarray) -> np.ndarray:
    return a if a.dtype == np.uint64 else a.astype(np.uint64)


def layout_inplace(layout: str, A: np.ndarray, b: int = 16, threads: int = THREADS) -> str:
    """Permute the sorted host array A (uint64 or uint32) into `layout` in place
    with the checker for that layout; returns the checker's name."""
    n = len(A)
    if n <= 1:
        return "trivial"
    ref = O.ref_cpu()
    if layout == "btree" and ref is not None and ref_level_count_ok(n, b):
        if A.dtype == np.uint64:
            ref.ref_cpu_permute_btree_u64(A, n, b, threads)
        else:
            w = _widen(A)
            ref.ref_cpu_permute_btree_u64(w, n, b, threads)
            A[:] = w
        return "reference timePermuteBtree (cpu/src/btree-cycles.h)"
    if layout == "bst" and ref is not None:
        w = _widen(A)
        ref.ref_cpu_permute_bst_u64(w, n, threads)
        if w is not A:
            A[:] = w
        return "reference timePermuteBST (cpu/src/bst-involutions.h)"
    if layout == "veb" and ref is not None:
        w = _widen(A)
        ref.ref_cpu_permute_veb_u64(w, n, threads)
        if w is not A:
            A[:] = w
        return "reference timePermutevEB (cpu/src/veb-cycles.h)"
    w = _widen(A)
    if layout == "btree":
        O.lib().orc_permute_btree(w, n, b)
    elif layout == "bst":
        O.lib().orc_permute_bst(w, n)
    elif layout == "mveb":
        O.lib().orc_permute_mveb(w, n)
    elif layout == "veb":
        O.lib().orc_permute_veb_std(w, n)
    else:
        raise ValueError(layout)
    if w is not A:
        A[:] = w
    return f"oracle restatement ({layout})"


def batched_layout_inplace(A: np.ndarray, offsets: np.ndarray, b: int, threads: int = THREADS) -> str:
    """Every instance A[offsets[j]:offsets[j+1]] permuted into a B-tree layout
    in place, one instance per host thread (the reference's single-threaded
    path, p = 1, for each)."""
    def one(j):
        s, e = int(offsets[j]), int(offsets[j + 1])
        if e - s > 1:
            view = A[s:e]
            layout_inplace("btree", view, b, 1)
    with ThreadPoolExecutor(threads) as ex:
        list(ex.map(one, range(len(offsets) - 1)))
    return "reference timePermuteBtree (cpu/src/btree-cycles.h), p = 1 per instance"


def padded(n: int, b: int, dtype=np.uint64):
    """(buffer, view): a host array of n keys followed by b all-ones words, the
    padding the reference's B-tree search needs past the last node."""
    buf = np.empty(n + max(b, 1), dtype=dtype)
    buf[n:] = np.iinfo(dtype).max
    return buf, buf[:n]


def answers(layout: str, tree: np.ndarray, queries: np.ndarray, b: int = 16, threads: int = THREADS,
            tree_padded: bool = False) -> tuple[np.ndarray, str]:
    """Expected answers (uint64: the key's layout position, or n) of `queries`
    over the host layout `tree`.  For the B-tree, tree_padded=True says that b
    all-ones words follow tree in memory (see padded())."""
    n = len(tree)
    q = np.ascontiguousarray(queries, dtype=np.uint64)
    ans = np.empty(len(q), dtype=np.uint64)
    ref = O.ref_cpu()
    if layout == "btree" and ref is not None and tree.dtype == np.uint64:
        t = tree
        if not tree_padded:
            buf, t = padded(n, b)
            t[:] = tree
        ref.ref_cpu_search_btree_u64(t, n, b, q, ans, len(q), threads)
        return ans, "reference searchAll (cpu/src/query-btree.h)"
    if layout == "bst" and ref is not None:
        ref.ref_cpu_search_bst_u64(_widen(tree), n, q, ans, len(q), threads)
        return ans, "reference searchAll (cpu/src/query-bst.h)"
    return O.search(layout, _widen(tree), q, b), f"oracle search ({layout})"


# ---------------------------------------------------------------- device <-> host
def host_u64(t, out=None) -> np.ndarray:
    """Host uint64 copy of a device key tensor (4-byte keys widened unsigned)."""
    import torch
    src = t if t.element_size() == 8 else t.to(torch.int64) & 0xFFFFFFFF
    if out is None:
        out = np.empty(t.numel(), dtype=np.uint64)
    torch.from_numpy(out.view(np.int64)).copy_(src)
    return out


def equal_on_device(t, host: np.ndarray) -> bool:
    """The device key tensor t equals the host uint64 array word for word (t
    widened unsigned if 4-byte)."""
    import torch
    exp = torch.from_numpy(host.view(np.int64)).to(t.device)
    got = t if t.element_size() == 8 else t.to(torch.int64) & 0xFFFFFFFF
    return bool(torch.equal(got, exp))


def check_layout(layout: str, b: int, sorted_dev, layout_dev, keep_host: bool = False):
    """Bit-exact check of a device layout against the checker's layout of the
    same sorted keys.  Returns (report, host layout or None)."""
    import time
    t0 = time.time()
    n = sorted_dev.numel()
    if layout == "btree":
        _, host = padded(n, b)
    else:
        host = np.empty(n, dtype=np.uint64)
    host_u64(sorted_dev, host)
    checker = layout_inplace(layout, host, b)
    ok = equal_on_device(layout_dev, host)
    rep = {"bit_exact": ok, "keys": n, "checker": checker, "check_s": round(time.time() - t0, 1)}
    return rep, (host if keep_host else None)


def check_answers(layout: str, b: int, host_layout: np.ndarray, Q, ans, k: int, seed: int) -> dict:
    """A seeded sample of k device answers against the checker's answers over
    the host layout (as check_layout leaves it: padded for the B-tree)."""
    import torch
    rng = np.random.default_rng(seed)
    idx = np.sort(rng.choice(Q.numel(), size=min(k, Q.numel()), replace=False))
    it = torch.from_numpy(idx).to(Q.device)
    q = host_u64(Q[it])
    got = ans[it].cpu().numpy().view(np.uint64)
    exp, checker = answers(layout, host_layout, q, b, tree_padded=layout == "btree")
    bad = int((got != exp).sum())
    return {"exact": bad == 0, "sampled": len(idx), "mismatches": bad, "checker": checker}


def check_batched(b: int, sizes, sorted_dev, layout_dev, off_dev, Q=None, inst=None, ans=None) -> dict:
    """Every instance of a batched layout against the checker, and (with
    queries) every answer: a hit names the key's own position, a miss answers
    n_j for a key absent from instance j."""
    import time

    import torch
    t0 = time.time()
    offs = off_dev.cpu().numpy()
    host = host_u64(sorted_dev)
    checker = batched_layout_inplace(host, offs, b)
    ok = equal_on_device(layout_dev, host)
    del host
    rep = {"bit_exact": ok, "instances": len(sizes), "keys": int(offs[-1]), "checker": checker}
    if Q is not None:
        inst64 = inst.to(torch.int64)
        lo, nj = off_dev[inst64], off_dev[inst64 + 1] - off_dev[inst64]
        hit = ans < nj
        good = bool((ans[~hit] == nj[~hit]).all()) and bool((layout_dev[(lo + ans)[hit]] == Q[hit]).all())
        # (instance, key) pairs sort globally: keys restart per instance below 2^32
        comp = torch.repeat_interleave(torch.arange(len(sizes), device=Q.device),
                                       torch.from_numpy(np.asarray(sizes)).to(Q.device))
        comp <<= 32
        comp |= sorted_dev
        qc = (inst64 << 32) | Q
        pos = torch.searchsorted(comp, qc).clamp_max(comp.numel() - 1)
        good = good and bool(((comp[pos] == qc) == hit).all())
        rep["answers_exact"] = good
        rep["answers_checked"] = int(Q.numel())
    rep["check_s"] = round(time.time() - t0, 1)
    return rep
