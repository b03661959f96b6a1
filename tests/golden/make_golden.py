"""Generates the golden fixtures that pin the oracle to the reference itself.

  python tests/golden/make_golden.py cpu   -> tests/golden/golden_cpu.json
      B-tree / BST layouts and query answers from the reference's own CPU code
      (cpu/src/btree-cycles.h, cpu/src/bst-involutions.h, cpu/src/query-*.h) and
      mvEB position tables from the reference's buildTable
      (gpu/src/query-mveb.cu, host code); standard vEB layouts, tables and
      hit-only query answers from cpu/src/veb-cycles.h, cpu/src/query-veb.cpp
      and cpu/src/query-veb.h; all compiled from the reference sources by
      oracle/Makefile into oracle/_ref/.
  python tests/golden/make_golden.py gpu OUT.json
      mvEB layouts from the reference's own GPU permutation
      (gpu/src/mveb-cycles.cuh, timePermutevEB) run on a B200; needs
      oracle/_ref/libref_gpu.so and a GPU.  The output is committed as
      tests/golden/golden_mveb_gpu.json.

Layouts are stored as SHA-256 digests of the permuted identity (uint64 little
endian) plus a few small explicit arrays; answers likewise.
"""
from __future__ import annotations

import ctypes as C
import hashlib
import json
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tree-layouts_b200"))

import oracle as O  # noqa: E402
from tree_layouts import data  # noqa: E402

BTREE_BS = [1, 2, 3, 4, 8, 16, 17, 32]
MVEB_SIZES = (list(range(1, 300)) + [511, 1023, 4095, 4096, 4097, 8191, 65535, 65536, 65537, 100000, 131071,
                                      262143, 300001, 1048575, 1048576, 2097151, 3000017, 4194303])


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.uint64).tobytes()).hexdigest()[:24]


def ref_level_count_ok(n: int, b: int) -> bool:
    """False where the reference's double-precision level count
    (log10(n)/log10(b+1), gpu/src/btree-cycles.cuh:81) is off by one; the
    reference's own arithmetic underflows at those n and it crashes."""
    hf = int(math.log10(n) / math.log10(b + 1))
    h, p = 0, 1
    while p * (b + 1) <= n:
        p *= b + 1
        h += 1
    return hf == h


def btree_sizes(b: int):
    base = list(range(b + 1, b + 400)) + [1000, 4095, 4096, 4097, 8191, 8192, 9001, 65535, 65536, 100003,
                                          (b + 1) ** 3 - 1, (b + 1) ** 3, (b + 1) ** 3 + 1, 300007, 1000000]
    return [n for n in sorted(set(base)) if n > b and ref_level_count_ok(n, b)]


def make_cpu(out_path: str) -> None:
    ref = O.ref_cpu()
    assert ref is not None, "build oracle/_ref/libref_cpu.so first (make -C oracle)"
    out = {"source": "reference cpu/src compiled by oracle/Makefile", "btree": [], "bst": [],
           "query_btree": [], "query_bst": [], "tables": [], "examples": [],
           "veb_std": [], "veb_std_tables": [], "query_veb_std": []}
    for b in BTREE_BS:
        for n in btree_sizes(b):
            A = np.arange(n, dtype=np.uint64)
            ref.ref_cpu_permute_btree_u64(A, n, b, 1)
            out["btree"].append({"b": b, "n": n, "sha": sha(A)})
    for n in list(range(1, 600)) + [4095, 4096, 65535, 65536, 1048575, 1048576, 1000003]:
        A = np.arange(n, dtype=np.uint64)
        ref.ref_cpu_permute_bst_u64(A, n, 1)
        out["bst"].append({"n": n, "sha": sha(A)})
    for (b, n) in [(3, 20), (16, 40), (1, 12)]:
        A = np.arange(n, dtype=np.uint64)
        if b == 1:
            ref.ref_cpu_permute_bst_u64(A, n, 1)
        else:
            ref.ref_cpu_permute_btree_u64(A, n, b, 1)
        out["examples"].append({"layout": "bst" if b == 1 else "btree", "b": b, "n": n, "perm": A.tolist()})
    # queries: seeded keys (gaps in [1,16]) and a 50/50 hit/miss mix
    for (b, n, q, seed) in [(16, 100000, 20000, 3), (16, 83520, 5000, 5), (8, 50000, 5000, 7), (3, 12345, 5000, 9),
                            (32, 70000, 5000, 11)]:
        keys = data.sorted_keys_np(n, 1, 16, seed)
        Q = data.queries_np(keys, q, 0.5, seed + 1)
        A = keys.copy()
        ref.ref_cpu_permute_btree_u64(A, n, b, 1)
        padded = np.concatenate([A, np.full(b, np.iinfo(np.uint64).max, dtype=np.uint64)])
        ans = np.empty(q, dtype=np.uint64)
        ref.ref_cpu_search_btree_u64(padded, n, b, Q, ans, q, 1)
        out["query_btree"].append({"b": b, "n": n, "q": q, "seed": seed, "sha": sha(ans),
                                   "hits": int((ans != n).sum())})
    for (n, q, seed) in [(2**20 - 1, 20000, 1), (100000, 5000, 2), (777, 3000, 4)]:
        keys = data.sorted_keys_np(n, 1, 16, seed)
        Q = data.queries_np(keys, q, 0.5, seed + 1)
        A = keys.copy()
        ref.ref_cpu_permute_bst_u64(A, n, 1)
        ans = np.empty(q, dtype=np.uint64)
        ref.ref_cpu_search_bst_u64(A, n, Q, ans, q, 1)
        out["query_bst"].append({"n": n, "q": q, "seed": seed, "sha": sha(ans), "hits": int((ans != n).sum())})
    gpu = C.CDLL(O.ref_gpu_path())
    gpu.ref_gpu_build_table.argtypes = [C.c_void_p, C.c_uint64, C.c_uint32, C.c_uint32]
    for n in [3, 7, 15, 31, 63, 127, 255, 511, 1023, 2**16 - 1, 2**20 - 1, 2**24 - 1, 2**29 - 1, 2**30 - 1,
              2**31 - 1, 2**33 - 1]:
        d = n.bit_length()
        t = np.zeros(d, dtype=O.VEB_DTYPE)
        gpu.ref_gpu_build_table(t.ctypes.data, n, d, 0)
        out["tables"].append({"n": n, "d": d, "L": t["L"].tolist(), "R": t["R"].tolist(), "D": t["D"].tolist()})
    # standard vEB (the reference's CPU layout): layouts, tables, hit-only answers
    for n in MVEB_SIZES:
        A = np.arange(n, dtype=np.uint64)
        ref.ref_cpu_permute_veb_u64(A, n, 1)
        out["veb_std"].append({"n": n, "sha": sha(A)})
    for n in [3, 7, 15, 31, 63, 127, 255, 511, 1023, 2**16 - 1, 2**17 - 1, 2**20 - 1, 2**29 - 1, 2**30 - 1,
              2**31 - 1, 2**33 - 1]:
        d = n.bit_length()
        t = np.zeros(d, dtype=O.VEB_DTYPE)
        ref.ref_cpu_build_table(t.ctypes.data, n, d, 0)
        out["veb_std_tables"].append({"n": n, "d": d, "L": t["L"].tolist(), "R": t["R"].tolist(),
                                      "D": t["D"].tolist()})
    for (n, q, seed) in [(2**20 - 1, 20000, 21), (100000, 5000, 22), (777, 3000, 23), (3000017, 20000, 24),
                         (65536, 5000, 25)]:
        keys = data.sorted_keys_np(n, 1, 16, seed)
        Q = data.queries_np(keys, q, 1.0, seed + 1)  # hits only (see ref_cpu_search_veb_u64)
        A = keys.copy()
        ref.ref_cpu_permute_veb_u64(A, n, 1)
        tables, idx, table_idx, d = O.veb_tables(n, standard=True)
        ans = np.empty(q, dtype=np.uint64)
        if len(idx) == 1:
            ref.ref_cpu_search_veb_u64(A, tables.ctypes.data, n, d, Q, ans, q, 1)
        else:
            ref.ref_cpu_search_veb_nonperfect_u64(A, tables.ctypes.data, table_idx, idx, len(idx), d, Q, ans, q, 1)
        out["query_veb_std"].append({"n": n, "q": q, "seed": seed, "sha": sha(ans), "hits": int((ans != n).sum())})
    with open(out_path, "w") as f:
        json.dump(out, f, separators=(",", ":"))


def make_gpu(out_path: str) -> None:
    gpu = C.CDLL(O.ref_gpu_path())
    gpu.ref_gpu_permute_mveb_u64.argtypes = [np.ctypeslib.ndpointer(np.uint64, flags="C"), C.c_uint64]
    gpu.ref_gpu_permute_mveb_u32.argtypes = [np.ctypeslib.ndpointer(np.uint32, flags="C"), C.c_uint64]
    out = {"source": "reference gpu/src/mveb-cycles.cuh timePermutevEB on a B200", "mveb": [], "mveb_u32": [],
           "examples": []}
    for n in MVEB_SIZES:
        A = np.arange(n, dtype=np.uint64)
        rc = gpu.ref_gpu_permute_mveb_u64(A, n)
        out["mveb"].append({"n": n, "sha": sha(A), "rc": rc})
    for n in [1000, 65537, 1048575, 3000017]:
        A = np.arange(n, dtype=np.uint32)
        rc = gpu.ref_gpu_permute_mveb_u32(A, n)
        out["mveb_u32"].append({"n": n, "sha": sha(A.astype(np.uint64)), "rc": rc})
    for n in [15, 20, 100]:
        A = np.arange(n, dtype=np.uint64)
        gpu.ref_gpu_permute_mveb_u64(A, n)
        out["examples"].append({"n": n, "perm": A.tolist()})
    with open(out_path, "w") as f:
        json.dump(out, f, separators=(",", ":"))


if __name__ == "__main__":
    which = sys.argv[1] if len(sys.argv) > 1 else "cpu"
    if which == "cpu":
        make_cpu(os.path.join(HERE, "golden_cpu.json"))
    else:
        make_gpu(sys.argv[2] if len(sys.argv) > 2 else os.path.join(HERE, "golden_mveb_gpu.json"))
