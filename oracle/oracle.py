"""ctypes wrapper around the CPU oracle (liboracle.so) and the reference's own code
built from its sources (_ref/libref_cpu.so, _ref/libref_gpu.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by the smoke check and by the
benchmark's CPU-baseline leg, always as the checker or the timed baseline, never
as the product path.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")


class VebTable(C.Structure):
    """Same layout as the reference's vEB_table (gpu/src/query-mveb.cuh:27-31)."""
    _fields_ = [("L", C.c_uint64), ("R", C.c_uint64), ("D", C.c_uint32)]


VEB_DTYPE = np.dtype({"names": ["L", "R", "D"], "formats": [np.uint64, np.uint64, np.uint32],
                      "offsets": [0, 8, 16], "itemsize": 24})


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
        L = C.CDLL(path)
        L.orc_permute_btree.argtypes = [_u64p, C.c_uint64, C.c_uint64]
        L.orc_permute_bst.argtypes = [_u64p, C.c_uint64]
        L.orc_permute_mveb.argtypes = [_u64p, C.c_uint64]
        L.orc_permute_veb_std.argtypes = [_u64p, C.c_uint64]
        L.orc_build_table_std.argtypes = [C.c_void_p, C.c_uint64, C.c_uint32, C.c_uint32]
        L.orc_veb_tables_size_std.argtypes = [C.c_uint64, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
        L.orc_build_veb_tables_std.argtypes = [C.c_uint64, C.c_void_p, _u64p, _u32p]
        L.orc_search_bst.argtypes = [_u64p, C.c_uint64, _u64p, C.c_uint64, _u64p]
        L.orc_search_btree.argtypes = [_u64p, C.c_uint64, C.c_uint64, _u64p, C.c_uint64, _u64p]
        L.orc_build_table.argtypes = [C.c_void_p, C.c_uint64, C.c_uint32, C.c_uint32]
        L.orc_veb_tables_size.argtypes = [C.c_uint64, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
        L.orc_build_veb_tables.argtypes = [C.c_uint64, C.c_void_p, _u64p, _u32p]
        L.orc_search_veb.argtypes = [_u64p, C.c_void_p, C.c_uint64, C.c_uint32, _u64p,
                                     C.c_uint64, _u64p]
        L.orc_search_veb_nonperfect.argtypes = [_u64p, C.c_void_p, _u64p, _u32p, C.c_uint64,
                                                C.c_uint32, C.c_uint32, _u64p, C.c_uint64, _u64p]
        L.orc_time_permute_btree.argtypes = [_u64p, C.c_uint64, C.c_uint64]
        L.orc_time_permute_btree.restype = C.c_double
        _lib = L
    return _lib


# ---------------------------------------------------------------- permutations
def permutation(layout: str, n: int, b: int = 16) -> np.ndarray:
    """perm[p] = sorted rank stored at layout position p."""
    A = np.arange(n, dtype=np.uint64)
    if layout == "bst":
        lib().orc_permute_bst(A, n)
    elif layout == "btree":
        lib().orc_permute_btree(A, n, b)
    elif layout == "mveb":
        lib().orc_permute_mveb(A, n)
    elif layout == "veb":
        lib().orc_permute_veb_std(A, n)
    else:
        raise ValueError(layout)
    return A


def permute(layout: str, keys: np.ndarray, b: int = 16) -> np.ndarray:
    perm = permutation(layout, len(keys), b)
    return keys[perm.astype(np.int64)]


# ---------------------------------------------------------------- queries
def search(layout: str, A: np.ndarray, queries: np.ndarray, b: int = 16) -> np.ndarray:
    A64 = np.ascontiguousarray(A, dtype=np.uint64)
    q64 = np.ascontiguousarray(queries, dtype=np.uint64)
    ans = np.empty(len(q64), dtype=np.uint64)
    n = len(A64)
    if layout == "bst":
        lib().orc_search_bst(A64, n, q64, len(q64), ans)
    elif layout == "btree":
        lib().orc_search_btree(A64, n, b, q64, len(q64), ans)
    elif layout in ("mveb", "veb"):
        tables, idx, table_idx, d = veb_tables(n, standard=layout == "veb")
        if len(idx) == 1:
            lib().orc_search_veb(A64, tables.ctypes.data, n, d, q64, len(q64), ans)
        else:
            lib().orc_search_veb_nonperfect(A64, tables.ctypes.data, idx, table_idx, n, d,
                                            len(idx), q64, len(q64), ans)
    else:
        raise ValueError(layout)
    return ans


def search_sorted(keys: np.ndarray, queries: np.ndarray) -> np.ndarray:
    """Binary search over the sorted keys, as binarySearch in
    gpu/src/binary-search.cuh:27-46 does for hits (the index of the key); a miss
    answers n here (the reference returns its predecessor's index, and does not
    terminate for a query below keys[0])."""
    keys = np.ascontiguousarray(keys)
    queries = np.ascontiguousarray(queries, dtype=keys.dtype)
    n = len(keys)
    lb = np.searchsorted(keys, queries, side="left")
    hit = lb < n
    hit[hit] = keys[lb[hit]] == queries[hit]
    return np.where(hit, lb, n).astype(np.uint64)


def build_table(n: int, d: int, standard: bool = False) -> np.ndarray:
    t = np.zeros(max(d, 1), dtype=VEB_DTYPE)
    (lib().orc_build_table_std if standard else lib().orc_build_table)(t.ctypes.data, n, d, 0)
    return t


def veb_tables(n: int, standard: bool = False):
    """(tables, idx, table_idx, d) exactly as the reference's query drivers build
    them: gpu/test/query-mveb-fixedN.cu:43-165 (mvEB), cpu/test/query-veb-fixedN.cpp:
    37-150 (standard vEB); one table for perfect n."""
    suf = "_std" if standard else ""
    nt = C.c_uint32()
    ts = C.c_uint32()
    getattr(lib(), f"orc_veb_tables_size{suf}")(n, C.byref(nt), C.byref(ts))
    tables = np.zeros(ts.value, dtype=VEB_DTYPE)
    idx = np.zeros(nt.value, dtype=np.uint64)
    table_idx = np.zeros(nt.value, dtype=np.uint32)
    getattr(lib(), f"orc_build_veb_tables{suf}")(n, tables.ctypes.data, idx, table_idx)
    return tables, idx, table_idx, int(n).bit_length()


# ---------------------------------------------------------------- reference builds
_ref_cpu = None


def ref_cpu():
    """The reference's own CPU code, compiled from its sources (None if absent)."""
    global _ref_cpu
    if _ref_cpu is None:
        path = os.path.join(HERE, "_ref", "libref_cpu.so")
        if not os.path.exists(path):
            return None
        L = C.CDLL(path)
        L.ref_cpu_permute_btree_u64.argtypes = [_u64p, C.c_uint64, C.c_uint64, C.c_uint32]
        L.ref_cpu_permute_btree_u64.restype = C.c_double
        L.ref_cpu_permute_bst_u64.argtypes = [_u64p, C.c_uint64, C.c_uint32]
        L.ref_cpu_permute_bst_u64.restype = C.c_double
        L.ref_cpu_search_btree_u64.argtypes = [_u64p, C.c_uint64, C.c_uint64, _u64p, _u64p,
                                               C.c_uint64, C.c_uint32]
        L.ref_cpu_search_bst_u64.argtypes = [_u64p, C.c_uint64, _u64p, _u64p, C.c_uint64,
                                             C.c_uint32]
        L.ref_cpu_permute_veb_u64.argtypes = [_u64p, C.c_uint64, C.c_uint32]
        L.ref_cpu_permute_veb_u64.restype = C.c_double
        L.ref_cpu_build_table.argtypes = [C.c_void_p, C.c_uint64, C.c_uint32, C.c_uint32]
        L.ref_cpu_search_veb_u64.argtypes = [_u64p, C.c_void_p, C.c_uint64, C.c_uint32, _u64p, _u64p,
                                             C.c_uint64, C.c_uint32]
        L.ref_cpu_search_veb_nonperfect_u64.argtypes = [_u64p, C.c_void_p, _u32p, _u64p, C.c_uint32,
                                                        C.c_uint32, _u64p, _u64p, C.c_uint64, C.c_uint32]
        _ref_cpu = L
    return _ref_cpu


def ref_gpu_path() -> str:
    return os.path.join(HERE, "_ref", "libref_gpu.so")
