"""Python binding of libtreelayouts.so (the C ABI in include/tree_layouts.h).

The library is the product: hand-written sm_100a kernels behind a C ABI.  This
module is thin plumbing over it (ctypes + torch device tensors) used by the
tests and the benchmark.  There is no fallback: if the shared library is
missing, every call raises.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "libtreelayouts.so")

LAYOUT_BST, LAYOUT_BTREE, LAYOUT_MVEB, LAYOUT_VEB = 0, 1, 2, 3
# "veb": the standard van Emde Boas layout of the reference's CPU code
LAYOUTS = {"bst": LAYOUT_BST, "btree": LAYOUT_BTREE, "mveb": LAYOUT_MVEB, "veb": LAYOUT_VEB}

SUCCESS = 0
ERROR_INVALID_VALUE = 1
ERROR_CUDA = 2
ERROR_TIMEOUT = 3
ERROR_OUT_OF_MEMORY = 4
ERROR_WORKSPACE_TOO_SMALL = 5
ERROR_UNSUPPORTED = 6

VEB_DTYPE = np.dtype({"names": ["L", "R", "D"], "formats": [np.uint64, np.uint64, np.uint32],
                      "offsets": [0, 8, 16], "itemsize": 24})


class TreeLayoutError(RuntimeError):
    def __init__(self, status: int, what: str):
        self.status = status
        super().__init__(f"{what}: status {status} ({status_string(status)})")


def build() -> None:
    """Compile libtreelayouts.so for sm_100a in place (nvcc cross-compiles)."""
    subprocess.run(["make", "-s", "-C", PKG_DIR], check=True)


_lib = None
_v = C.c_void_p
_u64 = C.c_uint64
_u32 = C.c_uint32
_f32p = C.POINTER(C.c_float)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with tree_layouts.build() "
                               "(there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        L.tl_status_string.restype = C.c_char_p
        L.tl_permute.argtypes = [C.c_int, _v, _u64, _u64, _u32, _v, _u64, _v, _f32p]
        L.tl_permute_workspace_bytes.argtypes = [C.c_int, _u64, _u64, _u32, C.POINTER(_u64)]
        L.tl_layout_position.argtypes = [C.c_int, _u64, _u64, _u64, C.POINTER(_u64)]
        L.tl_debug_emulate_permute.argtypes = [C.c_int, _u64, _u64, _v, C.POINTER(_u64)]
        L.tl_debug_emulate_unpermute.argtypes = [C.c_int, _u64, _u64, _v]
        L.tl_unpermute.argtypes = [C.c_int, _v, _u64, _u64, _u32, _v, _u64, _v, _f32p]
        L.tl_permute_algorithm.argtypes = [C.c_int, C.c_int, _v, _u64, _u64, _u32, _v, _f32p]
        L.tl_unpermute_workspace_bytes.argtypes = [C.c_int, _u64, _u64, _u32, C.POINTER(_u64)]
        L.tl_debug_set_wait.argtypes = [C.c_uint, C.c_int]
        L.tl_build_table.argtypes = [_v, _u64, _u32, _u32]
        L.tl_build_table.restype = None
        for suf in ("", "_std"):
            getattr(L, f"tl_veb_tables_size{suf}").argtypes = [_u64, C.POINTER(_u32), C.POINTER(_u32),
                                                               C.POINTER(_u32)]
            getattr(L, f"tl_build_veb_tables{suf}").argtypes = [_u64, _v, _v, _v]
        for w in ("u32", "u64"):
            getattr(L, f"tl_query_bst_{w}").argtypes = [_v, _u64, _v, _u64, _v, _v, _f32p]
            getattr(L, f"tl_query_sorted_{w}").argtypes = [_v, _u64, _v, _u64, _v, _v, _f32p]
            getattr(L, f"tl_query_btree_{w}").argtypes = [_v, _u64, _u64, _v, _u64, _v, _v, _f32p]
            getattr(L, f"tl_query_veb_{w}").argtypes = [_v, _v, _u64, _u32, _v, _u64, _v, _v, _f32p]
            getattr(L, f"tl_query_veb_nonperfect_{w}").argtypes = [_v, _v, _v, _v, _u64, _u32, _u32, _v,
                                                                    _u64, _v, _v, _f32p]
        _lib = L
    return _lib


def status_string(status: int) -> str:
    try:
        return lib().tl_status_string(status).decode()
    except Exception:  # library not loadable
        return "?"


def _check(rc: int, what: str) -> None:
    if rc != SUCCESS:
        raise TreeLayoutError(rc, what)


def _stream_ptr(stream) -> int:
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    return getattr(stream, "cuda_stream", stream)


def _key_bytes(t) -> int:
    kb = t.element_size()
    if kb not in (4, 8):
        raise ValueError("keys must be 4 or 8 bytes wide")
    return kb


# ------------------------------------------------------------------ host-only
def layout_position(layout: str, n: int, rank: int, b: int = 16) -> int:
    out = _u64()
    _check(lib().tl_layout_position(LAYOUTS[layout], n, b, rank, C.byref(out)), "tl_layout_position")
    return out.value


def emulate_permute(layout: str, keys: np.ndarray, b: int = 16):
    """Host replay of the kernels' tile schedule; returns (layout array, violations)."""
    A = np.ascontiguousarray(keys, dtype=np.uint64).copy()
    viol = _u64()
    _check(lib().tl_debug_emulate_permute(LAYOUTS[layout], len(A), b, A.ctypes.data, C.byref(viol)),
           "tl_debug_emulate_permute")
    return A, viol.value


def emulate_algorithm(layout: str, algorithm: str, keys: np.ndarray, b: int = 16):
    """Host replay of tl_permute_algorithm's steps for "cycles" / "hybrid";
    returns (layout array, number of steps)."""
    L = lib()
    L.tl_debug_emulate_algorithm.argtypes = [C.c_int, C.c_int, _u64, _u64, _v, C.POINTER(_u64)]
    A = np.ascontiguousarray(keys, dtype=np.uint64).copy()
    steps = _u64()
    _check(L.tl_debug_emulate_algorithm(LAYOUTS[layout], ALGORITHMS[algorithm], len(A), b, A.ctypes.data,
                                        C.byref(steps)), "tl_debug_emulate_algorithm")
    return A, steps.value


def emulate_unpermute(layout: str, A: np.ndarray, b: int = 16) -> np.ndarray:
    """Host replay of the reverse permutation's gather; returns the sorted array."""
    out = np.ascontiguousarray(A, dtype=np.uint64).copy()
    _check(lib().tl_debug_emulate_unpermute(LAYOUTS[layout], len(out), b, out.ctypes.data),
           "tl_debug_emulate_unpermute")
    return out


def unpermute_workspace_bytes(layout: str, n: int, b: int = 16, key_bytes: int = 8) -> int:
    out = _u64()
    _check(lib().tl_unpermute_workspace_bytes(LAYOUTS[layout], n, b, key_bytes, C.byref(out)),
           "tl_unpermute_workspace_bytes")
    return out.value


def workspace_bytes(layout: str, n: int, b: int = 16, key_bytes: int = 8) -> int:
    out = _u64()
    _check(lib().tl_permute_workspace_bytes(LAYOUTS[layout], n, b, key_bytes, C.byref(out)),
           "tl_permute_workspace_bytes")
    return out.value


def build_table(n: int, d: int) -> np.ndarray:
    t = np.zeros(max(d, 1), dtype=VEB_DTYPE)
    lib().tl_build_table(t.ctypes.data, n, d, 0)
    return t


def veb_tables(n: int, standard: bool = False):
    """(tables, idx, table_idx, d): the table set of an mvEB layout of n keys
    (standard=True: of a standard vEB layout)."""
    suf = "_std" if standard else ""
    nt, ts, d = _u32(), _u32(), _u32()
    _check(getattr(lib(), f"tl_veb_tables_size{suf}")(n, C.byref(nt), C.byref(ts), C.byref(d)),
           "tl_veb_tables_size")
    tables = np.zeros(ts.value, dtype=VEB_DTYPE)
    idx = np.zeros(nt.value, dtype=np.uint64)
    tidx = np.zeros(nt.value, dtype=np.uint32)
    _check(getattr(lib(), f"tl_build_veb_tables{suf}")(n, tables.ctypes.data, idx.ctypes.data,
                                                        tidx.ctypes.data), "tl_build_veb_tables")
    return tables, idx, tidx, d.value


def set_wait(spin_limit: int = 0, force_timeout: bool = False) -> None:
    """Fault-injection hook: bound device waits / make them expire."""
    lib().tl_debug_set_wait(spin_limit, int(force_timeout))


# ------------------------------------------------------------------ device calls
def permute(layout: str, keys, b: int = 16, stream=None, workspace=None, timed: bool = False):
    """Permute a sorted CUDA tensor in place into `layout`.  Returns device ms
    when timed, else None."""
    ms = C.c_float(0.0)
    ws_ptr, ws_bytes = (0, 0) if workspace is None else (workspace.data_ptr(), workspace.numel()
                                                           * workspace.element_size())
    rc = lib().tl_permute(LAYOUTS[layout], keys.data_ptr(), keys.numel(), b, _key_bytes(keys),
                          ws_ptr or None, ws_bytes, _stream_ptr(stream), C.byref(ms) if timed else None)
    _check(rc, f"tl_permute({layout}, n={keys.numel()})")
    return ms.value if timed else None


ALGORITHMS = {"stream": 0, "involutions": 1, "cycles": 2, "hybrid": 3}


def permute_algorithm(layout: str, algorithm: str, keys, b: int = 16, stream=None, timed: bool = False):
    """tl_permute_algorithm: the layout by one of the reference's algorithm
    families ("involutions": BST, B-tree, mvEB; "cycles": the cycle-leader
    family, BST, B-tree, mvEB; "hybrid": the BST by cycles and involutions) or
    by this library's own ("stream")."""
    ms = C.c_float(0.0)
    rc = lib().tl_permute_algorithm(LAYOUTS[layout], ALGORITHMS[algorithm], keys.data_ptr(), keys.numel(), b,
                                    _key_bytes(keys), _stream_ptr(stream), C.byref(ms) if timed else None)
    _check(rc, f"tl_permute_algorithm({layout}, {algorithm}, n={keys.numel()})")
    return ms.value if timed else None


def unpermute(layout: str, keys, b: int = 16, stream=None, workspace=None, timed: bool = False):
    """Permute a CUDA tensor holding `layout` (as permute leaves it) back to
    sorted order in place.  Returns device ms when timed, else None."""
    ms = C.c_float(0.0)
    ws_ptr, ws_bytes = (0, 0) if workspace is None else (workspace.data_ptr(), workspace.numel()
                                                           * workspace.element_size())
    rc = lib().tl_unpermute(LAYOUTS[layout], keys.data_ptr(), keys.numel(), b, _key_bytes(keys),
                            ws_ptr or None, ws_bytes, _stream_ptr(stream), C.byref(ms) if timed else None)
    _check(rc, f"tl_unpermute({layout}, n={keys.numel()})")
    return ms.value if timed else None


class VebTablesDevice:
    """Device copies of the table set for an mvEB (or, standard=True, a standard
    vEB) layout of n keys."""

    def __init__(self, n: int, device="cuda", standard: bool = False):
        import torch
        tables, idx, tidx, d = veb_tables(n, standard)
        self.n, self.d, self.num_tables = n, d, len(idx)
        self.tables = torch.from_numpy(tables.view(np.uint8).copy()).to(device)
        self.idx = torch.from_numpy(idx.view(np.int64).copy()).to(device)
        self.table_idx = torch.from_numpy(tidx.view(np.int32).copy()).to(device)


def query(layout: str, tree, queries, answers, b: int = 16, tables: VebTablesDevice | None = None,
          stream=None, timed: bool = False):
    """answers[i] = position of queries[i] in the layout `tree`, or n.  Layout
    "sorted": binary search over the sorted (unpermuted) keys."""
    L = lib()
    w = "u64" if _key_bytes(tree) == 8 else "u32"
    assert queries.element_size() == tree.element_size()
    n, q = tree.numel(), queries.numel()
    ms = C.c_float(0.0)
    msp = C.byref(ms) if timed else None
    s = _stream_ptr(stream)
    if layout in ("bst", "sorted"):
        rc = getattr(L, f"tl_query_{layout}_{w}")(tree.data_ptr(), n, queries.data_ptr(), q, answers.data_ptr(), s,
                                                   msp)
    elif layout == "btree":
        rc = getattr(L, f"tl_query_btree_{w}")(tree.data_ptr(), n, b, queries.data_ptr(), q, answers.data_ptr(),
                                               s, msp)
    elif layout in ("mveb", "veb"):
        if tables is None:
            tables = VebTablesDevice(n, tree.device, standard=layout == "veb")
        if tables.num_tables == 1:
            rc = getattr(L, f"tl_query_veb_{w}")(tree.data_ptr(), tables.tables.data_ptr(), n, tables.d,
                                                 queries.data_ptr(), q, answers.data_ptr(), s, msp)
        else:
            rc = getattr(L, f"tl_query_veb_nonperfect_{w}")(
                tree.data_ptr(), tables.tables.data_ptr(), tables.idx.data_ptr(), tables.table_idx.data_ptr(),
                n, tables.d, tables.num_tables, queries.data_ptr(), q, answers.data_ptr(), s, msp)
    else:
        raise ValueError(layout)
    _check(rc, f"tl_query_{layout}_{w}")
    return ms.value if timed else None
