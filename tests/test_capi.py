"""The C ABI library on the host: it loads, exports every declared symbol, its
host-side geometry and tables equal the oracle's, and the replay of the
kernels' tile schedule reproduces the oracle's layouts with no protocol
violation (no stale read, every store covered by a read-flag wait, waits only
on earlier tickets, every position and scratch slot written exactly once)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import oracle as O
import tree_layouts as T

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    syms = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", h)).read()
            syms |= set(re.findall(r"^\s*(?:int|void|const char \*)\s*(tl_\w+)\(", txt, re.M))
    return sorted(syms)


def test_library_exports_every_declared_symbol():
    lib = T.lib()
    syms = declared_symbols()
    assert len(syms) >= 20
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    assert lib.tl_version() == 1


SIZES = list(range(1, 130)) + [255, 256, 4095, 4096, 4097, 8191, 8193, 65535, 65536, 65537, 83520, 83521,
                               131071, 250001, 1048575, 1048576]


@pytest.mark.parametrize("layout,b", [("bst", 1), ("btree", 2), ("btree", 3), ("btree", 8), ("btree", 16),
                                      ("btree", 31), ("mveb", 0), ("veb", 0)])
def test_tile_schedule_replay_matches_oracle(layout, b):
    for n in SIZES:
        keys = np.arange(n, dtype=np.uint64) * 5 + 11
        got, viol = T.emulate_permute(layout, keys, b or 16)
        assert viol == 0, (layout, b, n, viol)
        exp = O.permute(layout, keys, b or 16)
        assert np.array_equal(got, exp), (layout, b, n)


def test_both_btree_schedules_are_exercised():
    lib = T.lib()
    lib.tl_debug_btree_plan.argtypes = [C.c_uint64, C.c_uint64]
    plans = {lib.tl_debug_btree_plan(n, b) for n in SIZES for b in (2, 3, 8, 16, 31) if n > b}
    assert plans == {0, 1}
    assert lib.tl_debug_btree_plan(500_000_000, 16) == 1  # top tree holds 82% of the keys
    assert lib.tl_debug_btree_plan(2**30, 16) == 0


@pytest.mark.parametrize("layout,b", [("bst", 1), ("btree", 16), ("btree", 5), ("mveb", 0)])
def test_layout_position_matches_oracle(layout, b):
    for n in [1, 2, 3, 16, 17, 100, 4097, 65537, 300001]:
        perm = O.permutation(layout, n, b or 16)
        for p in range(0, n, max(1, n // 97)):
            assert T.layout_position(layout, n, int(perm[p]), b or 16) == p


@pytest.mark.parametrize("n", [1, 2, 3, 6, 7, 100, 1000, 4096, 65535, 70000, 300000000, 2**30 - 1, 2**30 + 5])
def test_veb_tables_match_oracle(n):
    t1, i1, x1, d1 = T.veb_tables(n)
    t2, i2, x2, d2 = O.veb_tables(n)
    assert d1 == d2
    assert t1.tobytes() == t2.tobytes() and np.array_equal(i1, i2) and np.array_equal(x1, x2)
    single = T.build_table(n, n.bit_length())
    assert single.tobytes() == O.build_table(n, n.bit_length()).tobytes()


def test_invalid_arguments_rejected_before_any_device_work():
    lib = T.lib()
    ms = C.c_float()
    assert lib.tl_permute(1, None, 100, 16, 8, None, 0, None, None) == T.ERROR_INVALID_VALUE  # null data
    assert lib.tl_permute(1, C.c_void_p(16), 100, 0, 8, None, 0, None, None) == T.ERROR_INVALID_VALUE  # b = 0
    assert lib.tl_permute(0, C.c_void_p(16), 100, 1, 2, None, 0, None, None) == T.ERROR_INVALID_VALUE  # width
    assert lib.tl_permute(7, C.c_void_p(16), 100, 1, 8, None, 0, None, None) == T.ERROR_INVALID_VALUE  # layout
    assert lib.tl_permute(1, C.c_void_p(16), 10**6, 16, 8, C.c_void_p(256), 64, None, C.byref(ms)) == \
        T.ERROR_WORKSPACE_TOO_SMALL
    out = C.c_uint64()
    assert lib.tl_layout_position(1, 10, 16, 10, C.byref(out)) == T.ERROR_INVALID_VALUE
    assert lib.tl_veb_tables_size(0, C.byref(C.c_uint32()), C.byref(C.c_uint32()), None) == T.ERROR_INVALID_VALUE
    assert T.status_string(T.ERROR_TIMEOUT) == "bounded device wait expired"


def test_workspace_is_small_relative_to_input():
    n = 5 * 10**8
    # B-tree: scratch holds the top tree (n/(b+1) keys for perfect trees)
    assert T.workspace_bytes("btree", 17**7 * 17 - 1, 16, 8) < 8 * (17**8) // 16
    # mvEB: about one key in 256 goes through scratch
    assert T.workspace_bytes("mveb", 2**30 - 1, 0, 4) < 4 * 2**30 // 100
    assert T.workspace_bytes("btree", n, 16, 8) > 0


@pytest.mark.parametrize("layout,n,b", [("bst", 2**23 - 1, 1), ("btree", 29_000_000, 16), ("btree", 6_000_000, 8)])
def test_ordered_schedule_replay_at_scale(layout, n, b):
    """The ordered-tile schedule over thousands of tiles (the headline's shape at
    1/17 of its size): chains, scratch tiles and the fix pass replayed with the
    protocol checks, against the oracle."""
    lib = T.lib()
    lib.tl_debug_permute_plan.argtypes = [C.c_int, C.c_uint64, C.c_uint64, C.c_uint32]
    # the replay takes the ordered schedule at any size; tl_permute from 64
    # tiles (B-tree) or 16384 tiles (BST) up
    assert lib.tl_debug_permute_plan(T.LAYOUTS[layout], n if b > 1 else 2**27 - 1, b, 8) == 2
    if b == 1:
        assert lib.tl_debug_permute_plan(T.LAYOUTS[layout], n, b, 8) in (0, 1)
    keys = np.arange(n, dtype=np.uint64) * 3 + 7
    got, viol = T.emulate_permute(layout, keys, b)
    assert viol == 0
    assert np.array_equal(got, O.permute(layout, keys, b))


@pytest.mark.parametrize("layout,b", [("bst", 1), ("btree", 2), ("btree", 3), ("btree", 8), ("btree", 16),
                                      ("btree", 31), ("mveb", 0), ("veb", 0)])
def test_unpermute_replay_matches_oracle(layout, b):
    """The reverse permutation's gather, replayed on the host with the kernels'
    per-tile helpers, turns the oracle's layout back into sorted order."""
    for n in SIZES:
        keys = np.arange(n, dtype=np.uint64) * 5 + 11
        got = T.emulate_unpermute(layout, O.permute(layout, keys, b or 16), b or 16)
        assert np.array_equal(got, keys), (layout, b, n)


def test_algorithm_variants_not_built_are_refused_before_device_work():
    lib = T.lib()
    lib.tl_permute_algorithm.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint32,
                                         C.c_void_p, C.c_void_p]
    assert lib.tl_permute_algorithm(T.LAYOUT_VEB, 1, C.c_void_p(256), 1000, 16, 8, None, None) == T.ERROR_UNSUPPORTED
    assert lib.tl_permute_algorithm(T.LAYOUT_BST, 7, C.c_void_p(256), 1000, 1, 8, None, None) == T.ERROR_INVALID_VALUE
    # B-tree by involutions: b must be 1 .. 2^31 - 1
    assert lib.tl_permute_algorithm(T.LAYOUT_BTREE, 1, C.c_void_p(256), 1000, 0, 8, None, None) == T.ERROR_INVALID_VALUE
    assert lib.tl_permute_algorithm(T.LAYOUT_BTREE, 1, C.c_void_p(256), 1000, 1 << 31, 8, None,
                                    None) == T.ERROR_INVALID_VALUE
