"""The oracle (oracle/oracle.c) against the reference itself.

Golden fixtures in tests/golden/ were produced by the reference's own code
compiled from its sources (tests/golden/make_golden.py): B-tree/BST layouts and
query answers from cpu/src, mvEB tables from gpu/src/query-mveb.cu, mvEB
layouts from gpu/src/mveb-cycles.cuh run on a B200, and the standard vEB
layouts, tables and query answers of cpu/src/veb-cycles.h and query-veb.*.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle as O
from tree_layouts import data

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.uint64).tobytes()).hexdigest()[:24]


@pytest.fixture(scope="module")
def gold():
    with open(os.path.join(GOLD, "golden_cpu.json")) as f:
        return json.load(f)


def test_btree_layouts_match_reference(gold):
    bad = [(e["b"], e["n"]) for e in gold["btree"] if sha(O.permutation("btree", e["n"], e["b"])) != e["sha"]]
    assert not bad, bad[:10]
    assert len(gold["btree"]) > 3000


def test_bst_layouts_match_reference(gold):
    bad = [e["n"] for e in gold["bst"] if sha(O.permutation("bst", e["n"])) != e["sha"]]
    assert not bad, bad[:10]


def test_explicit_examples(gold):
    for e in gold["examples"]:
        assert O.permutation(e["layout"], e["n"], e["b"]).tolist() == e["perm"]


def test_btree_queries_match_reference(gold):
    for e in gold["query_btree"]:
        keys = data.sorted_keys_np(e["n"], 1, 16, e["seed"])
        Q = data.queries_np(keys, e["q"], 0.5, e["seed"] + 1)
        A = O.permute("btree", keys, e["b"])
        ans = O.search("btree", A, Q, e["b"])
        assert sha(ans) == e["sha"], e
        assert int((ans != e["n"]).sum()) == e["hits"]


def test_bst_queries_match_reference(gold):
    for e in gold["query_bst"]:
        keys = data.sorted_keys_np(e["n"], 1, 16, e["seed"])
        Q = data.queries_np(keys, e["q"], 0.5, e["seed"] + 1)
        A = O.permute("bst", keys)
        assert sha(O.search("bst", A, Q)) == e["sha"], e


def test_veb_tables_match_reference(gold):
    for e in gold["tables"]:
        t = O.build_table(e["n"], e["d"])
        assert t["L"].tolist() == e["L"] and t["R"].tolist() == e["R"] and t["D"].tolist() == e["D"], e["n"]


def test_standard_veb_layouts_match_reference(gold):
    bad = [e["n"] for e in gold["veb_std"] if sha(O.permutation("veb", e["n"])) != e["sha"]]
    assert not bad, bad[:10]
    assert len(gold["veb_std"]) > 300


def test_standard_veb_tables_match_reference(gold):
    for e in gold["veb_std_tables"]:
        t = O.build_table(e["n"], e["d"], standard=True)
        assert t["L"].tolist() == e["L"] and t["R"].tolist() == e["R"] and t["D"].tolist() == e["D"], e["n"]


def test_standard_veb_queries_match_reference(gold):
    for e in gold["query_veb_std"]:
        keys = data.sorted_keys_np(e["n"], 1, 16, e["seed"])
        Q = data.queries_np(keys, e["q"], 1.0, e["seed"] + 1)
        ans = O.search("veb", O.permute("veb", keys), Q)
        assert sha(ans) == e["sha"], e
        assert int((ans != e["n"]).sum()) == e["hits"] == e["q"]


def _mveb_pos_def(n, s):
    """mvEB position from the layout's definition (independent of oracle.c)."""
    pos, nn = 0, n
    while nn > 1:
        d = nn.bit_length()
        rd = (d - 2) // 2 + 1
        ld = d - rd
        if ld & (ld - 1):
            ld = 1 << (ld - 1).bit_length()
            rd = d - ld
        r, l = (1 << rd) - 1, (1 << ld) - 1
        nf = (nn - r) // l
        inc = nn - r - nf * l
        if s < nf * (l + 1):
            i, t = divmod(s, l + 1)
            if t == l:
                nn, s = r, i
            else:
                pos, nn, s = pos + r + i * l, l, t
        elif s < nf * (l + 1) + inc:
            pos, s, nn = pos + r + nf * l, s - nf * (l + 1), inc
        else:
            s, nn = nf + (s - nf * (l + 1) - inc), r
    return pos


@pytest.mark.parametrize("n", list(range(1, 200)) + [255, 256, 1000, 65535, 65536, 70001])
def test_mveb_oracle_matches_definition(n):
    perm = O.permutation("mveb", n)
    inv = np.empty(n, dtype=np.int64)
    inv[perm.astype(np.int64)] = np.arange(n)
    idx = range(n) if n <= 2000 else np.random.default_rng(n).integers(0, n, 2000)
    for s in idx:
        assert inv[int(s)] == _mveb_pos_def(n, int(s))


def test_mveb_oracle_matches_reference_gpu():
    path = os.path.join(GOLD, "golden_mveb_gpu.json")
    if not os.path.exists(path):
        pytest.skip("mvEB fixtures from the reference GPU run not generated yet")
    with open(path) as f:
        g = json.load(f)
    bad = [e["n"] for e in g["mveb"] if sha(O.permutation("mveb", e["n"])) != e["sha"]]
    assert not bad, bad[:10]
    for e in g["examples"]:
        assert O.permutation("mveb", e["n"]).tolist() == e["perm"]


def test_mveb_queries_find_every_key_and_reject_absent():
    for n in [1, 2, 3, 7, 100, 1023, 4097, 65535, 100000]:
        keys = data.sorted_keys_np(n, 2, 9, n)
        A = O.permute("mveb", keys)
        ans = O.search("mveb", A, keys)
        assert (A[ans.astype(np.int64)] == keys).all()
        absent = keys - 1  # gaps >= 2: never a key
        assert (O.search("mveb", A, absent) == n).all()


@pytest.mark.skipif(O.ref_cpu() is None, reason="reference build oracle/_ref absent")
def test_oracle_matches_reference_build_directly():
    ref = O.ref_cpu()
    rng = np.random.default_rng(0)
    for b in [2, 16, 33]:
        for n in rng.integers(b + 1, 200000, 5):
            n = int(n)
            from tests_golden_helper import ref_level_count_ok  # noqa
            if not ref_level_count_ok(n, b):
                continue
            A = np.arange(n, dtype=np.uint64)
            ref.ref_cpu_permute_btree_u64(A, n, b, 2)
            assert np.array_equal(A, O.permutation("btree", n, b))
