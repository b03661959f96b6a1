"""The drop-in header (include/tree_layouts.cuh): a program written against the
reference's GPU template API compiles against it with nvcc, links
-ltreelayouts, runs, and leaves layouts equal to the oracle's.

The CPU test compiles and links only; the GPU test runs the program."""
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "tree-layouts_b200")
SRC = os.path.join(ROOT, "tests", "dropin", "dropin_driver.cu")


def _compile(out_dir):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    exe = os.path.join(out_dir, "dropin_driver")
    cmd = [nvcc, "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
           "-I", os.path.join(ROOT, "include"), SRC, "-o", exe, "-L", LIBDIR, "-ltreelayouts",
           "-Xlinker", f"-rpath={LIBDIR}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    return exe


def test_dropin_header_compiles_and_links(tmp_path):
    if not os.path.exists(os.path.join(LIBDIR, "libtreelayouts.so")):
        pytest.skip("libtreelayouts.so not built")
    assert os.path.exists(_compile(str(tmp_path)))


@pytest.mark.gpu
def test_dropin_program_layouts_match_oracle(tmp_path):
    exe = _compile(str(tmp_path))
    r = subprocess.run([exe, str(tmp_path)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    cases = 0
    for line in r.stdout.splitlines():
        f = dict(kv.split("=") for kv in line.split()[1:])
        layout, n, b, bits = line.split()[0], int(f["n"]), int(f["b"]), int(f["bits"])
        assert float(f["permute_ms"]) > 0 and float(f["query_ms"]) > 0 and float(f["search_ms"]) > 0
        dt = np.uint32 if bits == 32 else np.uint64
        got = np.fromfile(os.path.join(str(tmp_path), f"{layout}_{n}_{b}_{bits}.bin"), dtype=dt)
        keys = np.arange(1, n + 1, dtype=dt)
        assert np.array_equal(got, O.permute(layout, keys, b or 16)), line
        cases += 1
    assert cases == 7
