"""Seeded synthetic workloads (keys and queries) for the tests and the benchmark.

The reference has no datasets; its drivers fill keys 1..n (gpu/src/common.cuh:35)
and draw hit-only queries with rand() (:45-60).  The workloads here follow the
shapes the benchmark is quoted on: strictly increasing keys built as prefix sums
of uniform random gaps, and query batches mixing uniform hits with uniform
values in [min key, max key] (mostly absent).

Two generators with the same distributions: numpy on the host (small cases,
checked against the oracle) and torch on the device (full-size cases, generated
in HBM).  They are not bit-identical to each other; each is deterministic in its
seed.
"""
from __future__ import annotations

import numpy as np


# ------------------------------------------------------------------ host (numpy)
def sorted_keys_np(n: int, gap_lo: int, gap_hi: int, seed: int, dtype=np.uint64) -> np.ndarray:
    rng = np.random.default_rng(seed)
    keys = np.cumsum(rng.integers(gap_lo, gap_hi + 1, size=n, dtype=np.uint64), dtype=np.uint64)
    if dtype == np.uint32:
        assert n == 0 or int(keys[-1]) < 2**32, "keys overflow uint32"
    return keys.astype(dtype)


def queries_np(keys: np.ndarray, q: int, hit_frac: float, seed: int) -> np.ndarray:
    """hit_frac of the queries drawn uniformly from the keys, the rest uniform in
    [min key, max key]; shuffled."""
    rng = np.random.default_rng(seed)
    nh = int(round(q * hit_frac))
    hits = keys[rng.integers(0, len(keys), size=nh)]
    lo, hi = int(keys[0]), int(keys[-1])
    miss = rng.integers(lo, hi + 1, size=q - nh, dtype=np.uint64).astype(keys.dtype)
    out = np.concatenate([hits, miss])
    rng.shuffle(out)
    return out


# ------------------------------------------------------------------ device (torch)
def sorted_keys_torch(n: int, gap_lo: int, gap_hi: int, seed: int, key_bytes: int = 8, device="cuda"):
    """Strictly increasing keys in HBM.  4-byte keys come back as int32 tensors
    holding the uint32 bit patterns (the library compares them unsigned)."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    out = torch.empty(n, dtype=torch.int64, device=device)
    chunk = 1 << 27
    carry = 0
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        part = torch.randint(gap_lo, gap_hi + 1, (e - s,), generator=g, device=device, dtype=torch.int64)
        torch.cumsum(part, 0, out=out[s:e])
        out[s:e] += carry
        carry = int(out[e - 1].item())
    if key_bytes == 4:
        assert carry < 2**32, "keys overflow uint32"
        return out.to(torch.int32)  # two's-complement truncation keeps the uint32 bits
    return out


def queries_torch(keys, q: int, hit_frac: float, seed: int, lo: int | None = None, hi: int | None = None):
    """Same mix as queries_np, on the device.  `keys` is the sorted key tensor."""
    import torch
    dev = keys.device
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    n = keys.numel()
    nh = int(round(q * hit_frac))
    hits = keys[torch.randint(0, n, (nh,), generator=g, device=dev)]
    if lo is None:
        lo = _as_unsigned(keys[0].item(), keys.element_size())
        hi = _as_unsigned(keys[-1].item(), keys.element_size())
    span = hi - lo + 1
    r = torch.randint(0, 2**62, (q - nh,), generator=g, device=dev, dtype=torch.int64) % span + lo
    miss = r.to(keys.dtype) if keys.element_size() == 8 else r.to(torch.int32)
    out = torch.cat([hits, miss])
    return out[torch.randperm(q, generator=g, device=dev)]


def _as_unsigned(v: int, nbytes: int) -> int:
    return v & ((1 << (8 * nbytes)) - 1)
