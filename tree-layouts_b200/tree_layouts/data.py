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


# ------------------------------------------------------------------ skewed keys, Zipf queries
def skewed_keys_torch(n: int, seed: int, device="cuda", oversample: float = 1.08):
    """n unique sorted keys (int64 tensor, values in [0, 2^62]): the sorted,
    deduplicated union of (a) lognormal(mu=0, sigma=2) samples scaled into
    [0, 2^62] (x / e^12 * 2^62, clamped: e^12 is the +6 sigma point) and
    (b) 5% of the keys from 1000 clusters with uniform centres and width 2^20;
    thinned evenly to exactly n."""
    import math

    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    n_a = int(n * 0.95 * oversample)
    n_b = int(n * 0.05 * oversample)
    z = torch.randn(n_a, generator=g, device=device, dtype=torch.float64)
    z.mul_(2.0).exp_().div_(math.exp(12.0)).clamp_(max=1.0).mul_(float(2**62))
    a = z.to(torch.int64)
    del z
    centres = torch.randint(0, 2**62 - 2**20, (1000,), generator=g, device=device, dtype=torch.int64)
    cid = torch.randint(0, 1000, (n_b,), generator=g, device=device, dtype=torch.int64)
    bk = centres[cid] + torch.randint(0, 2**20, (n_b,), generator=g, device=device, dtype=torch.int64)
    del cid
    allk = torch.unique(torch.cat([a, bk]))
    del a, bk
    m = allk.numel()
    if m < n:
        raise RuntimeError(f"only {m} unique keys for n={n}; raise oversample")
    idx = torch.arange(n, device=device, dtype=torch.int64).mul_(m).div_(n, rounding_mode="floor")
    return allk[idx]


def zipf_queries_torch(keys, q: int, seed: int, s: float = 1.1, hit_frac: float = 0.9):
    """hit_frac of the queries are keys whose popularity rank follows Zipf(s)
    (inverse CDF of the continuous power law on [1, n+1)), popularity rank k
    mapped to key index (k * 2654435761) mod n so that popular keys spread over
    the key space; the rest are uniform values in [min key, max key]."""
    import torch
    dev = keys.device
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    n = keys.numel()
    nh = int(round(q * hit_frac))
    u = torch.rand(nh, generator=g, device=dev, dtype=torch.float64)
    a = 1.0 - s
    k = (((float(n + 1) ** a - 1.0) * u + 1.0) ** (1.0 / a)).floor_().clamp_(1, n).to(torch.int64) - 1
    ranks = (k * 2654435761) % n
    hits = keys[ranks]
    lo, hi = int(keys[0].item()), int(keys[-1].item())
    miss = torch.randint(0, 2**62, (q - nh,), generator=g, device=dev, dtype=torch.int64) % (hi - lo + 1) + lo
    out = torch.cat([hits, miss])
    return out[torch.randperm(q, generator=g, device=dev)]


# ------------------------------------------------------------------ batched workload
def batch_keys_torch(sizes, gap_hi: int, seed: int, device="cuda"):
    """Concatenated sorted instances (each: prefix sums of uniform gaps in
    [1, gap_hi], its own seed-derived stream) and the int64 offset table."""
    import numpy as np
    import torch
    sizes = np.asarray(sizes, dtype=np.int64)
    offsets = np.zeros(len(sizes) + 1, dtype=np.int64)
    np.cumsum(sizes, out=offsets[1:])
    total = int(offsets[-1])
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    gaps = torch.randint(1, gap_hi + 1, (total,), generator=g, device=device, dtype=torch.int64)
    keys = torch.cumsum(gaps, 0)
    off_t = torch.from_numpy(offsets).to(device)
    # restart every instance's prefix sum at its own first gap
    starts = off_t[:-1]
    base = torch.zeros(len(sizes), dtype=torch.int64, device=device)
    nz = starts > 0
    base[nz] = keys[starts[nz] - 1]
    keys -= torch.repeat_interleave(base, torch.from_numpy(sizes).to(device))
    return keys, off_t


def batch_queries_torch(keys, offsets, q: int, hit_frac: float, seed: int):
    """q queries, each tagged with a uniform instance id: hit_frac drawn from that
    instance's keys, the rest uniform in its [min, max]."""
    import torch
    dev = keys.device
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    num = offsets.numel() - 1
    inst = torch.randint(0, num, (q,), generator=g, device=dev, dtype=torch.int64)
    lo_i, hi_i = offsets[inst], offsets[inst + 1]
    size = hi_i - lo_i
    u = torch.rand(q, generator=g, device=dev, dtype=torch.float64)
    pos = lo_i + (u * size.double()).long().clamp_max(size - 1)
    hits = keys[pos]
    kmin, kmax = keys[lo_i], keys[hi_i - 1]
    r = torch.randint(0, 2**62, (q,), generator=g, device=dev, dtype=torch.int64)
    miss = kmin + r % (kmax - kmin + 1)
    is_hit = torch.rand(q, generator=g, device=dev) < hit_frac
    return torch.where(is_hit, hits, miss), inst.to(torch.int32)
