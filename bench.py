#!/usr/bin/env python3
"""Benchmark of the tree-layout hot path on B200.

Default workload (the configuration the headline metric is quoted on): in-place
permutation of n = 500,000,000 sorted uint64 keys (prefix sums of uniform gaps
in [1,16], seed 3) into a level-order B-tree with b = 16 keys per node, then
q = 2^27 point queries (seed 4, 50% hits / 50% uniform in [min, max]).

One step = one permutation of the full array.  Between steps the array is
restored from a pristine sorted copy (untimed, like the reference drivers'
re-initialisation); the 4 GB input is far larger than the 126 MB L2, so no
extra flush is needed.

Besides the headline the line carries, each outside the timed region:
parity (the permuted array compared word for word with the reference's own CPU
permutation of the same keys, and a sample of query answers with its CPU
search); layouts (every layout at 2^30-class sizes, timed the same way and
checked the same way); first_call (host wall time of a first call for a new
geometry); the reverse permutation, the involutions variant, queries, the
learned-start query, the batched mode, the CPU baseline (all host threads and
one) and the end-to-end permutation with host buffers.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints ONE JSON line (rank 0).  Multi-GPU (torchrun): every rank permutes its
own replica (a single array's permutation does not shard), value = all ranks'
bytes / max-over-ranks time ("weak" scaling).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "tree-layouts_b200"))

WORKLOADS = {
    # name: (layout, b, n, key_bytes, gap_hi, key seed, q, query seed)
    "btree-b16-n500M-u64": ("btree", 16, 500_000_000, 8, 16, 3, 2**27, 4),
    "btree-b16-n2^30-u64": ("btree", 16, 2**30, 8, 16, 8, 2**27, 9),
    "mveb-n2^30-1-u32": ("mveb", 0, 2**30 - 1, 4, 3, 5, 2**27, 6),
    "mveb-n300M-u32": ("mveb", 0, 300_000_000, 4, 3, 5, 2**27, 6),
    # the standard vEB layout of the reference's CPU code
    "veb-n2^30-1-u32": ("veb", 0, 2**30 - 1, 4, 3, 5, 2**27, 6),
    "veb-n300M-u32": ("veb", 0, 300_000_000, 4, 3, 5, 2**27, 6),
    "bst-n2^30-1-u64": ("bst", 1, 2**30 - 1, 8, 16, 1, 2**27, 2),
    "bst-n2^20-1-u64": ("bst", 1, 2**20 - 1, 8, 16, 1, 2**20, 2),
    # small cases for ncu captures (inputs above L2, a few GB on the device)
    "btree-b8-n60M-u64": ("btree", 8, 60_000_000, 8, 16, 3, 2**24, 4),
    "bst-n2^26-1-u64": ("bst", 1, 2**26 - 1, 8, 16, 1, 2**24, 2),
}
DEFAULT = "btree-b16-n500M-u64"
METRIC = "permute GB/s (2*n*key_bytes / device time), in-place sorted -> level-order B-tree"


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


L2_BYTES = 126e6  # B200 L2


def query_bytes_model(layout, n, b, kb):
    """Algorithmic HBM bytes of one exact query: the key (w) and the answer (8)
    plus one node fetch for every level below the L2-resident depth (the
    largest k whose levels 0..k-1 hold at most half of L2).  A node fetch is
    ceil(b w / 32) 32-byte sectors for the B-tree, one sector for BST and vEB.
    Returns (bytes, l2_levels, levels)."""
    if layout == "btree":
        k = b + 1
        h, pw = 0, 1
        while pw <= (n + 1) // k:  # levels of the largest perfect top tree
            pw *= k
            h += 1
        sizes = [(k ** lv) * b for lv in range(h)]
        if pw - 1 != n:
            sizes.append(n - (pw - 1))  # the last level's keys
        fetch = -(-b * kb // 32) * 32
    else:
        d = n.bit_length()
        sizes = [min(1 << lv, n - ((1 << lv) - 1)) for lv in range(d)]
        fetch = 32
    acc, l2_levels = 0, 0
    for sz in sizes:
        if acc + sz * kb > L2_BYTES / 2:
            break
        acc += sz * kb
        l2_levels += 1
    return kb + 8 + fetch * (len(sizes) - l2_levels), l2_levels, len(sizes)


def query_grouped(layout, n, kb, q):
    """Whether the library searches a batch grouped by value first: BST and vEB
    batches of 2^21 queries or more over a BST layout of 64 MB or more or a vEB
    layout of 4 MB or more (the thresholds of csrc/query.cu's launch_query)."""
    return (layout in ("bst", "mveb", "veb") and (1 << 21) <= q < (1 << 32)
            and n * kb >= (64 << 20 if layout == "bst" else 4 << 20))


def query_kernel_name(layout, b, kb):
    """The kernel the library launches for a query batch over a 32-byte aligned
    layout (torch allocations are)."""
    if layout == "btree":
        nb = b * kb
        if nb in (64, 128, 256):
            return f"btree_query_group32_kernel ({max(2, nb // 64)} lanes per node, 32-byte loads)"
        if nb % 32 == 0 and nb <= 256:
            return "btree_query_v32_kernel (a thread per query, 32-byte loads)"
        if nb % 16 == 0 and nb <= 256:
            return "btree_query_vec_kernel (a thread per query, 16-byte loads)"
        return "btree_query_kernel (a lane per key)"
    if layout == "bst":
        return "bst_query_kernel"
    return "veb_query_kernel"


def dist_setup(n_gpus):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return rank, world, local


def barrier(world):
    import torch
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()


def reduce_max(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class ClockSampler:
    """SM clock and throttle reasons sampled through NVML every few ms while the
    timed region runs (same counters as nvidia-smi's clocks/clocks_event_reasons)."""
    REASONS = {  # NVML clocks-event-reason bits
        "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
        "hw_power_brake_slowdown": 0x80, "sw_power_cap": 0x4,
    }

    def __init__(self, index, period_s=0.005):
        self.index, self.period = index, period_s
        self.samples, self.reasons, self.max_mhz = [], set(), None
        self.ok = False
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM))
            self.ok = True
        except Exception as e:  # no NVML: report it rather than invent numbers
            self.err = repr(e)

    def _run(self):
        while not self.stop_evt.is_set():
            try:
                self.samples.append(float(self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM)))
                bits = self.nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                for name, bit in self.REASONS.items():
                    if bits & bit:
                        self.reasons.add(name)
            except Exception:
                pass
            self.stop_evt.wait(self.period)

    def start(self):
        import threading
        if not self.ok:
            return
        self.stop_evt = threading.Event()
        self.t = threading.Thread(target=self._run, daemon=True)
        self.t.start()

    def stop(self):
        if not self.ok:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [f"nvml unavailable: {self.err}"]}
        self.stop_evt.set()
        self.t.join()
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None,
                "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons), "samples": len(self.samples)}


REF_FUNCS = {"bst": "timePermuteBST (cpu/src/bst-involutions.h)",
             "btree": "timePermuteBtree (cpu/src/btree-cycles.h)",
             "veb": "timePermutevEB (cpu/src/veb-cycles.h)"}


def sample_keys(n_sample, gap_hi, seed):
    import numpy as np
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.integers(1, gap_hi + 1, size=n_sample, dtype=np.uint64), dtype=np.uint64)


def cpu_reference_permute(layout, b, n_sample, key_bytes, reps, min_seconds=8.0, gap_hi=16, seed=3, threads=0,
                          pristine=None):
    """The reference's own CPU OpenMP permutation (compiled from its sources into
    oracle/_ref/libref_cpu.so: B-tree, BST, standard vEB) on n_sample uint64 keys
    (prefix sums of uniform gaps in [1, gap_hi] from a numpy stream seeded with
    `seed`; the permutation never looks at key values) with `threads` host
    threads (0: all).  The reference has no CPU mvEB (its CPU tree is the
    standard vEB), and the oracle's single-thread C restatement of its mvEB
    stands in there, as it does for every layout when that build is absent."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    threads = threads or os.cpu_count() or 1
    ref = O.ref_cpu() if layout != "mveb" else None
    kind = "reference" if ref is not None else "port"
    if ref is None:
        threads = 1
    if pristine is None:
        pristine = sample_keys(n_sample, gap_hi, seed)
    A = np.empty(n_sample, dtype=np.uint64)
    times = []
    t_begin = time.time()
    for r in range(reps):
        A[:] = pristine  # re-initialised between runs (untimed)
        if ref is not None:
            if layout == "bst":
                ms = ref.ref_cpu_permute_bst_u64(A, n_sample, threads)
            elif layout == "veb":
                ms = ref.ref_cpu_permute_veb_u64(A, n_sample, threads)
            else:
                ms = ref.ref_cpu_permute_btree_u64(A, n_sample, b, threads)
        elif layout in ("mveb", "veb"):
            t0 = time.perf_counter()
            (O.lib().orc_permute_mveb if layout == "mveb" else O.lib().orc_permute_veb_std)(A, n_sample)
            ms = (time.perf_counter() - t0) * 1e3
        else:
            ms = O.lib().orc_time_permute_btree(A, n_sample, b if layout != "bst" else 1)
        times.append(ms)
        if time.time() - t_begin > min_seconds and r >= 1:
            break
    ms = statistics.median(times)
    gbs = 2.0 * n_sample * 8 / (ms * 1e-3) / 1e9
    what = REF_FUNCS[layout] if ref is not None else f"the oracle's C port of the reference's {layout} permutation"
    return {"value": round(gbs, 3), "unit": "GB/s", "cores": threads, "kind": kind,
            "sample": f"{layout}{'' if layout != 'btree' else f' b={b}'} n={n_sample} uint64 keys (prefix sums "
                      f"of uniform gaps in [1,{gap_hi}], seed {seed}), median of {len(times)} runs of {what} on "
                      f"{threads} thread(s) ({ms:.1f} ms); GB/s counts 8-byte keys"}


def workload_config(args, layout, b, n, kb, gap_hi, kseed, world):
    """The config block both arms print for a workload."""
    return {"workload": args.workload, "layout": layout, "b": b, "n": n, "key_bytes": kb,
            "keys": f"prefix sums of uniform gaps in [1,{gap_hi}], seed {kseed}",
            "l2": "inputs larger than L2 (no flush needed)",
            "restore": "array re-initialised from a pristine copy between steps, untimed",
            "parallelism": "replicas" if world > 1 else "single GPU"}


def run_reference(args, rank):
    layout, b, n, kb, gap_hi, kseed, *_ = WORKLOADS[args.workload]
    if rank != 0:
        return
    # the single-thread mvEB port runs on a bounded sample (about 2 s a run)
    n_sample = min(n, args.ref_n) if args.ref_n else (n if layout != "mveb" else min(n, 2**28 - 1))
    steps = []
    keys = sample_keys(n_sample, gap_hi, kseed)
    for _ in range(args.warmup):
        cpu_reference_permute(layout, b, n_sample, kb, 1, 0, gap_hi=gap_hi, seed=kseed, pristine=keys)
    for _ in range(args.steps):
        steps.append(cpu_reference_permute(layout, b, n_sample, kb, 1, 0, gap_hi=gap_hi, seed=kseed, pristine=keys))
    vals = [s["value"] for s in steps]
    v = statistics.median(vals)
    ms = 2.0 * n_sample * 8 / (v * 1e9) * 1e3
    cb = dict(steps[0])
    cb["value"] = v
    metric = METRIC if layout == "btree" else METRIC.replace("level-order B-tree", layout)
    print(json.dumps({
        "impl": "reference", "metric": metric, "value": v, "unit": "GB/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64" if kb == 8 else "u32", "data": "synthetic",
        "config": workload_config(args, layout, b, n, kb, gap_hi, kseed, 1),
        "reference": {"sample_n": n_sample,
                      "note": f"{cb['kind']} CPU permutation on the host cores: {cb['sample']}"},
        "cpu_baseline": cb,
        "e2e": {"value": v, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


# segments of the learned query's rank model: measured on B200 (2^30 skewed
# keys, 2^28 queries) 2^16: 1.28x the plain query, 2^18: 1.44x, 2^20: 1.55x,
# 2^21: 1.57x, 2^22: 1.57x
LEARNED_LEAVES = 1 << 21


def learned_section(args, dev):
    """Learned-start vs plain B-tree queries on skewed keys: n = 2^30 unique
    uint64 keys (lognormal + clusters, seed 8), b = 16, q = 2^28 queries (seed 9,
    90% Zipf(1.1) hits, 10% uniform misses).  The model is trained on the sorted
    keys by the library's own kernels, then the keys are permuted in place."""
    import numpy as np
    import torch

    import tree_layouts as T
    import tree_layouts.learned as LL
    from tree_layouts import data

    n, b, q = args.learned_n, 16, args.learned_q
    t0 = time.time()
    keys = data.skewed_keys_torch(n, 8, dev)
    gen_s = time.time() - t0
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    model, leaves = LL.train(keys, num_leaves=LEARNED_LEAVES, steps=args.learned_steps, batch=65536, lr=3e-3,
                             seed=1)
    ev1.record()
    torch.cuda.synchronize()
    train_ms = ev0.elapsed_time(ev1)
    # the same method without the trained root (segments indexed by the
    # normalised key directly), for the ablation line
    model0, leaves0 = LL.train(keys, num_leaves=LEARNED_LEAVES, steps=args.learned_steps, batch=65536, lr=3e-3,
                               seed=1, train_root=False)
    Q = data.zipf_queries_torch(keys, q, 9)
    sorted_keys = keys.clone() if args.parity else None
    T.permute("btree", keys, b)  # keys now hold the layout
    tree = keys
    par, host = None, None
    if args.parity:  # the layout against the reference's CPU permutation, untimed
        par, host = parity_module().check_layout("btree", b, sorted_keys, tree, keep_host=True)
        del sorted_keys
    plain = torch.empty(q, dtype=torch.int64, device=dev)
    learned = torch.empty_like(plain)
    stats = torch.zeros(2, dtype=torch.int64, device=dev)
    for _ in range(2):
        T.query("btree", tree, Q, plain, b)
        LL.query(tree, model, leaves, Q, learned, b)
    p_ms, l_ms = [], []
    for _ in range(3):
        p_ms.append(T.query("btree", tree, Q, plain, b, timed=True))
        l_ms.append(LL.query(tree, model, leaves, Q, learned, b, timed=True))
    LL.query(tree, model, leaves, Q, learned, b, stats=stats)
    exact = bool(torch.equal(plain, learned))
    LL.query(tree, model0, leaves0, Q, learned, b)
    l0_ms = statistics.median([LL.query(tree, model0, leaves0, Q, learned, b, timed=True) for _ in range(3)])
    exact0 = bool(torch.equal(plain, learned))
    del leaves0
    if par is not None:
        par["answers"] = parity_module().check_answers("btree", b, host, Q, plain, 1 << 20, 9)
        del host
    lv = LL.leaves_numpy(leaves)
    used = lv["empty"] == 0
    win = (lv["eps_lo"].astype(np.int64) + lv["eps_hi"])[used]
    pm, lm = statistics.median(p_ms), statistics.median(l_ms)
    out = {"workload": f"B-tree b=16 over n={n} skewed u64 keys (lognormal sigma=2 + 5% in 1000 clusters), "
                       f"{q} queries 90% Zipf(1.1) / 10% uniform misses",
           "n": n, "q": q, "plain_queries_per_s": round(q / (pm * 1e-3), 1),
           "learned_queries_per_s": round(q / (lm * 1e-3), 1), "speedup": round(pm / lm, 3),
           "exact": exact, "plain_ms": round(pm, 3), "learned_ms": round(lm, 3),
           "kernels": {"plain": query_kernel_name("btree", b, 8),
                       "learned": "learned_query_group_kernel (2 lanes per node, a per-warp queue of "
                                  "prepared starts)"},
           "fallback_frac": round(int(stats[0].item()) / q, 4),
           "mean_start_depth": round(int(stats[1].item()) / q, 3),
           "train_ms": round(train_ms, 1), "train_loss": model.train_loss, "keygen_s": round(gen_s, 1),
           "leaves": LEARNED_LEAVES, "leaves_used": int(used.sum()), "window_median": int(np.median(win)),
           "window_p99": int(np.percentile(win, 99)),
           "leaf_only": {"learned_ms": round(l0_ms, 3), "speedup": round(pm / l0_ms, 3), "exact": exact0,
                         "note": "the same two-stage method with an untrained root (segments indexed by the "
                                 "normalised key), same keys and queries"},
           "parity": par}
    del keys, tree, Q, plain, learned, leaves
    torch.cuda.empty_cache()
    return out


def batched_section(args, dev):
    """Batched permute + queries: 4096 sorted uint64 arrays, sizes log-uniform in
    [2^10, 2^22] (seed 7), keys prefix sums of uniform gaps in [1, 64], int64
    offsets; each permuted to a B-tree with b = 8 by one persistent launch
    replayed from a CUDA graph; 2^26 queries with uniform instance ids, 70% hits.
    The autotuner picks the tuning first (on the same data, left sorted)."""
    import torch

    import tree_layouts.batched as TB
    from tree_layouts import data

    sizes = TB.batch_sizes_np(args.batch_num, 10, args.batch_hi, 7)
    keys, off = data.batch_keys_torch(sizes, 64, 7, dev)
    total = int(sizes.sum())
    Q, inst = data.batch_queries_torch(keys, off, args.batch_q, 0.7, 8)
    plan = TB.BatchPlan(off, b=8)
    t0 = time.time()
    report = plan.autotune(keys, Q, inst) if args.batch_tune else dict(plan.tuning())
    tune_s = time.time() - t0
    pristine = keys.clone()
    ws = plan.workspace()
    s = torch.cuda.Stream()
    plan.permute(keys, ws, stream=s)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        plan.permute(keys, ws, stream=s, check=False)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ms = []
    for i in range(args.warmup + args.steps):
        keys.copy_(pristine)
        torch.cuda.synchronize()
        with torch.cuda.stream(s):  # CUDAGraph.replay launches on the current stream
            e0.record(s)
            g.replay()
            e1.record(s)
        torch.cuda.synchronize()
        if i >= args.warmup:
            ms.append(e0.elapsed_time(e1))
    plan.status(ws)
    ans = torch.empty(Q.numel(), dtype=torch.int64, device=dev)
    for _ in range(2):
        plan.query(keys, Q, inst, ans)
    qms = statistics.median(plan.query(keys, Q, inst, ans, timed=True) for _ in range(3))
    # every instance against the reference's CPU permutation and every answer
    # checked (untimed)
    par = parity_module().check_batched(8, sizes, pristine, keys, off, Q, inst, ans) if args.parity else None
    del g
    pm = statistics.median(ms)
    out = {"workload": f"{len(sizes)} uint64 arrays, sizes log-uniform [2^10, 2^{args.batch_hi}], b = 8, one persistent launch "
                       f"replayed from a CUDA graph; {args.batch_q} queries, 70% hits",
           "arrays": len(sizes), "total_keys": total,
           "permute_ms": round(pm, 3), "permute_GBps": round(2.0 * total * 8 / (pm * 1e-3) / 1e9, 1),
           "permute_frac_of_peak": round(2.0 * total * 8 / (pm * 1e-3) / 1e9 / peaks()[0], 4),
           "queries": Q.numel(), "query_ms": round(qms, 3), "queries_per_s": round(Q.numel() / (qms * 1e-3), 1),
           "autotune_s": round(tune_s, 2), "tuning": {k: report[k] for k in ("threads", "query_chunk")},
           "ordered_instances": plan.ordered()[0], "ordered_keys": plan.ordered()[1],
           "parity": par}
    del keys, pristine, Q, inst, ans, ws
    torch.cuda.empty_cache()
    return out


def parity_module():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import parity
    return parity


def time_permutation(L, layout, b, n, kb, pristine, A, stream, warmup, steps, world=1, clocks_index=None):
    """W untimed and K timed permutations of A (restored from `pristine`,
    untimed, before each); per step the device time of the stream pass and of
    the second pass (CUDA events on `stream`)."""
    import ctypes as CT

    import tree_layouts as T
    lay = T.LAYOUTS[layout]
    phases = (CT.c_float * 2)()

    def step():
        A.copy_(pristine)  # re-initialise (untimed)
        rc = L.tl_debug_permute_phases(lay, A.data_ptr(), n, b or 16, kb, stream.cuda_stream, phases)
        if rc:
            raise T.TreeLayoutError(rc, "permute")
        return phases[0], phases[1]

    for _ in range(warmup):
        step()
    clocks = ClockSampler(clocks_index if clocks_index is not None else 0)
    barrier(world)
    clocks.start()
    t_stream, t_pass2 = [], []
    for _ in range(steps):
        a, c = step()
        t_stream.append(a)
        t_pass2.append(c)
    barrier(world)
    return t_stream, t_pass2, clocks.stop()


def permute_stats(L, layout, b, n, kb, t_stream, t_pass2, peak, peak_kind):
    """Roofline block of one timed permutation: the stream kernel (the
    dominant one) against the measured HBM peak, the second pass, the schedule."""
    import ctypes as CT

    import tree_layouts as T
    lay = T.LAYOUTS[layout]
    bytes_step = 2.0 * n * kb
    step_ms = [a + c for a, c in zip(t_stream, t_pass2)]
    ms = sum(step_ms) / len(step_ms)
    stream_ms = sum(t_stream) / len(t_stream)
    pass2_ms = sum(t_pass2) / len(t_pass2)
    achieved = bytes_step / (stream_ms * 1e-3) / 1e9
    skeys = CT.c_uint64(0)
    L.tl_debug_permute_scratch_keys.argtypes = [CT.c_int, CT.c_uint64, CT.c_uint64, CT.c_uint32,
                                                CT.POINTER(CT.c_uint64)]
    if L.tl_debug_permute_scratch_keys(lay, n, b or 16, kb, CT.byref(skeys)):
        raise RuntimeError("tl_debug_permute_scratch_keys")
    pass2_bytes = 2.0 * skeys.value * kb
    stalls, polls = CT.c_uint64(0), CT.c_uint64(0)  # of the last timed permutation
    L.tl_debug_wait_stats(CT.byref(stalls), CT.byref(polls))
    L.tl_debug_permute_plan.argtypes = [CT.c_int, CT.c_uint64, CT.c_uint64, CT.c_uint32]
    plan = L.tl_debug_permute_plan(lay, n, b or 16, kb)
    pass2_kernel = {0: "btree_copy_kernel", 1: "btree_copy_kernel",
                    2: "btree_copy_kernel + btree_fix_kernel"}.get(plan, "mveb_scatter_kernel")
    return {"bound": "hbm", "kernel": "mveb_stream_kernel" if layout in ("mveb", "veb") else "btree_stream_kernel",
            "schedule": {0: "right-to-left", 1: "left-to-right", 2: "ordered tiles"}.get(plan, "vEB units"),
            "stalled_waits": stalls.value, "stall_polls": polls.value,
            "blocks_per_sm": L.tl_debug_stream_blocks_per_sm(lay, kb),
            "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "peak_source": f"hbm_gbs of {peak_kind}",
            "traffic": None, "algorithmic_bytes_per_launch": int(bytes_step),
            "stream_ms": round(stream_ms, 4), "pass2_kernel": pass2_kernel,
            "pass2_ms": round(pass2_ms, 4), "pass2_bytes_per_launch": int(pass2_bytes),
            "pass2_achieved": round(pass2_bytes / (pass2_ms * 1e-3) / 1e9, 1) if pass2_ms > 0 else None,
            "whole_ms": round(ms, 4), "whole_GBps": round(bytes_step / (ms * 1e-3) / 1e9, 1),
            "whole_permute_frac": round(bytes_step / (ms * 1e-3) / 1e9 / peak, 4)}


def measured_traffic(workload, n):
    """DRAM bytes of one stream-kernel launch from the committed ncu summary
    (profiles/stream_traffic_<workload>.json), or None: the capture's reads and
    writes, each scaled to this launch's keys."""
    prof = os.path.join(ROOT, "profiles", f"stream_traffic_{workload}.json")
    if not os.path.exists(prof):
        return None
    with open(prof) as f:
        t = json.load(f)
    scale = n / float(t["n_captured"])
    return int(round((t["dram_bytes_read"] + t["dram_bytes_write"]) * scale))


LAYOUT_WORKLOADS = ["btree-b16-n2^30-u64", "bst-n2^30-1-u64", "mveb-n2^30-1-u32", "mveb-n300M-u32",
                    "veb-n2^30-1-u32"]


def layouts_section(args, L, dev, stream, local, peak, peak_kind):
    """The permutation of 2^30-class arrays into every layout, each timed like
    the headline (device time, W warm-up and K timed steps, clocks sampled) and
    checked bit for bit against the CPU checker after the timed steps; then
    2^27 plain queries on the layout (median of 3 after 2 warm-up batches),
    a 2^20 sample of the answers checked against the CPU checker."""
    import torch

    from tree_layouts import data
    import tree_layouts as T
    P = parity_module()
    out = {}
    for name in LAYOUT_WORKLOADS:
        layout, b, n, kb, gap_hi, kseed, q, qseed = WORKLOADS[name]
        pristine = data.sorted_keys_torch(n, 1, gap_hi, kseed, kb, dev)
        A = torch.empty_like(pristine)
        t_stream, t_pass2, clk = time_permutation(L, layout, b, n, kb, pristine, A, stream, args.warmup,
                                                  args.steps, 1, local)
        st = permute_stats(L, layout, b, n, kb, t_stream, t_pass2, peak, peak_kind)
        keep = args.layout_queries and q > 0
        rep, host = P.check_layout(layout, b or 16, pristine, A, keep_host=keep)
        out[name] = {"layout": layout, "n": n, "key_bytes": kb,
                     "keys": f"prefix sums of uniform gaps in [1,{gap_hi}], seed {kseed}",
                     "whole_GBps": st["whole_GBps"], "whole_permute_frac": st["whole_permute_frac"],
                     "ms": st["whole_ms"], "stream_frac": st["frac"], "stream_ms": st["stream_ms"],
                     "pass2_ms": st["pass2_ms"], "schedule": st["schedule"], "kernel": st["kernel"],
                     "stalled_waits": st["stalled_waits"], "steps": args.steps, "clocks": clk, "parity": rep}
        if keep:
            # the plain queries of the layout (device time; BST and vEB batches
            # this large are searched grouped by value, the grouping included)
            Q = data.queries_torch(pristine, q, 0.5, qseed)
            ans = torch.empty(q, dtype=torch.int64, device=dev)
            tabs = T.VebTablesDevice(n, dev, standard=layout == "veb") if layout in ("mveb", "veb") else None
            for _ in range(2):
                T.query(layout, A, Q, ans, b or 16, tables=tabs)
            qms = statistics.median([T.query(layout, A, Q, ans, b or 16, tables=tabs, timed=True)
                                     for _ in range(3)])
            qbytes, l2lv, nlv = query_bytes_model(layout, n, b or 16, kb)
            qps = q / (qms * 1e-3)
            grouped = query_grouped(layout, n, kb, q)
            out[name]["queries"] = {
                "q": q, "ms": round(qms, 3), "queries_per_s": round(qps, 1),
                "frac_of_byte_model": round(qps * qbytes / (peak * 1e9), 4), "bytes_per_query": qbytes,
                "kernel": query_kernel_name(layout, b or 16, kb) + (", batch grouped by value" if grouped else ""),
                "hits": int((ans != n).sum().item()),
                "parity": P.check_answers(layout, b or 16, host, Q, ans, 1 << 20, qseed)}
            del Q, ans, tabs
        del pristine, A, host
        torch.cuda.empty_cache()
    return out


def run_ours(args, rank, world, local):
    import ctypes as CT

    import torch

    import tree_layouts as T
    from tree_layouts import data

    layout, b, n, kb, gap_hi, kseed, q, qseed = WORKLOADS[args.workload]
    if args.n:
        n = args.n
    L = T.lib()
    L.tl_debug_set_schedule(1 if args.schedule == "fixed" else 0)
    L.tl_debug_set_query_variant.argtypes = [CT.c_int]
    L.tl_debug_set_query_variant(args.query_variant)
    L.tl_debug_permute_phases.argtypes = [CT.c_int, CT.c_void_p, CT.c_uint64, CT.c_uint64, CT.c_uint32,
                                          CT.c_void_p, CT.POINTER(CT.c_float)]
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream()
    lay = T.LAYOUTS[layout]
    peak, peak_kind = peaks()

    # first call for a new geometry through the drop-in path (host wall time, as
    # timePermuteBtree returns it), after a small permutation has set up the
    # context and loaded the kernels; then the same call again
    small = data.sorted_keys_torch(100_003, 1, gap_hi, 1, kb, dev)
    T.permute(layout, small, b or 16)
    del small
    pristine = data.sorted_keys_torch(n, 1, gap_hi, kseed + rank, kb, dev)
    A = torch.empty_like(pristine)
    first = []
    for _ in range(2):
        A.copy_(pristine)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rc = L.tl_permute(lay, CT.c_void_p(A.data_ptr()), n, b or 16, kb, None, 0, CT.c_void_p(stream.cuda_stream),
                          None)
        first.append((time.perf_counter() - t0) * 1e3)
        if rc:
            raise T.TreeLayoutError(rc, "permute (first call)")
    first_call = {"first_ms": round(first[0], 3), "warm_ms": round(first[1], 3),
                  "note": "host wall time of tl_permute (library-allocated workspace, synchronous) for a geometry "
                          "not seen before in the process, then for the same geometry again"}

    t_stream, t_pass2, clk = time_permutation(L, layout, b, n, kb, pristine, A, stream, args.warmup, args.steps,
                                              world, local)
    launches_per_step = L.tl_debug_permute_launches()
    step_ms = [a + c for a, c in zip(t_stream, t_pass2)]
    ms_local = sum(step_ms) / len(step_ms)
    ms = reduce_max(ms_local, world)
    bytes_step = 2.0 * n * kb
    value = world * bytes_step / (ms * 1e-3) / 1e9
    roof = permute_stats(L, layout, b, n, kb, t_stream, t_pass2, peak, peak_kind)
    roof["traffic"] = measured_traffic(args.workload, n)
    if roof["traffic"] is not None:
        roof["traffic_per_algorithmic_byte"] = round(roof["traffic"] / bytes_step, 4)
        roof["traffic_source"] = (f"profiles/stream_traffic_{args.workload}.json: ncu dram__bytes_read.sum + "
                                  "dram__bytes_write.sum of one launch at 2e8 keys, scaled by keys")

    # bit-exact check of the last timed permutation against the CPU checker
    # (the reference's own CPU code where it has one), outside the timed region
    parity = None
    host_layout = None
    if args.parity:
        P = parity_module()
        parity, host_layout = P.check_layout(layout, b or 16, pristine, A, keep_host=args.queries and q > 0)
        parity["config"] = args.workload

    # the reverse permutation (layout -> sorted order) of the same array, device time
    rinfo = None
    if args.reverse:
        layout_copy = A.clone()
        ws = torch.empty(max(1, T.unpermute_workspace_bytes(layout, n, b or 16, kb)), dtype=torch.uint8, device=dev)
        rms = []
        for i in range(args.warmup + min(args.steps, 5)):
            A.copy_(layout_copy)  # untimed
            r = T.unpermute(layout, A, b or 16, workspace=ws, timed=True)
            if i >= args.warmup:
                rms.append(r)
        assert torch.equal(A, pristine), "reverse permutation check failed"
        r_med = statistics.median(rms)
        rinfo = {"kernel": "device copy + " + ("veb_gather_kernel" if layout in ("mveb", "veb") else "btree_gather_kernel"),
                 "ms": round(r_med, 4), "GBps": round(bytes_step / (r_med * 1e-3) / 1e9, 1),
                 "frac_of_peak": round(bytes_step / (r_med * 1e-3) / 1e9 / peak, 4),
                 "equal_to_sorted": True,
                 "note": "2*n*w / device time; the pass moves 4*n*w (a copy to the workspace, then the gather)"}
        del layout_copy, ws
        A.copy_(pristine)
        T.permute(layout, A, b or 16)  # the layout again, for the queries below

    # the reference's algorithm families as variants (involutions, cycle-leader,
    # hybrid), device time, each checked against the stream permutation's layout
    vinfo = None
    if args.variants and layout in ("bst", "btree", "mveb"):
        perm_ref = A.clone()  # the stream permutation's layout (A holds it here)
        kern = {("bst", "involutions"): "bitrev + lowrev swaps (+ 2 involutions and 3 reversals if non-perfect)",
                ("btree", "involutions"): "per level: 2 base-(b+1) digit-reversal swap passes + 2 modular "
                                          "involutions (+ 4 involutions and 6 reversals for the partial last level)",
                ("mveb", "involutions"): "per split: a (l+1)-way unshuffle and an l-way shuffle (4 modular "
                                         "involutions), balanced bottoms by 2-digit swaps + 2 involutions per round, "
                                         "rotations for non-perfect trees",
                ("bst", "cycles"): "the B-tree cycle-leader steps with b = 1",
                ("btree", "cycles"): "per round: equidistant gathers (cycle-leader walks + two reversal passes) over "
                                     "partitions of (b+1)^2 c keys; the partial last level first",
                ("mveb", "cycles"): "root gathers, rotations, balanced bottoms by rounds of partition gathers",
                ("bst", "hybrid"): "last level by cycle-leader gathers, perfect part by 2 involutions"}
        algos = ["involutions", "cycles"] + (["hybrid"] if layout == "bst" else [])
        vinfo = {}
        for algo in algos:
            vms = []
            for i in range(1 + 2):
                A.copy_(pristine)  # untimed
                r = T.permute_algorithm(layout, algo, A, b or 1, timed=True)
                if i >= 1:
                    vms.append(r)
            v_med = statistics.median(vms)
            vinfo[algo] = {"ms": round(v_med, 4), "GBps": round(bytes_step / (v_med * 1e-3) / 1e9, 1),
                           "kernels": kern[(layout, algo)], "equal_to_stream": bool(torch.equal(A, perm_ref))}
        del perm_ref
        A.copy_(pristine)
        T.permute(layout, A, b or 16)  # the library's layout again, for the queries below

    # plain B-tree / BST / mvEB queries on the permuted layout (device time)
    qinfo = None
    if args.queries and q:
        Q = data.queries_torch(pristine, q, 0.5, qseed)
        ans = torch.empty(q, dtype=torch.int64, device=dev)
        tabs = T.VebTablesDevice(n, dev, standard=layout == "veb") if layout in ("mveb", "veb") else None
        for _ in range(2):
            T.query(layout, A, Q, ans, b or 16, tables=tabs)
        qms = []
        for _ in range(3):
            qms.append(T.query(layout, A, Q, ans, b or 16, tables=tabs, timed=True))
        hits = int((ans != n).sum().item())
        qms_med = statistics.median(qms)
        # the binary-search comparator on the same queries over the sorted keys
        sans = torch.empty_like(ans)
        T.query("sorted", pristine, Q, sans)
        sms = statistics.median([T.query("sorted", pristine, Q, sans, timed=True) for _ in range(3)])
        qbytes, l2lv, nlv = query_bytes_model(layout, n, b or 16, kb)
        qps = q / (qms_med * 1e-3)
        qinfo = {"q": q, "ms": round(qms_med, 3), "queries_per_s": round(qps, 1),
                 "roofline": {"bytes_per_query": qbytes, "levels": nlv, "l2_resident_levels": l2lv,
                              "roofline_queries_per_s": round(peak * 1e9 / qbytes, 1),
                              "frac": round(qps * qbytes / (peak * 1e9), 4),
                              "model": "w + 8 + one node fetch per level below the L2-resident depth"},
                 "hits": hits, "kernel": query_kernel_name(layout, b or 16, kb)
                 + (", batch grouped by value" if query_grouped(layout, n, kb, q) else ""),
                 "binary_search_queries_per_s": round(q / (sms * 1e-3), 1),
                 "binary_search_hits": int((sans != n).sum().item())}
        if host_layout is not None:
            qinfo["parity"] = parity_module().check_answers(layout, b or 16, host_layout, Q, ans, 1 << 20, qseed)
        del Q, ans, sans
    host_layout = None

    # end to end through the C ABI with host buffers: H2D keys, permute, D2H layout
    e2e = None
    if args.e2e_steps > 0:
        host_in = torch.empty(n, dtype=pristine.dtype, pin_memory=True)
        host_in.copy_(pristine)
        host_out = torch.empty_like(host_in, pin_memory=True)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        tms = []
        for i in range(args.e2e_steps + 1):
            torch.cuda.synchronize()
            e0.record(stream)
            A.copy_(host_in, non_blocking=True)
            rc = L.tl_permute(lay, CT.c_void_p(A.data_ptr()), n, b or 16, kb, None, 0,
                              CT.c_void_p(stream.cuda_stream), None)
            if rc:
                raise T.TreeLayoutError(rc, "permute (e2e)")
            host_out.copy_(A, non_blocking=True)
            e1.record(stream)
            torch.cuda.synchronize()
            if i:  # first one warms the pinned path
                tms.append(e0.elapsed_time(e1))
        assert torch.equal(host_out[:1024].to(dev), A[:1024])
        ems = reduce_max(statistics.median(tms), world)
        e2e = {"value": round(world * bytes_step / (ems * 1e-3) / 1e9, 3), "unit": "GB/s",
               "h2d_bytes_per_step": n * kb, "d2h_bytes_per_step": n * kb, "ms_per_step": round(ems, 3)}
        del host_in, host_out

    lrn = None
    del A, pristine
    torch.cuda.empty_cache()
    if args.learned and layout == "btree" and rank == 0:
        lrn = learned_section(args, dev)

    bat = None
    if args.batched and layout == "btree" and rank == 0:
        bat = batched_section(args, dev)

    lays = None
    if args.layouts and rank == 0 and world == 1 and args.workload == DEFAULT:
        lays = layouts_section(args, L, dev, stream, local, peak, peak_kind)

    cpu = None
    if rank == 0 and world == 1 and args.cpu_sample > 0:
        cpu = cpu_reference_permute(layout, b, min(n, args.cpu_sample), kb, 5, gap_hi=gap_hi, seed=kseed)
        one = cpu_reference_permute(layout, b, min(n, args.cpu_sample // 10), kb, 3, 4.0, gap_hi=gap_hi,
                                    seed=kseed, threads=1)
        cpu["single_thread"] = {"value": one["value"], "unit": "GB/s", "cores": 1, "sample": one["sample"]}

    if rank == 0:
        line = {
            "metric": METRIC if layout == "btree" else METRIC.replace("level-order B-tree", layout),
            "value": round(value, 3), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64" if kb == 8 else "u32", "data": "synthetic",
            "config": workload_config(args, layout, b, n, kb, gap_hi, kseed, world),
            "roofline": roof,
            "parity": parity,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "first_call": first_call,
            "layouts": lays,
            "reverse": rinfo,
            "variants": vinfo,
            "queries": qinfo,
            "learned": lrn,
            "batched": bat,
            "clocks": clk,
            "gpu_launches": launches_per_step * args.steps,
        }
        print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=DEFAULT, choices=sorted(WORKLOADS))
    ap.add_argument("--n", type=int, default=0, help="override n (profiling runs)")
    ap.add_argument("--queries", type=int, default=1)
    ap.add_argument("--reverse", type=int, default=1, help="reverse permutation (layout -> sorted) section")
    ap.add_argument("--variants", type=int, default=1,
                    help="the reference's algorithm families as variants (involutions, cycle-leader, hybrid BST)")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--cpu-sample", type=int, default=50_000_000)
    ap.add_argument("--ref-n", type=int, default=0, help="reference arm keys (0: the workload's full n)")
    ap.add_argument("--learned", type=int, default=1, help="learned-vs-plain query section (B-tree workloads)")
    ap.add_argument("--learned-n", type=int, default=2**30)
    ap.add_argument("--learned-q", type=int, default=2**28)
    ap.add_argument("--learned-steps", type=int, default=1500)
    ap.add_argument("--batched", type=int, default=1, help="batched permute/query section (B-tree workloads)")
    ap.add_argument("--batch-num", type=int, default=4096)
    ap.add_argument("--batch-q", type=int, default=2**26)
    ap.add_argument("--batch-hi", type=int, default=22, help="batched arrays: log2 of the largest size (profiling runs)")
    ap.add_argument("--batch-tune", type=int, default=1, help="batched: run the autotuner first (0: default tuning)")
    ap.add_argument("--parity", type=int, default=1, help="bit-exact check against the CPU checker (untimed)")
    ap.add_argument("--layout-queries", type=int, default=1,
                    help="time 2^27 plain queries on each layout of the layouts section")
    ap.add_argument("--layouts", type=int, default=1,
                    help="every layout at 2^30-class sizes, timed and checked (default workload only)")
    ap.add_argument("--query-variant", type=int, default=0,
                    help="query kernel variant for measurements (tl_debug_set_query_variant; 0: the default)")
    ap.add_argument("--schedule", default="auto", choices=["auto", "fixed"],
                    help="B-tree/BST stream schedule: the library's choice, or the fixed-direction ones only")
    args = ap.parse_args()
    if args.impl == "reference":
        rank = int(os.environ.get("RANK", "0"))
        run_reference(args, rank)
        return
    rank, world, local = dist_setup(args.gpus)
    try:
        run_ours(args, rank, world, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
