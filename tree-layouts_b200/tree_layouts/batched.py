"""Binding of the batched mode (tl_batch_* in include/tree_layouts.h): many
sorted arrays behind an int64 offset table, permuted to B-tree layouts by one
persistent kernel and queried by (key, instance) pairs."""
from __future__ import annotations

import ctypes as C
import json

import numpy as np

from . import _check, _stream_ptr, lib

NCLASS = 48
_bound = False


def _lib():
    global _bound
    L = lib()
    if not _bound:
        v, u64, u32 = C.c_void_p, C.c_uint64, C.c_uint32
        L.tl_batch_plan_create.argtypes = [v, u32, u64, u32, v, C.POINTER(v)]
        L.tl_batch_plan_destroy.argtypes = [v]
        L.tl_batch_workspace_bytes.argtypes = [v, C.POINTER(u64)]
        L.tl_batch_permute.argtypes = [v, v, v, u64, v]
        L.tl_batch_status.argtypes = [v, v, v]
        L.tl_batch_query_workspace_bytes.argtypes = [v, u64, C.POINTER(u64)]
        L.tl_batch_query.argtypes = [v, v, v, v, u64, v, v, u64, v, C.POINTER(C.c_float)]
        L.tl_batch_set_tuning.argtypes = [v, v, v, u32, u32, v, v]
        L.tl_batch_get_tuning.argtypes = [v, v, v, C.POINTER(u32), C.POINTER(u32)]
        L.tl_batch_autotune.argtypes = [v, v, v, v, v, u64, v, C.c_char_p, u64]
        L.tl_debug_batch_ordered.argtypes = [v, C.POINTER(u64), C.POINTER(u64)]
        _bound = True
    return L


class BatchPlan:
    def __init__(self, offsets, b: int = 8, key_bytes: int = 8, stream=None):
        import torch
        assert offsets.dtype == torch.int64 and offsets.is_cuda
        self.offsets = offsets
        self.num = offsets.numel() - 1
        self.key_bytes = key_bytes
        self.handle = C.c_void_p()
        _check(_lib().tl_batch_plan_create(offsets.data_ptr(), self.num, b, key_bytes, _stream_ptr(stream),
                                           C.byref(self.handle)), "tl_batch_plan_create")
        self._ws = None

    def __del__(self):
        try:
            if self.handle:
                _lib().tl_batch_plan_destroy(self.handle)
        except Exception:
            pass

    def workspace_bytes(self) -> int:
        out = C.c_uint64()
        _check(_lib().tl_batch_workspace_bytes(self.handle, C.byref(out)), "tl_batch_workspace_bytes")
        return out.value

    def workspace(self):
        import torch
        need = self.workspace_bytes()
        if self._ws is None or self._ws.numel() < need:
            self._ws = torch.empty(need, dtype=torch.uint8, device=self.offsets.device)
        return self._ws

    def permute(self, keys, workspace=None, stream=None, check=True):
        ws = self.workspace() if workspace is None else workspace
        _check(_lib().tl_batch_permute(self.handle, keys.data_ptr(), ws.data_ptr(), ws.numel(),
                                       _stream_ptr(stream)), "tl_batch_permute")
        if check:
            self.status(ws, stream)

    def status(self, workspace=None, stream=None):
        ws = self._ws if workspace is None else workspace
        _check(_lib().tl_batch_status(self.handle, ws.data_ptr(), _stream_ptr(stream)), "tl_batch_status")

    def query(self, keys, queries, inst, answers, workspace=None, stream=None, timed=False):
        import torch
        q = queries.numel()
        need = C.c_uint64()
        _check(_lib().tl_batch_query_workspace_bytes(self.handle, q, C.byref(need)), "query ws")
        ws = workspace if workspace is not None else torch.empty(need.value, dtype=torch.uint8,
                                                                  device=keys.device)
        ms = C.c_float()
        _check(_lib().tl_batch_query(self.handle, keys.data_ptr(), queries.data_ptr(), inst.data_ptr(), q,
                                     answers.data_ptr(), ws.data_ptr(), ws.numel(), _stream_ptr(stream),
                                     C.byref(ms) if timed else None), "tl_batch_query")
        return ms.value if timed else None

    def ordered(self):
        """(instances, keys) of the plan on the ordered-tile schedule."""
        i, k = C.c_uint64(), C.c_uint64()
        _check(_lib().tl_debug_batch_ordered(self.handle, C.byref(i), C.byref(k)), "tl_debug_batch_ordered")
        return i.value, k.value

    def tuning(self):
        tk = (C.c_uint32 * NCLASS)()
        pl = (C.c_uint32 * NCLASS)()
        qc, th = C.c_uint32(), C.c_uint32()
        _check(_lib().tl_batch_get_tuning(self.handle, tk, pl, C.byref(qc), C.byref(th)), "get_tuning")
        return {"tile_keys": list(tk), "pin_levels": list(pl), "query_chunk": qc.value, "threads": th.value}

    def set_tuning(self, tile_keys=None, pin_levels=None, query_chunk=0, threads=0, stream=None):
        tk = (C.c_uint32 * NCLASS)(*tile_keys) if tile_keys is not None else None
        pl = (C.c_uint32 * NCLASS)(*pin_levels) if pin_levels is not None else None
        _check(_lib().tl_batch_set_tuning(self.handle, tk, pl, query_chunk, threads, self.offsets.data_ptr(),
                                          _stream_ptr(stream)), "set_tuning")

    def autotune(self, keys, queries=None, inst=None, stream=None) -> dict:
        buf = C.create_string_buffer(8192)
        q = 0 if queries is None else queries.numel()
        _check(_lib().tl_batch_autotune(self.handle, self.offsets.data_ptr(), keys.data_ptr(),
                                        None if queries is None else queries.data_ptr(),
                                        None if inst is None else inst.data_ptr(), q, _stream_ptr(stream),
                                        buf, len(buf)), "tl_batch_autotune")
        return json.loads(buf.value.decode())


def batch_sizes_np(num: int, lo_log2: float, hi_log2: float, seed: int) -> np.ndarray:
    """Sizes log-uniform in [2^lo, 2^hi]."""
    rng = np.random.default_rng(seed)
    return np.floor(2.0 ** rng.uniform(lo_log2, hi_log2, num)).astype(np.int64)
