"""Binding of the learned-start B-tree query (tl_rank_model_* and
tl_query_btree_learned_u64 in include/tree_layouts.h)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import TreeLayoutError, _check, _stream_ptr, lib

H = 32
NPARAMS = H + H + H * H + H + H + 1


class RankModel(C.Structure):
    _fields_ = [("w1", C.c_float * H), ("b1", C.c_float * H), ("w2", (C.c_float * H) * H),
                ("b2", C.c_float * H), ("w3", C.c_float * H), ("b3", C.c_float), ("train_loss", C.c_float),
                ("x_lo", C.c_double), ("x_scale", C.c_double), ("n", C.c_uint64), ("log_feature", C.c_uint32),
                ("num_leaves", C.c_uint32), ("train_root", C.c_uint32), ("reserved", C.c_uint32)]

    def flat(self) -> np.ndarray:
        return np.concatenate([np.ctypeslib.as_array(self.w1), np.ctypeslib.as_array(self.b1),
                               np.ctypeslib.as_array(self.w2).reshape(-1), np.ctypeslib.as_array(self.b2),
                               np.ctypeslib.as_array(self.w3), [self.b3]]).astype(np.float64)


class TrainConfig(C.Structure):
    _fields_ = [("num_leaves", C.c_uint32), ("steps", C.c_uint32), ("batch", C.c_uint32),
                ("log_feature", C.c_uint32), ("train_root", C.c_uint32), ("monotone", C.c_uint32),
                ("lr", C.c_float), ("seed", C.c_uint64)]


LEAF_DTYPE = np.dtype({"names": ["kmin", "base", "slope", "eps_lo", "eps_hi", "empty"],
                       "formats": [np.uint64, np.uint64, np.float32, np.uint32, np.uint32, np.uint32],
                       "offsets": [0, 8, 16, 20, 24, 28], "itemsize": 32})

_bound = False


def _lib():
    global _bound
    L = lib()
    if not _bound:
        v, u64, u32 = C.c_void_p, C.c_uint64, C.c_uint32
        L.tl_rank_model_train.argtypes = [v, u64, C.POINTER(TrainConfig), C.POINTER(RankModel), v, v]
        L.tl_rank_model_predict.argtypes = [C.POINTER(RankModel), v, v, u64, v, v, v]
        L.tl_rank_model_gradient.argtypes = [C.POINTER(RankModel), v, v, u32, C.POINTER(C.c_float),
                                             C.POINTER(C.c_float), v]
        L.tl_query_btree_learned_u64.argtypes = [v, u64, u64, C.POINTER(RankModel), v, v, u64, v, v, v,
                                                 C.POINTER(C.c_float)]
        _bound = True
    return L


def train(sorted_keys, num_leaves=65536, steps=1500, batch=65536, lr=3e-3, seed=1, log_feature=True,
          train_root=True, monotone=False, stream=None):
    """Returns (RankModel, leaves tensor of num_leaves * 32 bytes on the device)."""
    import torch
    assert sorted_keys.dtype == torch.int64 and sorted_keys.is_cuda
    cfg = TrainConfig(num_leaves=num_leaves, steps=steps, batch=batch, log_feature=int(log_feature),
                      train_root=int(train_root), monotone=int(monotone), lr=lr, seed=seed)
    model = RankModel()
    leaves = torch.empty(num_leaves * LEAF_DTYPE.itemsize, dtype=torch.uint8, device=sorted_keys.device)
    rc = _lib().tl_rank_model_train(sorted_keys.data_ptr(), sorted_keys.numel(), C.byref(cfg), C.byref(model),
                                    leaves.data_ptr(), _stream_ptr(stream))
    _check(rc, "tl_rank_model_train")
    return model, leaves


def leaves_numpy(leaves) -> np.ndarray:
    return leaves.cpu().numpy().view(LEAF_DTYPE)


def predict(model, leaves, keys, stream=None):
    import torch
    rank = torch.empty(keys.numel(), dtype=torch.int64, device=keys.device)
    eps = torch.empty(keys.numel(), dtype=torch.int32, device=keys.device)
    rc = _lib().tl_rank_model_predict(C.byref(model), leaves.data_ptr(), keys.data_ptr(), keys.numel(),
                                      rank.data_ptr(), eps.data_ptr(), _stream_ptr(stream))
    _check(rc, "tl_rank_model_predict")
    return rank, eps


def gradient(model, x, y, stream=None):
    """GPU gradient (float32 kernels) of the root network's MSE on (x, y)."""
    g = (C.c_float * NPARAMS)()
    loss = C.c_float()
    rc = _lib().tl_rank_model_gradient(C.byref(model), x.data_ptr(), y.data_ptr(), x.numel(), g, C.byref(loss),
                                       _stream_ptr(stream))
    _check(rc, "tl_rank_model_gradient")
    return np.ctypeslib.as_array(g).astype(np.float64), float(loss.value)


def query(tree, model, leaves, queries, answers, b=16, stats=None, stream=None, timed=False):
    ms = C.c_float(0.0)
    rc = _lib().tl_query_btree_learned_u64(tree.data_ptr(), tree.numel(), b, C.byref(model), leaves.data_ptr(),
                                           queries.data_ptr(), queries.numel(), answers.data_ptr(),
                                           None if stats is None else stats.data_ptr(), _stream_ptr(stream),
                                           C.byref(ms) if timed else None)
    _check(rc, "tl_query_btree_learned_u64")
    return ms.value if timed else None
