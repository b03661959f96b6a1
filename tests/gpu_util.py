"""Host <-> device helpers for the GPU tests (4-byte keys travel as int32 bit patterns)."""
import numpy as np


def to_dev(a: np.ndarray):
    import torch
    if a.dtype == np.uint64:
        return torch.from_numpy(a.view(np.int64).copy()).cuda()
    if a.dtype == np.uint32:
        return torch.from_numpy(a.view(np.int32).copy()).cuda()
    raise TypeError(a.dtype)


def from_dev(t) -> np.ndarray:
    a = t.cpu().numpy()
    return a.view(np.uint64) if a.dtype == np.int64 else a.view(np.uint32)
