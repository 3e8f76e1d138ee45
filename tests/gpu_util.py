"""Helpers shared by the GPU tests."""
import numpy as np
import torch


def dev(a, dtype=None):
    t = torch.as_tensor(np.ascontiguousarray(a))
    if dtype is not None:
        t = t.to(dtype)
    return t.cuda()


def host(t):
    return t.detach().cpu().numpy()


def tdtype(np_dtype):
    return torch.float32 if np.dtype(np_dtype) == np.float32 else torch.float64
