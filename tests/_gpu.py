"""Helpers for GPU tests that call the engine through its C ABI."""

import ctypes

import numpy as np
import torch

from rapids_singlecell_b200 import _lib


def lib():
    return _lib.load()


def stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def dev(a, dtype=None):
    t = torch.as_tensor(np.ascontiguousarray(a), device="cuda")
    return t if dtype is None else t.to(dtype)


def ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def rel_maxabs(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
