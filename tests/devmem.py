"""Device-memory helpers for the GPU tests: host<->device copies of raw
device pointers returned by the C ABI (through the CUDA runtime that torch
already loaded)."""
from __future__ import annotations

import ctypes as C
import glob
import os

import numpy as np
import torch

_rt = None


def cudart() -> C.CDLL:
    global _rt
    if _rt is None:
        torch.cuda.init()
        cands = glob.glob(os.path.join(os.path.dirname(torch.__file__), "..", "nvidia",
                                       "cuda_runtime", "lib", "libcudart.so*"))
        cands += ["libcudart.so.12", "/usr/local/cuda/lib64/libcudart.so"]
        for c in cands:
            try:
                _rt = C.CDLL(c)
                break
            except OSError:
                continue
        _rt.cudaMemcpy.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int]
        _rt.cudaMemcpy.restype = C.c_int
        _rt.cudaMemset.argtypes = [C.c_void_p, C.c_int, C.c_size_t]
        _rt.cudaMemset.restype = C.c_int
    return _rt


def d2h(ptr: int, count: int, dtype) -> np.ndarray:
    out = np.zeros(count, dtype)
    if count:
        rc = cudart().cudaMemcpy(out.ctypes.data, C.c_void_p(ptr), out.nbytes, 2)
        assert rc == 0, rc
    return out


def to_device(data: np.ndarray, offset: int = 0) -> tuple[torch.Tensor, int]:
    """Copies bytes to a fresh device buffer at `offset`; returns (tensor, ptr)."""
    t = torch.zeros(data.size + offset + 256, dtype=torch.uint8, device="cuda")
    if data.size:
        src = data if data.flags.writeable else data.copy()
        t[offset:offset + data.size] = torch.from_numpy(np.ascontiguousarray(src))
    return t, t.data_ptr() + offset


def index_arrays(ix) -> dict:
    W, L = ix.num_words, ix.num_levels
    out = {
        "S": d2h(ix.d_string, W, np.uint64),
        "LB": d2h(ix.d_leveled, W * L, np.uint64),
        "NL": d2h(ix.d_newline, ix.num_lines, np.int64),
    }
    if ix.d_escape:
        out["E"] = d2h(ix.d_escape, W, np.uint64)
        out["Q"] = d2h(ix.d_quote, W, np.uint64)
    return out
