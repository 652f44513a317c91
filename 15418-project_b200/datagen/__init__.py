"""Seeded synthetic corpora (see gpjson_datagen.c) for benchmarks and tests.

Built with gcc on first use into datagen/_build/; host-only code.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SRC = HERE / "gpjson_datagen.c"
LIB = HERE / "_build" / "libgpjson_datagen.so"
_lib = None


def build(force: bool = False) -> Path:
    if not force and LIB.exists() and LIB.stat().st_mtime >= SRC.stat().st_mtime:
        return LIB
    LIB.parent.mkdir(exist_ok=True)
    tmp = LIB.with_suffix(".so.tmp%d" % os.getpid())
    subprocess.run(["gcc", "-O2", "-fPIC", "-shared", str(SRC), "-o", str(tmp), "-lm"],
                   check=True)
    os.replace(tmp, LIB)
    return LIB


def _l() -> C.CDLL:
    global _lib
    if _lib is None:
        build()
        l = C.CDLL(str(LIB))
        l.gdg_tweets.restype = C.c_uint64
        l.gdg_tweets.argtypes = [C.c_uint64, C.c_uint64, C.c_int, C.c_void_p, C.c_uint64]
        l.gdg_products.restype = C.c_uint64
        l.gdg_products.argtypes = [C.c_uint64, C.c_uint64, C.c_void_p, C.c_uint64]
        _lib = l
    return _lib


def tweets(seed: int, target_bytes: int, deep: bool = False, out: np.ndarray | None = None) -> np.ndarray:
    """NDJSON of post-like records (~2 KiB each) until target_bytes."""
    cap = target_bytes + 256 * 1024
    buf = out if out is not None else np.empty(cap, np.uint8)
    n = _l().gdg_tweets(seed, target_bytes, int(deep), buf.ctypes.data, buf.size)
    return buf[:n]


def products(seed: int, target_bytes: int, out: np.ndarray | None = None) -> np.ndarray:
    """One top-level array of product-like records, one element per line."""
    cap = target_bytes + 256 * 1024
    buf = out if out is not None else np.empty(cap, np.uint8)
    n = _l().gdg_products(seed, target_bytes, buf.ctypes.data, buf.size)
    return buf[:n]
