"""CPU oracle for the GpJSON index + query path -- TEST INFRASTRUCTURE ONLY.

Imported only by tests/, __graft_entry__.smoke() and the CPU-baseline /
reference arm of bench.py, as the checker and the CPU baseline.  The product
library never links or calls it.  The C restatement lives in gpjson_oracle.c;
this module builds it with gcc on first use and binds it with ctypes.

Pinning: tests/test_oracle_golden.py checks it against every known-answer
vector and fixture of the reference's own index and query tests
(tests/golden/reference_kats.json, extracted by tests/golden/make_golden.py).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SRC = HERE / "gpjson_oracle.c"
BUILD = HERE / "_build"
LIB = BUILD / "liboracle.so"

_lib = None


def build(force: bool = False) -> Path:
    if not force and LIB.exists() and LIB.stat().st_mtime >= max(
            SRC.stat().st_mtime, (HERE / "gpjson_oracle.h").stat().st_mtime):
        return LIB
    BUILD.mkdir(exist_ok=True)
    tmp = LIB.with_suffix(".so.tmp%d" % os.getpid())
    subprocess.run(["gcc", "-O2", "-std=c11", "-fPIC", "-shared", str(SRC), "-o", str(tmp)],
                   check=True)
    os.replace(tmp, LIB)
    return LIB


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        build()
        l = C.CDLL(str(LIB))
        vp, u64, i32 = C.c_void_p, C.c_uint64, C.c_int
        l.orc_num_words.restype = u64
        l.orc_num_words.argtypes = [u64]
        l.orc_newline_index.restype = u64
        l.orc_newline_index.argtypes = [vp, u64, vp, u64]
        l.orc_escape_index.argtypes = [vp, u64, vp]
        l.orc_escape_index_unbounded.argtypes = [vp, u64, vp]
        l.orc_quote_index.argtypes = [vp, u64, vp, vp]
        l.orc_string_index.argtypes = [vp, u64, vp]
        l.orc_leveled_bitmap_index.argtypes = [vp, u64, vp, i32, vp]
        l.orc_build_index.restype = u64
        l.orc_build_index.argtypes = [vp, u64, i32, vp, vp, vp, vp, vp, u64]
        l.orc_query.restype = i32
        l.orc_query.argtypes = [vp, u64, vp, u64, vp, vp, u64, i32, i32, vp, u64, i32, vp]
        l.orc_query_status.restype = i32
        l.orc_query_status.argtypes = [vp, u64, vp, u64, vp, vp, u64, i32, i32, vp, u64, i32,
                                       vp, vp]
        _lib = l
    return _lib


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data if a.size else 0


def as_bytes(data) -> np.ndarray:
    if isinstance(data, np.ndarray):
        return np.ascontiguousarray(data, dtype=np.uint8)
    if isinstance(data, str):
        data = data.encode()
    return np.frombuffer(bytes(data), dtype=np.uint8)


class OracleIndex:
    """E, Q, S, LB (level-major) and NL of one partition, as numpy arrays."""

    def __init__(self, data, num_levels: int):
        b = as_bytes(data)
        n = b.size
        W = (n + 63) // 64
        self.data = b
        self.n = n
        self.W = W
        self.num_levels = num_levels
        self.E = np.zeros(W, np.uint64)
        self.Q = np.zeros(W, np.uint64)
        self.S = np.zeros(W, np.uint64)
        self.LB = np.zeros(W * num_levels, np.uint64)
        lines = int(np.count_nonzero(b == 10)) + 1
        self.NL = np.zeros(lines, np.int64)
        got = lib().orc_build_index(_ptr(b), n, num_levels, _ptr(self.E), _ptr(self.Q),
                                    _ptr(self.S), _ptr(self.LB), _ptr(self.NL), lines)
        assert got == lines
        self.num_lines = lines

    # status bits of the last query: ORC_STATUS_OVERFLOW, a record had more
    # results than slots (only the extension opcodes can); ORC_STATUS_REF_ASSERT,
    # a device assert of the reference's query kernel would fire on this input
    STATUS_OVERFLOW = 1
    STATUS_REF_ASSERT = 2
    last_status = 0

    def query(self, ir: bytes, num_results: int, base_level: int = 0) -> np.ndarray:
        """int64 [num_lines, num_results, 2], -1 = no match."""
        out = np.full(self.num_lines * num_results * 2, -1, np.int64)
        irb = np.frombuffer(ir, np.uint8) if ir else np.zeros(1, np.uint8)
        st = np.zeros(1, np.uint32)
        lib().orc_query_status(_ptr(self.data), self.n, _ptr(self.NL), self.num_lines,
                               _ptr(self.S), _ptr(self.LB), self.W, self.num_levels, base_level,
                               _ptr(irb), len(ir), num_results, _ptr(out), _ptr(st))
        self.last_status = int(st[0])
        return out.reshape(self.num_lines, num_results, 2)


def escape_unbounded(data) -> np.ndarray:
    b = as_bytes(data)
    E = np.zeros((b.size + 63) // 64, np.uint64)
    lib().orc_escape_index_unbounded(_ptr(b), b.size, _ptr(E))
    return E
