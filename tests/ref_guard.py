"""CPU pre-check of the reference's device asserts, run before any input is
handed to the reference library (oracle/_ref) on a GPU.

The reference's library is built without NDEBUG, so its device asserts are
live, and a failed device assert ends the process with the context lost.
Every input and query the parity test and the bench's reference-GPU column
send to it is checked here first, on the CPU:

* orig/uncombined/escape-index.cu:49 -- no thread's chunk of the escape
  kernel may be all backslashes.  With the harness's launch shape
  (oracle/ref/ref_dump.cpp: one 64-byte word per thread) a chunk is one
  aligned 64-byte word;
* sharemem/leveled-bitmaps-index.cu:100, 173 -- the depth never drops below
  -1; and the signed-char depth must not wrap (nesting below 128);
* query.cu:230, 265, 276, 290, 321, 334, 370, 384, 430 -- the structural
  character a search lands on is the one the reference expects, and a string
  filter only meets strings: the oracle replays every query and reports any
  such condition (ORC_STATUS_REF_ASSERT).

Test infrastructure only.
"""
from __future__ import annotations

import numpy as np

import oracle


def escape_chunks_ok(data: np.ndarray, chunk: int = 64) -> bool:
    b = oracle.as_bytes(data)
    full = b.size // chunk
    if full == 0:
        return True
    words = b[:full * chunk].reshape(full, chunk)
    return not bool((words == 0x5C).all(axis=1).any())


def depth_ok(data: np.ndarray, ix: oracle.OracleIndex | None = None) -> bool:
    b = oracle.as_bytes(data)
    if b.size == 0:
        return True
    ix = ix or oracle.OracleIndex(b, 1)
    in_string = np.unpackbits(ix.S.view(np.uint8), bitorder="little")[:b.size].astype(bool)
    opens = ((b == ord("{")) | (b == ord("["))) & ~in_string
    closes = ((b == ord("}")) | (b == ord("]"))) & ~in_string
    depth = np.cumsum(opens.astype(np.int64) - closes.astype(np.int64))  # -1 + depth after
    return bool(depth.min() >= 0) and bool(depth.max() <= 127)


def problems(data, compiled, levels: int, base_level: int = 0) -> list[str]:
    """Reasons the reference would trip a device assert on this input and
    these compiled queries (empty: safe to run)."""
    b = oracle.as_bytes(data)
    out = []
    if not escape_chunks_ok(b):
        out.append("a 64-byte word of backslashes (orig escape_index assert)")
    ix = oracle.OracleIndex(b, max(1, levels))
    if not depth_ok(b, ix):
        out.append("depth below -1 or beyond signed char (leveled bitmap asserts)")
    for c in compiled:
        ix.query(c.ir_bytes, c.num_result_slots, base_level)
        if ix.last_status & oracle.OracleIndex.STATUS_REF_ASSERT:
            out.append(f"query {c.query_text!r} reaches a query-kernel assert")
    return out
