"""Oracle parity for inputs too large for one oracle thread: the CPU oracle
runs on newline-aligned slices of an NDJSON partition in parallel and every
slice is compared with the matching bit range of the GPU's whole-partition
index and with its records' results.

NDJSON partitions are independent by the reference's own rule
(src/gpjson/engine.cpp:131-166, partition ends at file_reader.cpp:65-66):
after a complete record the string state is "outside", the depth is -1 and
the escape carry is 0, so the slice [a, b) indexes exactly as the same bytes
inside the whole partition.  The slice's string mask, leveled bitmaps and
newline offsets, shifted by a, are the partition's; its records are the
partition's records that start inside it, and their (start, end) pairs
shifted by a are the partition's results.

Test infrastructure (used by tests/ and by the parity gate of bench.py's
CPU-baseline leg): imports the oracle as the checker, never as a product
path.
"""
from __future__ import annotations

import concurrent.futures as cf
import os

import numpy as np

import oracle


def newline_slices(data: np.ndarray, target: int) -> list[tuple[int, int]]:
    """[a, b) ranges of about `target` bytes; every b but the last sits on a
    newline that belongs to neither slice (the separator)."""
    n = int(data.size)
    out, a = [], 0
    while n - a > target:
        nl = np.flatnonzero(data[a + target:min(n, a + target + (1 << 22))] == 10)
        if nl.size == 0:
            break
        b = a + target + int(nl[0])
        out.append((a, b))
        a = b + 1
    out.append((a, n))
    return out


def bit_range(words: np.ndarray, start: int, nbits: int) -> np.ndarray:
    """Bits [start, start + nbits) of a bitmap (bit b of word w = bit 64w+b)
    as words of their own, bit 0 first; bits past nbits are cleared."""
    nw = (nbits + 63) // 64
    if nw == 0:
        return np.zeros(0, np.uint64)
    w0, r = start // 64, start % 64
    src = words[w0:w0 + nw + 1]
    if src.size < nw + 1:
        src = np.concatenate([src, np.zeros(nw + 1 - src.size, np.uint64)])
    if r == 0:
        out = src[:nw].copy()
    else:
        out = (src[:nw] >> np.uint64(r)) | (src[1:nw + 1] << np.uint64(64 - r))
    tail = nbits % 64
    if tail:
        out[-1] &= np.uint64((1 << tail) - 1)
    return out


def _masked_last(words: np.ndarray, nbits: int) -> np.ndarray:
    out = words.copy()
    tail = nbits % 64
    if out.size and tail:
        out[-1] &= np.uint64((1 << tail) - 1)
    return out


def check_ndjson_partition(data: np.ndarray, levels: int, S: np.ndarray | None,
                           LB: np.ndarray | None, NL: np.ndarray | None, queries,
                           results, slice_bytes: int = 64 << 20,
                           threads: int | None = None) -> dict:
    """Compares a GPU index and query results of one NDJSON partition with the
    oracle run slice by slice.

    S: uint64[W], LB: uint64[levels * W] level-major, NL: int64[lines] (any
    may be None to skip it); queries: compiled queries (ir_bytes,
    num_result_slots); results: per query, int64 [lines, slots, 2] with
    partition offsets (-1 = none).  Raises AssertionError naming the first
    difference; returns a summary."""
    n = int(data.size)
    W = (n + 63) // 64
    slices = newline_slices(data, slice_bytes)
    threads = threads or os.cpu_count() or 1
    # first record (line) of each slice: its line index in the partition
    first_line = [0]
    for a, b in slices[:-1]:
        first_line.append(first_line[-1] + int(np.count_nonzero(data[a:b] == 10)) + 1)

    def one(k: int):
        a, b = slices[k]
        ix = oracle.OracleIndex(data[a:b], levels)
        nb = b - a
        if S is not None:
            got = bit_range(S, a, nb)
            if not np.array_equal(got, _masked_last(ix.S, nb)):
                return f"string mask differs in slice {k} [{a}, {b})"
        if LB is not None:
            for lv in range(levels):
                got = bit_range(LB[lv * W:(lv + 1) * W], a, nb)
                want = _masked_last(ix.LB[lv * ix.W:(lv + 1) * ix.W], nb)
                if not np.array_equal(got, want):
                    return f"leveled bitmap {lv} differs in slice {k} [{a}, {b})"
        r0 = first_line[k]
        if NL is not None:
            # the slice's first record starts at the separator before it
            got = NL[r0 + 1:r0 + ix.num_lines]
            if not np.array_equal(got, ix.NL[1:] + a) or (k > 0 and NL[r0] != a - 1):
                return f"newline index differs in slice {k} [{a}, {b})"
        for qi, (c, res) in enumerate(zip(queries, results)):
            want = ix.query(c.ir_bytes, c.num_result_slots)
            want = np.where(want >= 0, want + a, want)
            got = res[r0:r0 + ix.num_lines]
            if not np.array_equal(got, want):
                bad = np.argwhere((got != want).any(axis=(1, 2)))[:3].ravel()
                return (f"query {qi} results differ in slice {k} [{a}, {b}) at records "
                        f"{[int(r0 + x) for x in bad]}")
        return None

    with cf.ThreadPoolExecutor(threads) as pool:
        errors = [e for e in pool.map(one, range(len(slices))) if e]
    lines = first_line[-1] + int(np.count_nonzero(data[slices[-1][0]:] == 10)) + 1
    if NL is not None:
        assert NL.size >= lines, (NL.size, lines)
    for res in results:
        assert res.shape[0] == lines, (res.shape, lines)
    assert not errors, errors[:3]
    return {"slices": len(slices), "bytes": n, "lines": lines, "threads": threads}
