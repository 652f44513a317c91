"""Batched path (many files, one captured launch chain) vs the CPU oracle run
file by file: every file's string mask, leveled bitmaps, newline index and
query results must be bit-identical."""
import random

import numpy as np
import pytest
import torch

import oracle
from devmem import d2h

pytestmark = pytest.mark.gpu

QUERIES = [("$.user.lang", 0), ("$.categoryPath[1:3].id", 1), ("$.a[0:3].b", 0)]


def _files(seed: int, count: int):
    from gpjson_b200 import datagen
    rng = random.Random(seed)
    out = []
    for i in range(count):
        kind = i % 3
        size = rng.choice([0, 1, 50, 127, 128, 129, 1000, 5000, 40000, 70000, 250000])
        if kind == 0:
            data = bytes(datagen.tweets(seed * 1000 + i, max(size, 1)))[:max(size * 3, 2000)]
        elif kind == 1:
            data = bytes(datagen.products(seed * 1000 + i, max(size, 3)))
        else:
            data = bytes(rng.choices(b'{}[]:,"\\\n ab', weights=[6, 6, 3, 3, 5, 5, 8, 1, 2, 3, 8, 8],
                                     k=size))
        if size == 0:
            data = b""
        out.append((data, kind))
    return out


def _run_batch(gpj, files, flags, runs=1):
    comp = [(gpj.compile(q), base) for q, base in QUERIES]
    queries = [(c, base, c.max_depth + base) for c, base in comp]
    buf, offsets = gpj.pack_files([d for d, _ in files])
    dev = torch.from_numpy(buf).cuda()
    table = [(o, len(d), k) for o, (d, k) in zip(offsets, files)]
    with gpj.Batch(dev.data_ptr(), buf.size, table, queries, flags=flags) as b:
        for _ in range(runs):
            b.run()
        torch.cuda.synchronize()
        v = b.view()
        info = d2h(v.d_file_info, v.num_files * gpj.FILE_INFO_WORDS, np.uint64).reshape(-1, 8)
        totals = d2h(v.d_totals, 4, np.uint64)
        out = {
            "info": info, "totals": totals, "view": (v.num_records, v.result_ints, v.uses_graph,
                                                     v.index_threads, v.query_block,
                                                     v.index_variant),
            "S": d2h(v.d_string, v.string_words, np.uint64),
            "LB": d2h(v.d_leveled, v.leveled_words, np.uint64),
            "NL": d2h(v.d_newline, v.newline_slots, np.int64),
            "R": d2h(v.d_results, v.result_ints, np.int32),
            "layout": [b.file_layout(f) for f in range(len(files))],
        }
    return comp, queries, out


def _check(files, comp, queries, got):
    assert got["totals"][3] == 0
    for f, (data, kind) in enumerate(files):
        c, base, levels = queries[kind]
        row = got["info"][f]
        want = oracle.OracleIndex(data, levels)
        lines, nl_off, rec_off, out_off = (int(x) for x in row[:4])
        assert lines == want.num_lines, f
        np.testing.assert_array_equal(got["NL"][nl_off:nl_off + lines], want.NL, err_msg=str(f))
        s_off, lb_off, lv = got["layout"][f]
        W = (len(data) + 63) // 64
        np.testing.assert_array_equal(got["S"][s_off:s_off + W], want.S, err_msg=str(f))
        np.testing.assert_array_equal(got["LB"][lb_off:lb_off + W * lv], want.LB, err_msg=str(f))
        slots = c.num_result_slots
        res = got["R"][out_off:out_off + lines * slots * 2].astype(np.int64).reshape(lines, slots, 2)
        if len(data):
            np.testing.assert_array_equal(res, want.query(c.ir_bytes, slots, base), err_msg=str(f))
        else:
            assert (res == -1).all()


def test_batch_matches_oracle_per_file(gpj):
    if not torch.cuda.is_available():
        pytest.skip("CUDA device required")
    files = _files(1, 60)
    comp, queries, got = _run_batch(gpj, files, flags=0, runs=2)
    assert got["view"][2] == 1  # graph captured
    _check(files, comp, queries, got)


def test_batch_without_graph_and_autotuned(gpj):
    if not torch.cuda.is_available():
        pytest.skip("CUDA device required")
    files = _files(2, 40)
    comp, queries, a = _run_batch(gpj, files, flags=gpj.GPJ_BATCH_NO_GRAPH)
    _, _, b = _run_batch(gpj, files, flags=gpj.GPJ_BATCH_AUTOTUNE)
    _check(files, comp, queries, a)
    _check(files, comp, queries, b)
    assert b["view"][3] in (128, 256) and b["view"][4] in (128, 256)


@pytest.mark.parametrize("variant", [0, 1, 2, 3])
def test_batch_index_variants(gpj, variant):
    """Every indexer variant the batch autotuner chooses among (leveled walk
    from a per-warp list or per lane, look-back rounds of 32 or 64
    descriptors) gives the oracle's outputs file by file; a 3 MiB file makes
    the look-back cross more than 64 tiles."""
    if not torch.cuda.is_available():
        pytest.skip("CUDA device required")
    from gpjson_b200 import datagen
    flags = ((gpj.GPJ_BATCH_INDEX_LANE_WALK if variant & 1 else 0) |
             (gpj.GPJ_BATCH_INDEX_WIDE_LOOKBACK if variant & 2 else 0))
    files = _files(10 + variant, 30) + [(bytes(datagen.products(77, 3 << 20)), 1)]
    comp, queries, got = _run_batch(gpj, files, flags=flags)
    assert got["view"][5] == variant
    _check(files, comp, queries, got)


def test_batch_single_large_file_equals_plain_build(gpj, cuda_ctx):
    from gpjson_b200 import datagen
    data = datagen.products(5, 3 << 20)
    files = [(bytes(data), 1)]
    comp, queries, got = _run_batch(gpj, files, flags=0)
    _check(files, comp, queries, got)


def test_plain_per_file_launches_match_batch(gpj):
    if not torch.cuda.is_available():
        pytest.skip("CUDA device required")
    files = _files(3, 30)
    comp = [(gpj.compile(q), base) for q, base in QUERIES]
    queries = [(c, base, c.max_depth + base) for c, base in comp]
    buf, offsets = gpj.pack_files([d for d, _ in files])
    dev = torch.from_numpy(buf).cuda()
    table = [(o, len(d), k) for o, (d, k) in zip(offsets, files)]
    with gpj.Batch(dev.data_ptr(), buf.size, table, queries) as b:
        v = b.view()
        b.run()
        torch.cuda.synchronize()
        want = [d2h(p, n, t) for p, n, t in [(v.d_results, v.result_ints, np.int32),
                                              (v.d_newline, v.newline_slots, np.int64),
                                              (v.d_string, v.string_words, np.uint64),
                                              (v.d_leveled, v.leveled_words, np.uint64)]]
        for p, n, sz in [(v.d_results, v.result_ints, 4), (v.d_newline, v.newline_slots, 8),
                         (v.d_string, v.string_words, 8), (v.d_leveled, v.leveled_words, 8)]:
            from devmem import cudart
            cudart().cudaMemset(p, 0x5A, n * sz)
        b.run_per_file()
        torch.cuda.synchronize()
        got = [d2h(p, n, t) for p, n, t in [(v.d_results, v.result_ints, np.int32),
                                             (v.d_newline, v.newline_slots, np.int64),
                                             (v.d_string, v.string_words, np.uint64),
                                             (v.d_leveled, v.leveled_words, np.uint64)]]
    for g, w in zip(got, want):
        np.testing.assert_array_equal(g, w)


def test_batch_run_host_in_pieces(gpj):
    """gpj_batch_run_host on more than one 32 MiB piece: the packed files are
    copied piece by piece and each piece is indexed as soon as it lands.  The
    device buffer starts out as garbage, so a piece indexed before its bytes
    arrived would show; every file must still equal the oracle."""
    if not torch.cuda.is_available():
        pytest.skip("CUDA device required")
    from gpjson_b200 import datagen
    files = _files(4, 30)
    files.insert(7, (bytes(datagen.tweets(41, 40 << 20)), 0))
    files.insert(15, (bytes(datagen.products(42, 20 << 20)), 1))
    files += [(bytes(datagen.tweets(43 + i, 300000)), 0) for i in range(20)]
    comp = [(gpj.compile(q), base) for q, base in QUERIES]
    queries = [(c, base, c.max_depth + base) for c, base in comp]
    buf, offsets = gpj.pack_files([d for d, _ in files])
    assert buf.size > (64 << 20)
    dev = torch.from_numpy(buf).cuda()  # creation sizes the outputs on the real bytes
    host = torch.from_numpy(buf).pin_memory()
    table = [(o, len(d), k) for o, (d, k) in zip(offsets, files)]
    with gpj.Batch(dev.data_ptr(), buf.size, table, queries) as b:
        v = b.view()
        dev.fill_(ord("{"))
        torch.cuda.synchronize()
        results = torch.empty(max(1, v.result_ints), dtype=torch.int32).pin_memory()
        info = torch.empty(v.num_files * gpj.FILE_INFO_WORDS, dtype=torch.int64).pin_memory()
        b.run_host(host.data_ptr(), results.data_ptr(), info.data_ptr())
        got = {
            "info": info.numpy().view(np.uint64).reshape(-1, 8),
            "totals": d2h(v.d_totals, 4, np.uint64),
            "S": d2h(v.d_string, v.string_words, np.uint64),
            "LB": d2h(v.d_leveled, v.leveled_words, np.uint64),
            "NL": d2h(v.d_newline, v.newline_slots, np.int64),
            "R": results.numpy()[:v.result_ints],
            "layout": [b.file_layout(f) for f in range(len(files))],
        }
    assert torch.equal(dev.cpu(), torch.from_numpy(buf))
    _check(files, comp, queries, got)
