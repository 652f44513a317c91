"""Parity at the measured sizes: the index and query outputs of the workloads
the benchmark times, at their full sizes, against the CPU oracle.

* the 1 GiB single top-level array of product records (one element per
  line), $[*].categoryPath[1:3].id: escape, quote and string carries and
  depth sums cross 32,769 tiles of one file; every bitmap, the newline index
  and the results are compared with the oracle run over the whole file;
* the 4 GiB NDJSON of post records as ONE partition (above 2^31 bytes, so
  results are int64 and offsets really exceed int32), four queries over one
  index: compared with the oracle run on newline-aligned slices in parallel
  (NDJSON partitions are independent, src/gpjson/engine.cpp:131-166), bit
  ranges of the whole-partition bitmaps realigned per slice;
* the whole 10,000-file batch (8 GiB) that the default benchmark line times:
  every file's string mask, leveled bitmaps, newline index and results.

Integer/bit outputs: bit-exact, no tolerance.
"""
import concurrent.futures as cf
import os
import sys
from pathlib import Path

import numpy as np
import pytest
import torch

import oracle
import parity_slices as ps
from devmem import d2h, index_arrays

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parent.parent


def _host_memory_ok(need_gb: float) -> bool:
    try:
        import psutil
        return psutil.virtual_memory().available > need_gb * 1e9
    except Exception:
        return True


def _device_copy(data: np.ndarray) -> torch.Tensor:
    t = torch.empty(data.size + 256, dtype=torch.uint8, device="cuda")
    t[:data.size].copy_(torch.from_numpy(data))
    return t


def test_c1_full_1gib_array(cuda_ctx, gpj):
    from gpjson_b200 import datagen
    data = datagen.products(1, 1 << 30)
    c = gpj.compile("$.categoryPath[1:3].id")
    L = c.max_depth + 1  # "$[*]": query level 0 is bitmap level 1
    t = _device_copy(data)
    ix = cuda_ctx.build_index(t.data_ptr(), data.size, L, gpj.GPJ_INDEX_EMIT_ESCAPE_QUOTE)
    try:
        got = index_arrays(ix)
        out = torch.full((ix.num_lines * c.num_result_slots * 2,), -7, dtype=torch.int32,
                         device="cuda")
        cuda_ctx.query(ix, c, out.data_ptr(), base_level=1)
        torch.cuda.synchronize()
        res = out.cpu().numpy().astype(np.int64).reshape(ix.num_lines, -1, 2)
        lines = ix.num_lines
    finally:
        cuda_ctx.free_index(ix)
    del t
    want = oracle.OracleIndex(data, L)
    assert lines == want.num_lines
    for k in ("E", "Q", "S", "LB", "NL"):
        np.testing.assert_array_equal(got[k], getattr(want, k), err_msg=k)
    np.testing.assert_array_equal(res, want.query(c.ir_bytes, c.num_result_slots, 1))
    assert data.size > (1 << 30) and (res[:, :, 0] >= 0).sum() > 500_000


C2_QUERIES = ["$.user.lang", "$.entities.hashtags[*].text", "$.place.country_code",
              "$.retweeted_status.user.id"]


def test_c2_full_4gib_one_partition_int64(cuda_ctx, gpj):
    if not _host_memory_ok(16):
        pytest.skip("needs about 16 GB of free host memory")
    from gpjson_b200 import datagen
    data = datagen.tweets(2, 4 << 30, deep=True)
    n = int(data.size)
    assert n > (1 << 31)
    comp = [gpj.compile(q, wildcard_limit=8) for q in C2_QUERIES]
    L = max(c.max_depth for c in comp)
    t = _device_copy(data)
    ix = cuda_ctx.build_index(t.data_ptr(), n, L)
    results = []
    try:
        got = index_arrays(ix)
        for c in comp:
            out = torch.full((ix.num_lines * c.num_result_slots * 2,), -7, dtype=torch.int64,
                             device="cuda")
            cuda_ctx.query(ix, c, out.data_ptr(), wide=True)
            torch.cuda.synchronize()
            results.append(out.cpu().numpy().reshape(ix.num_lines, c.num_result_slots, 2))
            del out
    finally:
        cuda_ctx.free_index(ix)
    del t
    torch.cuda.empty_cache()
    info = ps.check_ndjson_partition(data, L, got["S"], got["LB"], got["NL"], comp, results)
    assert info["lines"] == int(np.count_nonzero(data == 10)) + 1
    # offsets past int32: the results really need the int64 path
    last = results[0][results[0][:, 0, 0] >= 0]
    assert last[-1, 0, 0] > (1 << 31) and last[-1, 0, 1] <= n


def test_c3_full_batch_every_file(gpj):
    if not torch.cuda.is_available():
        pytest.skip("CUDA device required")
    if not _host_memory_ok(40):
        pytest.skip("needs about 40 GB of free host memory")
    sys.path.insert(0, str(ROOT))
    import bench
    files = bench.c3_files(gpj)  # the default benchmark line's 10,000 files
    comp = bench.compile_all(gpj, bench.C3_QUERIES)
    queries = [(c, base, c.max_depth + base) for c, base in comp]
    buf, offsets = gpj.pack_files([d for d, _ in files])
    kinds = [k for _, k in files]
    sizes = [len(d) for d, _ in files]
    del files
    dev = torch.from_numpy(buf).cuda()
    table = [(o, n, k) for o, n, k in zip(offsets, sizes, kinds)]
    with gpj.Batch(dev.data_ptr(), buf.size, table, queries, flags=gpj.GPJ_BATCH_AUTOTUNE) as b:
        b.run()
        b.run()  # a replay of the captured graph: what the benchmark times
        torch.cuda.synchronize()
        v = b.view()
        info = d2h(v.d_file_info, v.num_files * gpj.FILE_INFO_WORDS, np.uint64).reshape(-1, 8)
        assert int(d2h(v.d_totals, 4, np.uint64)[3]) == 0
        S = d2h(v.d_string, v.string_words, np.uint64)
        LB = d2h(v.d_leveled, v.leveled_words, np.uint64)
        NL = d2h(v.d_newline, v.newline_slots, np.int64)
        R = d2h(v.d_results, v.result_ints, np.int32)
        layout = [b.file_layout(f) for f in range(len(table))]
    del dev
    torch.cuda.empty_cache()

    def one(f):
        o, n, k = table[f]
        c, base, lv = queries[k]
        d = buf[o:o + n]
        want = oracle.OracleIndex(d, lv)
        lines, nl_off, _, out_off = (int(x) for x in info[f, :4])
        s_off, lb_off, _ = layout[f]
        W = (n + 63) // 64
        slots = c.num_result_slots
        got = R[out_off:out_off + lines * slots * 2].astype(np.int64).reshape(lines, slots, 2)
        ok = (lines == want.num_lines
              and np.array_equal(NL[nl_off:nl_off + lines], want.NL)
              and np.array_equal(S[s_off:s_off + W], want.S)
              and np.array_equal(LB[lb_off:lb_off + W * lv], want.LB)
              and np.array_equal(got, want.query(c.ir_bytes, slots, base) if n else got * 0 - 1))
        return None if ok else f

    with cf.ThreadPoolExecutor(os.cpu_count() or 4) as pool:
        bad = [f for f in pool.map(one, range(len(table))) if f is not None]
    assert not bad, f"{len(bad)} files differ from the oracle, first {bad[:5]}"
    assert len(table) == 10_000 and sum(sizes) > 8e9
