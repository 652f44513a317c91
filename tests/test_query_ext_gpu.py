"""Query-language extensions on the GPU vs the CPU oracle (bit-exact):
numeric filters, "..name", slices counted from the end and open slices, and
the element-count check of "[*]" and the open slices with its overflow
status (context status word, gpj_query_host error, batch error
word).  The oracle's semantics for these are pinned on CPU against an
independent JSON evaluation (tests/test_query_ext_host.py)."""
import numpy as np
import pytest
import torch

import oracle
from devmem import d2h, to_device

pytestmark = pytest.mark.gpu

EXT_QUERIES = [
    ("$..id", 64), ("$..lang", 64), ("$..text", 64), ("$.user..id", 4), ("$.entities..indices", 32),
    ("$.user.followers_count[?(@ > 50000)]", 0), ("$.user.friends_count[?(@ <= 9e2)]", 0),
    ("$.id[?(@ >= 5E17)]", 0), ("$.user[?(@.followers_count >= 10000)].screen_name", 0),
    ("$.user.statuses_count[?(@ != 35105)]", 0), ("$.place.bounding_box.coordinates[0][0][0][0][?(@ < 0)]", 0),
    ("$.entities.hashtags[*].text", 8), ("$.entities.hashtags[*].indices[1]", 8),
    ("$.entities.hashtags[-3:-1].text", 0), ("$.entities.hashtags[1:].text", 4),
    ("$.entities.hashtags[:-1].indices[0]", 6), ("$.entities.hashtags[1:-1]", 3),
]


def _gpu_query(ctx, gpj, data, comp, levels, wide=False):
    t, ptr = to_device(data)
    ix = ctx.build_index(ptr, data.size, levels)
    outs = []
    try:
        for c in comp:
            out = torch.full((ix.num_lines * c.num_result_slots * 2,), -7,
                             dtype=torch.int64 if wide else torch.int32, device="cuda")
            ctx.query(ix, c, out.data_ptr(), wide=wide)
            torch.cuda.synchronize()
            outs.append((out.cpu().numpy().astype(np.int64).reshape(ix.num_lines, -1, 2),
                         ctx.query_status()))
    finally:
        ctx.free_index(ix)
    return outs


@pytest.mark.parametrize("wide", [False, True], ids=["int32", "int64"])
def test_extension_queries_match_oracle(cuda_ctx, gpj, wide):
    from gpjson_b200 import datagen
    data = datagen.tweets(43, 6 << 20, deep=True)
    comp = [gpj.compile(q, wildcard_limit=k) for q, k in EXT_QUERIES]
    L = max(c.max_depth for c in comp)
    want_ix = oracle.OracleIndex(data, L)
    for c, (got, status) in zip(comp, _gpu_query(cuda_ctx, gpj, data, comp, L, wide)):
        want = want_ix.query(c.ir_bytes, c.num_result_slots)
        np.testing.assert_array_equal(got, want, err_msg=c.query_text)
        overflow = want_ix.last_status & oracle.OracleIndex.STATUS_OVERFLOW
        assert status == (gpj.GPJ_QUERY_OVERFLOW if overflow else 0), c.query_text
        assert (got[:, :, 0] >= 0).any(), c.query_text


def test_extension_overflow_status(cuda_ctx, gpj):
    """A "[*]" array longer than the limit and more "..name" matches than
    slots raise GPJ_QUERY_OVERFLOW; the first K results still equal the
    oracle's, and the status clears after it is read."""
    from gpjson_b200 import datagen
    data = datagen.tweets(44, 2 << 20, deep=True)
    comp = [gpj.compile("$.entities.hashtags[*].text", wildcard_limit=2),
            gpj.compile("$..id", wildcard_limit=1)]
    L = max(c.max_depth for c in comp)
    want_ix = oracle.OracleIndex(data, L)
    for c, (got, status) in zip(comp, _gpu_query(cuda_ctx, gpj, data, comp, L)):
        np.testing.assert_array_equal(got, want_ix.query(c.ir_bytes, c.num_result_slots))
        assert want_ix.last_status & oracle.OracleIndex.STATUS_OVERFLOW
        assert status == gpj.GPJ_QUERY_OVERFLOW
    assert cuda_ctx.query_status() == 0


def test_query_host_reports_overflow(cuda_ctx, gpj):
    from gpjson_b200 import datagen
    data = datagen.tweets(45, 1 << 20)
    lines = data.tobytes().count(b"\n") + 1
    host_in = torch.from_numpy(data.copy()).pin_memory()
    for k, fails in ((2, True), (8, False)):
        c = gpj.compile("$.entities.hashtags[*].text", wildcard_limit=k)
        out = torch.empty(lines * c.num_result_slots * 2, dtype=torch.int32).pin_memory()
        call = lambda: cuda_ctx.query_host(host_in.data_ptr(), data.size, c.max_depth, [c],
                                           [out.data_ptr()], [out.numel()])
        if fails:
            with pytest.raises(gpj.CapacityError, match="more results than result slots"):
                call()
        else:
            assert call() == lines
        want = oracle.OracleIndex(data, c.max_depth).query(c.ir_bytes, c.num_result_slots)
        np.testing.assert_array_equal(out.numpy().astype(np.int64).reshape(lines, -1, 2), want)


def test_batch_extension_queries_and_overflow(gpj):
    from gpjson_b200 import datagen
    files = [bytes(datagen.tweets(900 + i, 40_000 + 7_000 * i, deep=True)) for i in range(12)]
    for k, overflow in ((8, False), (2, True)):
        comp = [gpj.compile("$.entities.hashtags[*].text", wildcard_limit=k),
                gpj.compile("$.user[?(@.followers_count >= 10000)].screen_name")]
        queries = [(c, 0, max(x.max_depth for x in comp)) for c in comp]
        buf, offsets = gpj.pack_files(files)
        dev = torch.from_numpy(buf).cuda()
        table = [(o, len(d), i % 2) for i, (o, d) in enumerate(zip(offsets, files))]
        with gpj.Batch(dev.data_ptr(), buf.size, table, queries) as b:
            b.run()
            torch.cuda.synchronize()
            v = b.view()
            info = d2h(v.d_file_info, v.num_files * gpj.FILE_INFO_WORDS, np.uint64).reshape(-1, 8)
            err = int(d2h(v.d_totals, 4, np.uint64)[3])
            R = d2h(v.d_results, v.result_ints, np.int32)
            assert bool(err & gpj.GPJ_QUERY_OVERFLOW) == overflow and not err & 7
            h_in = torch.from_numpy(buf).pin_memory()
            if overflow:
                with pytest.raises(gpj.CapacityError):
                    b.run_host(h_in.data_ptr())
            else:
                b.run_host(h_in.data_ptr())
        for f, d in enumerate(files):
            c, base, lv = queries[table[f][2]]
            lines, out_off = int(info[f, 0]), int(info[f, 3])
            got = R[out_off:out_off + lines * c.num_result_slots * 2].astype(np.int64)
            want = oracle.OracleIndex(d, lv).query(c.ir_bytes, c.num_result_slots, base)
            np.testing.assert_array_equal(got.reshape(lines, -1, 2), want, err_msg=str(f))


def test_slices_on_arrays_match_oracle(cuda_ctx, gpj):
    """Every slice form over arrays of 0-11 elements, empty arrays included."""
    from test_query_ext_host import SLICE_CASES, array_records
    data = np.frombuffer(array_records(11, 4000), np.uint8).copy()
    comp = [gpj.compile(q, wildcard_limit=k) for q, _, _, _, _, k in SLICE_CASES]
    L = max(c.max_depth for c in comp)
    want_ix = oracle.OracleIndex(data, L)
    for c, (got, status) in zip(comp, _gpu_query(cuda_ctx, gpj, data, comp, L)):
        want = want_ix.query(c.ir_bytes, c.num_result_slots)
        np.testing.assert_array_equal(got, want, err_msg=c.query_text)
        overflow = want_ix.last_status & oracle.OracleIndex.STATUS_OVERFLOW
        assert status == (gpj.GPJ_QUERY_OVERFLOW if overflow else 0), c.query_text
        assert (got[:, :, 0] >= 0).sum() > 100, c.query_text
