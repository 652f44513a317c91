"""Query kernel on the GPU vs the CPU oracle: bit-exact (start, end) result
arrays, plus the reference's own query known answers."""
import json
import random
from pathlib import Path

import numpy as np
import pytest
import torch

import oracle
from devmem import to_device

pytestmark = pytest.mark.gpu
KATS = json.loads((Path(__file__).parent / "golden" / "reference_kats.json").read_text())

TWEET_QUERIES = [
    "$.user.lang", "$.lang", '$.user.lang[?(@ == "nl")]', '$.user.lang[?(@ == "en")]',
    "$.entities.hashtags[0:8].text", "$.place.country_code", "$.retweeted_status.user.id",
    "$.entities.hashtags[-1].text", "$.entities.hashtags[-2:]", "$.coordinates.coordinates[1]",
    "$['user']['name']", "$.entities.urls[0,1].url", "$.place.bounding_box.coordinates[0][2][1]",
    "$.retweeted_status.entities.hashtags[1].indices[0]", "$.user", "$.nonexistent.key",
]


def run_gpu(ctx, gpj, data, queries, wide=False, levels=None):
    b = oracle.as_bytes(data)
    comp = [gpj.compile(q) for q in queries]
    L = levels or max(c.max_depth for c in comp)
    t, ptr = to_device(b)
    ix = ctx.build_index(ptr, b.size, L)
    outs = []
    try:
        for c in comp:
            dt = torch.int64 if wide else torch.int32
            out = torch.full((max(1, ix.num_lines * c.num_result_slots * 2),), -7, dtype=dt,
                             device="cuda")
            ctx.query(ix, c, out.data_ptr(), wide=wide)
            torch.cuda.synchronize()
            outs.append(out.cpu().numpy()[: ix.num_lines * c.num_result_slots * 2]
                        .reshape(ix.num_lines, c.num_result_slots, 2))
    finally:
        ctx.free_index(ix)
    return comp, L, outs


def check_against_oracle(ctx, gpj, data, queries, wide=False):
    comp, L, outs = run_gpu(ctx, gpj, data, queries, wide)
    want_ix = oracle.OracleIndex(data, L)
    for c, got in zip(comp, outs):
        want = want_ix.query(c.ir_bytes, c.num_result_slots)
        if b := oracle.as_bytes(data).size:
            np.testing.assert_array_equal(got.astype(np.int64), want, err_msg=c.query_text)
    return comp, outs


def texts(data: bytes, res):
    return [[data[s:e].decode() for s, e in line if s >= 0] for line in res]


def test_query_executor_kats(cuda_ctx, gpj):
    k = KATS["query_executor"]
    data = k["json_text"].encode()
    comp, outs = check_against_oracle(cuda_ctx, gpj, data, k["queries"])
    for qi, expected in k["expected"].items():
        assert texts(data, outs[int(qi)]) == [[expected]]
    assert texts(data, outs[k["queries"].index(k["unmatched_query"])]) == [[]]


def test_engine_kats(cuda_ctx, gpj):
    k = KATS["engine"]
    data = k["contents"].encode()
    comp, outs = check_against_oracle(cuda_ctx, gpj, data, k["queries"])
    for q, line, expected in k["expected"]:
        assert texts(data, outs[q])[line] == [expected]


@pytest.mark.parametrize("wide", [False, True], ids=["int32", "int64"])
def test_tweets_many_queries(cuda_ctx, gpj, wide):
    from gpjson_b200 import datagen
    data = datagen.tweets(11, 8 << 20)
    check_against_oracle(cuda_ctx, gpj, data, TWEET_QUERIES, wide)


def test_products_lines(cuda_ctx, gpj):
    from gpjson_b200 import datagen
    data = datagen.products(2, 8 << 20)
    check_against_oracle(cuda_ctx, gpj, data, ["$.categoryPath[1:3].id", "$.offers[0].type[1]",
                                               "$.shipping.ground", "$.sku"])


@pytest.mark.parametrize("seed", range(6))
def test_garbage_input_matches_oracle(cuda_ctx, gpj, seed):
    rng = random.Random(seed)
    alphabet = b'{}[]:,"\\\n ab'
    data = bytes(rng.choices(alphabet, weights=[6, 6, 3, 3, 5, 5, 8, 1, 2, 3, 8, 8], k=20000))
    check_against_oracle(cuda_ctx, gpj, data, ["$.a", "$.a.b", "$.b[1]", "$.a[-1]",
                                               '$.a[?(@ == "b")]', "$.a[0:3].b"])


def test_query_host_end_to_end(cuda_ctx, gpj):
    from gpjson_b200 import datagen
    data = datagen.tweets(4, 2 << 20)
    comp = [gpj.compile(q) for q in ["$.user.lang", "$.entities.hashtags[0:8].text"]]
    L = max(c.max_depth for c in comp)
    lines = data.tobytes().count(b"\n") + 1
    host_in = torch.from_numpy(data.copy()).pin_memory()
    outs = [torch.empty(lines * c.num_result_slots * 2, dtype=torch.int32).pin_memory()
            for c in comp]
    got_lines = cuda_ctx.query_host(host_in.data_ptr(), data.size, L, comp,
                                    [o.data_ptr() for o in outs], [o.numel() for o in outs])
    assert got_lines == lines
    want = oracle.OracleIndex(data, L)
    for c, o in zip(comp, outs):
        np.testing.assert_array_equal(o.numpy().astype(np.int64).reshape(lines, -1, 2),
                                      want.query(c.ir_bytes, c.num_result_slots))


def _pieces_input():
    """About 73 MiB of post records with, at each 32 MiB boundary, a record
    whose string holds a backslash run that ends right at the boundary, so
    that the escape, string and depth carries cross the piece boundaries."""
    from gpjson_b200 import datagen
    piece = 32 << 20
    out = bytearray()
    for k, boundary in enumerate((piece, 2 * piece)):
        rec = (b'{"a":"' + b"q" * 18 + b"\\\\\\" + b'"' + b"z" * 30 +
               b'","user":{"lang":"b%d"}}\n' % k)
        start = boundary - 27  # the quote after the three backslashes lands on the boundary
        seg = datagen.tweets(20 + k, start - len(out) - 4096).tobytes()
        seg = seg[: seg.rfind(b"\n") + 1]
        out += seg
        out += b" " * (start - len(out) - 1) + b"\n"
        assert len(out) == start
        out += rec
    out += datagen.tweets(30, 9 << 20).tobytes()
    return np.frombuffer(bytes(out), np.uint8).copy()


def test_query_host_pieces(cuda_ctx, gpj):
    """Host inputs of more than one 32 MiB piece are copied and indexed piece
    by piece (the index of a piece overlaps the copy of the next); results
    equal the oracle's on the whole input."""
    data = _pieces_input()
    assert data.size > (64 << 20) + (8 << 20)
    comp = [gpj.compile(q) for q in ["$.user.lang", "$.a", "$.entities.hashtags[0:8].text"]]
    L = max(c.max_depth for c in comp)
    lines = data.tobytes().count(b"\n") + 1
    host_in = torch.from_numpy(data).pin_memory()
    outs = [torch.empty(lines * c.num_result_slots * 2, dtype=torch.int32).pin_memory()
            for c in comp]
    got_lines = cuda_ctx.query_host(host_in.data_ptr(), data.size, L, comp,
                                    [o.data_ptr() for o in outs], [o.numel() for o in outs])
    assert got_lines == lines
    want = oracle.OracleIndex(data, L)
    texts_seen = set()
    for c, o in zip(comp, outs):
        got = o.numpy().astype(np.int64).reshape(lines, -1, 2)
        np.testing.assert_array_equal(got, want.query(c.ir_bytes, c.num_result_slots),
                                      err_msg=c.query_text)
        if c.query_text == "$.user.lang":
            b = data.tobytes()
            texts_seen = {b[s:e] for s, e in got[:, 0] if s >= 0}
    assert b'"b0"' in texts_seen and b'"b1"' in texts_seen


@pytest.mark.parametrize("query", ["$.categoryPath[1:3].id", "$.offers[0].type[1]", "$.sku",
                                   "$.categoryPath[*].name"])
def test_array_element_records(cuda_ctx, gpj, query):
    """$[*].X: the elements of the top-level array are the records (query
    level 0 = bitmap level 1)."""
    from gpjson_b200 import datagen
    data = datagen.products(2, 8 << 20)
    c = gpj.compile(query, wildcard_limit=6)
    L = c.max_depth + 1
    t, ptr = to_device(data)
    ix = cuda_ctx.build_index(ptr, data.size, L)
    try:
        out = torch.full((ix.num_lines * c.num_result_slots * 2,), -7, dtype=torch.int32,
                         device="cuda")
        cuda_ctx.query(ix, c, out.data_ptr(), base_level=1)
        torch.cuda.synchronize()
        got = out.cpu().numpy().astype(np.int64).reshape(ix.num_lines, -1, 2)
    finally:
        cuda_ctx.free_index(ix)
    want = oracle.OracleIndex(data, L).query(c.ir_bytes, c.num_result_slots, 1)
    np.testing.assert_array_equal(got, want)
    assert (got[1:-1, 0, 0] >= 0).mean() > 0.5  # most elements match slot 0


def test_copy_to_device_pageable_and_pinned(cuda_ctx, gpj):
    """gpj_copy_to_device: a pageable source (several 32 MiB staging chunks,
    an unaligned start) and a pinned one arrive bit for bit."""
    rng = np.random.default_rng(5)
    src = rng.integers(0, 256, (100 << 20) + 4099, dtype=np.uint8)
    view = src[3:]  # pageable, unaligned
    dst = torch.zeros(view.size + 16, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    cuda_ctx.copy_to_device(dst.data_ptr() + 1, view.ctypes.data, view.size, stream)
    torch.cuda.synchronize()
    got = dst.cpu().numpy()
    assert np.array_equal(got[1:1 + view.size], view) and got[0] == 0 and got[-1] == 0
    pinned = torch.from_numpy(src[: 5 << 20].copy()).pin_memory()
    dst2 = torch.zeros(pinned.numel(), dtype=torch.uint8, device="cuda")
    cuda_ctx.copy_to_device(dst2.data_ptr(), pinned.data_ptr(), pinned.numel(), stream)
    torch.cuda.synchronize()
    assert torch.equal(dst2.cpu(), pinned)


def test_query_host_pageable_pieces(cuda_ctx, gpj):
    """A pageable host input of more than one piece goes through the pinned
    staging ring piece by piece; results equal the oracle's."""
    data = _pieces_input()  # a numpy array: pageable memory
    comp = [gpj.compile(q) for q in ["$.user.lang", "$.a"]]
    L = max(c.max_depth for c in comp)
    lines = data.tobytes().count(b"\n") + 1
    outs = [np.full(lines * c.num_result_slots * 2, -9, np.int32) for c in comp]
    got_lines = cuda_ctx.query_host(data.ctypes.data, data.size, L, comp,
                                    [o.ctypes.data for o in outs], [o.size for o in outs])
    assert got_lines == lines
    want = oracle.OracleIndex(data, L)
    for c, o in zip(comp, outs):
        np.testing.assert_array_equal(o.astype(np.int64).reshape(lines, -1, 2),
                                      want.query(c.ir_bytes, c.num_result_slots))
