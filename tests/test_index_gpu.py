"""Fused structural indexer on the GPU vs the CPU oracle: bit-exact E, Q, S,
LB and newline index (integer/bit work: no tolerance)."""
import json
import random
from pathlib import Path

import numpy as np
import pytest

import oracle
from devmem import index_arrays, to_device

pytestmark = pytest.mark.gpu

KATS = json.loads((Path(__file__).parent / "golden" / "reference_kats.json").read_text())
TILE = 32768


def gpu_index(ctx, gpj, data, L, flags=1, offset=0):
    b = oracle.as_bytes(data)
    t, ptr = to_device(b, offset)
    ix = ctx.build_index(ptr, b.size, L, flags)
    try:
        arrs = index_arrays(ix)
        arrs["num_lines"] = ix.num_lines
        arrs["final_in_string"] = ix.final_in_string
        arrs["final_depth"] = ix.final_depth
    finally:
        ctx.free_index(ix)
    del t
    return arrs


def assert_same(got, want: oracle.OracleIndex, eq=True):
    assert got["num_lines"] == want.num_lines
    np.testing.assert_array_equal(got["NL"], want.NL)
    np.testing.assert_array_equal(got["S"], want.S)
    np.testing.assert_array_equal(got["LB"], want.LB)
    if eq:
        np.testing.assert_array_equal(got["E"], want.E)
        np.testing.assert_array_equal(got["Q"], want.Q)


def test_reference_kats(cuda_ctx, gpj):
    k = KATS["newline"]
    assert gpu_index(cuda_ctx, gpj, k["data"], 1)["NL"].tolist() == k["expected"]
    k = KATS["string"]
    assert gpu_index(cuda_ctx, gpj, k["data"], 1)["S"].tolist() == k["expected"]
    k = KATS["leveled"]
    assert gpu_index(cuda_ctx, gpj, k["data"], k["num_levels"])["LB"].tolist() == k["expected"]
    k = KATS["ld_json_fixture"]
    got = gpu_index(cuda_ctx, gpj, k["data"], k["max_depth"])
    assert_same(got, oracle.OracleIndex(k["data"], k["max_depth"]))


def _jsonish(rng: random.Random, n: int, backslash_weight=3) -> bytes:
    alphabet = b'{}[]:,"\\\n a1\xc3'
    weights = [4, 4, 3, 3, 5, 5, 8, backslash_weight, 1, 6, 12, 4, 1]
    return bytes(rng.choices(alphabet, weights=weights, k=n))


SIZES = [0, 1, 2, 63, 64, 65, 127, 128, 129, 255, 4095, 4096, 4097,
         TILE - 1, TILE, TILE + 1, TILE + 64, 2 * TILE + 100, 5 * TILE + 12345]


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("flags", [1, 3], ids=["tma", "no_tma"])
def test_sizes_random(cuda_ctx, gpj, n, flags):
    rng = random.Random(n * 7 + flags)
    data = _jsonish(rng, n)
    L = rng.choice([1, 2, 3, 4, 5, 8, 9, 22])
    assert_same(gpu_index(cuda_ctx, gpj, data, L, flags), oracle.OracleIndex(data, L))


@pytest.mark.parametrize("levels", [0, 1, 2, 3, 4, 5, 8, 9, 16, 22])
def test_levels(cuda_ctx, gpj, levels):
    rng = random.Random(levels)
    data = _jsonish(rng, 3 * TILE + 77)
    assert_same(gpu_index(cuda_ctx, gpj, data, levels), oracle.OracleIndex(data, levels))


@pytest.mark.parametrize("levels", [1, 2, 4])
def test_listed_walk_dense_and_sparse_quarters(cuda_ctx, gpj, levels):
    """Indexes of up to four levels walk the 32-byte quarters that hold two
    or more brackets from a per-warp list and the others straight-line:
    bracket-dense runs (every quarter of a warp listed, four passes) next to
    sparse records (empty and single-event quarters), and bracket runs deep
    enough to wrap the signed-char depth inside listed quarters."""
    rng = random.Random(100 + levels)
    parts = []
    for _ in range(80):
        k = rng.randrange(4)
        if k == 0:
            parts.append(b"[" * rng.randrange(1, 300))
        elif k == 1:
            parts.append(b"]" * rng.randrange(1, 300))
        elif k == 2:
            parts.append(bytes(rng.choices(b"{}[]:,", k=rng.randrange(100, 5000))))
        else:
            parts.append(b'{"a":1,"b":"x' + b" " * rng.randrange(0, 3000) + b'"}\n')
    data = b"".join(parts)
    assert_same(gpu_index(cuda_ctx, gpj, data, levels), oracle.OracleIndex(data, levels))


@pytest.mark.parametrize("offset", [1, 3, 8, 13])
def test_unaligned_input(cuda_ctx, gpj, offset):
    rng = random.Random(offset)
    data = _jsonish(rng, 2 * TILE + 999)
    assert_same(gpu_index(cuda_ctx, gpj, data, 4, 1, offset), oracle.OracleIndex(data, 4))


def test_backslash_runs_across_word_and_tile_edges(cuda_ctx, gpj):
    parts = bytearray()
    rng = random.Random(1)
    # runs of 1..140 backslashes ending right before a quote, placed so that
    # they straddle 64-byte words and 32 KiB tiles
    for run in list(range(1, 141)) + [63, 64, 65, 127, 128, 129] * 4:
        target = rng.choice([64, TILE])
        pad = (-(len(parts) + run // 2)) % target
        parts += b"a" * pad + b"\\" * run + b'"xy"' + b"{:[,]}"
    data = bytes(parts)
    assert_same(gpu_index(cuda_ctx, gpj, data, 3), oracle.OracleIndex(data, 3))


def test_all_backslash_words(cuda_ctx, gpj):
    data = (b"a" * 63 + b"\\" + b"\\" * 64 + b'"x"') * 300 + b"\\" * 64 * 600 + b'"q"'
    assert_same(gpu_index(cuda_ctx, gpj, data, 2), oracle.OracleIndex(data, 2))


def test_deep_nesting_wraps_signed_char(cuda_ctx, gpj):
    data = (b"[" * 300 + b"1" + b"]" * 300 + b",") * 200 + b"{" * 40000 + b"}" * 39000
    got = gpu_index(cuda_ctx, gpj, data, 22)
    want = oracle.OracleIndex(data, 22)
    assert_same(got, want)
    assert got["final_depth"] == ((-1 + 1000 + 128) % 256) - 128


def test_unbalanced_quotes_and_newlines_in_strings(cuda_ctx, gpj):
    data = (b'{"a":"x\ny",\n"b":[1,2]}\n' * 5000) + b'{"open":"never closed ' + b"z" * 100
    got = gpu_index(cuda_ctx, gpj, data, 3)
    want = oracle.OracleIndex(data, 3)
    assert_same(got, want)
    assert got["final_in_string"] == 1


def test_newline_capacity_retry(cuda_ctx, gpj):
    data = b"\n" * (3 * TILE + 5) + b'{"a":1}\n' * 100
    got = gpu_index(cuda_ctx, gpj, data, 1)
    want = oracle.OracleIndex(data, 1)
    assert got["num_lines"] == data.count(b"\n") + 1
    assert_same(got, want)


def test_synthetic_tweets_64mib(cuda_ctx, gpj):
    from gpjson_b200 import datagen
    data = datagen.tweets(0, 64 << 20)
    assert_same(gpu_index(cuda_ctx, gpj, data, 2), oracle.OracleIndex(data, 2))


def test_synthetic_products_16mib(cuda_ctx, gpj):
    from gpjson_b200 import datagen
    data = datagen.products(1, 16 << 20)
    assert_same(gpu_index(cuda_ctx, gpj, data, 4), oracle.OracleIndex(data, 4))


def test_async_build_into_caller_buffers(cuda_ctx, gpj):
    import torch
    from gpjson_b200 import datagen
    data = datagen.tweets(3, 3 << 20)
    t, ptr = to_device(data)
    n = data.size
    W = (n + 63) // 64
    S = torch.empty(W, dtype=torch.int64, device="cuda")
    LB = torch.empty(W * 3, dtype=torch.int64, device="cuda")
    E = torch.empty(W, dtype=torch.int64, device="cuda")
    Q = torch.empty(W, dtype=torch.int64, device="cuda")
    NL = torch.empty(n // 64 + 16, dtype=torch.int64, device="cuda")
    summ = torch.zeros(4, dtype=torch.int64, device="cuda")
    ix = gpj.Index()
    ix.d_string, ix.d_leveled, ix.d_escape, ix.d_quote = S.data_ptr(), LB.data_ptr(), \
        E.data_ptr(), Q.data_ptr()
    ix.d_newline, ix.newline_capacity = NL.data_ptr(), NL.numel()
    stream = torch.cuda.current_stream().cuda_stream
    cuda_ctx.build_index_async(ptr, n, 3, ix, summ.data_ptr(), flags=1, stream=stream)
    torch.cuda.synchronize()
    want = oracle.OracleIndex(data, 3)
    s = summ.cpu().numpy()
    assert s[0] == want.num_lines and s[3] == 0
    np.testing.assert_array_equal(S.cpu().numpy().view(np.uint64), want.S)
    np.testing.assert_array_equal(LB.cpu().numpy().view(np.uint64), want.LB)
    np.testing.assert_array_equal(E.cpu().numpy().view(np.uint64), want.E)
    np.testing.assert_array_equal(Q.cpu().numpy().view(np.uint64), want.Q)
    np.testing.assert_array_equal(NL.cpu().numpy()[: want.num_lines], want.NL)


def test_async_summary_is_four_words(cuda_ctx, gpj):
    """gpj_index_build_async writes exactly d_summary[0..3] (lines, in-string,
    depth, error bits): a guard word right after them stays untouched."""
    import torch
    from gpjson_b200 import datagen
    guard = 0x5A5A5A5A5A5A5A5A
    for data in (datagen.tweets(6, 100_000), np.zeros(0, np.uint8)):
        n = data.size
        t, ptr = to_device(data)
        W = max(1, (n + 63) // 64)
        S = torch.empty(W, dtype=torch.int64, device="cuda")
        LB = torch.empty(W * 2, dtype=torch.int64, device="cuda")
        NL = torch.empty(n // 16 + 16, dtype=torch.int64, device="cuda")
        summ = torch.full((5,), guard, dtype=torch.int64, device="cuda")
        ix = gpj.Index()
        ix.d_string, ix.d_leveled = S.data_ptr(), LB.data_ptr()
        ix.d_newline, ix.newline_capacity = NL.data_ptr(), NL.numel()
        cuda_ctx.build_index_async(ptr, n, 2, ix, summ.data_ptr())
        torch.cuda.synchronize()
        s = summ.cpu().numpy()
        want = oracle.OracleIndex(data, 2)
        assert s[0] == want.num_lines and s[1] == 0 and s[2] == -1 and s[3] == 0
        assert s[4] == guard


def test_lookback_wait_runs_out_and_reports_timeout(cuda_ctx, gpj):
    """A look-back whose predecessor never publishes (tile 0 left out of the
    launch) gives up after a bounded number of polls: the kernel returns, the
    error word carries the look-back bit, the host reports GPJ_ERR_TIMEOUT,
    and the context keeps working for the next build."""
    import torch
    from gpjson_b200 import datagen
    data = datagen.tweets(5, 8 * TILE)
    n = data.size
    t, ptr = to_device(data)
    diag = gpj.GPJ_INDEX_DIAG_TILE0_UNPUBLISHED
    with pytest.raises(gpj.DeviceTimeoutError, match="bounded wait"):
        cuda_ctx.build_index(ptr, n, 2, diag)
    W = (n + 63) // 64
    S = torch.empty(W, dtype=torch.int64, device="cuda")
    LB = torch.empty(W * 2, dtype=torch.int64, device="cuda")
    NL = torch.empty(n // 16 + 16, dtype=torch.int64, device="cuda")
    summ = torch.zeros(4, dtype=torch.int64, device="cuda")
    ix = gpj.Index()
    ix.d_string, ix.d_leveled = S.data_ptr(), LB.data_ptr()
    ix.d_newline, ix.newline_capacity = NL.data_ptr(), NL.numel()
    cuda_ctx.build_index_async(ptr, n, 2, ix, summ.data_ptr(), flags=diag)
    torch.cuda.synchronize()
    assert int(summ[3].item()) & 1  # look-back timeout bit
    with pytest.raises(ValueError, match="two tiles"):
        cuda_ctx.build_index(ptr, 1000, 2, diag)
    # the same context, a normal build: bit-exact again
    assert_same(gpu_index(cuda_ctx, gpj, data, 2), oracle.OracleIndex(data, 2))


def test_released_blocks_are_reused(gpj):
    """gpj_index_free keeps released blocks in the context: a later build of
    a similar size takes one (no cudaMalloc) and its indexes are bit-exact;
    a block more than 1.5x (+ 16 MiB) too large is left alone.  An index
    freed after its context is gone is released with a null context."""
    from gpjson_b200 import datagen
    big = datagen.tweets(17, 48 << 20)
    small = datagen.tweets(18, 2 << 20)
    tb, pb = to_device(big)
    ts, ps = to_device(small)
    want_small = oracle.OracleIndex(small, 3)
    with gpj.Context(0) as ctx:
        a = ctx.build_index(pb, big.size, 3)
        block_a, first = a.owner, index_arrays(a)
        ctx.free_index(a)
        a = ctx.build_index(pb, big.size, 3)
        assert a.owner == block_a
        again = index_arrays(a)
        for k in ("S", "LB", "NL"):
            np.testing.assert_array_equal(again[k], first[k], err_msg=k)
        s = ctx.build_index(ps, small.size, 3)  # the big block is live
        block_s = s.owner
        assert block_s != block_a
        ctx.free_index(s)
        ctx.free_index(a)
        s = ctx.build_index(ps, small.size, 3)  # the small block fits best
        assert s.owner == block_s
        got = index_arrays(s)
        np.testing.assert_array_equal(got["S"], want_small.S)
        np.testing.assert_array_equal(got["LB"], want_small.LB)
        np.testing.assert_array_equal(got["NL"][:s.num_lines], want_small.NL)
        ctx.free_index(s)
        tiny = datagen.tweets(19, 64 << 10)
        tt, pt = to_device(tiny)
        t = ctx.build_index(pt, tiny.size, 3)  # the big block is too large
        assert t.owner not in (block_a,)
        ctx.free_index(t)
        late = ctx.build_index(pb, big.size, 3)
    ctx.free_index(late)  # context closed: plain cudaFree
    assert late.owner is None
