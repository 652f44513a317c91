"""Device-side result compaction (gpj_results_compact) vs the same
compaction done in numpy on the copied-back result array: matches in (line,
slot) order with global offsets, and the arena of matched bytes, bit for bit.
The reference does this on the host per line and slot
(query_executor_host.cu:80-119), raising an execution error for an invalid
range; so does the compaction."""
import numpy as np
import pytest
import torch

from devmem import to_device

pytestmark = pytest.mark.gpu

QUERIES = ["$.user.lang", "$.entities.hashtags[0:8].text", "$.place.country_code", "$.user",
           "$.nonexistent.key"]


def _expected(data: bytes, res: np.ndarray, lines: int, slots: int, base: int):
    pairs = res.reshape(lines * slots, 2).astype(np.int64)
    idx = np.nonzero((pairs[:, 0] >= 0) & (pairs[:, 1] >= 0))[0]
    starts, ends = pairs[idx, 0], pairs[idx, 1]
    lengths = ends - starts
    text = np.concatenate([[0], np.cumsum(lengths)[:-1]]) if idx.size else np.zeros(0, np.int64)
    arena = b"".join(data[s:e] for s, e in zip(starts, ends))
    return idx // slots, idx % slots, starts + base, ends + base, lengths, text, arena


@pytest.mark.parametrize("base", [0, 123456789])
def test_compaction_matches_host_loop(cuda_ctx, gpj, base):
    from gpjson_b200 import datagen
    data = datagen.tweets(8, 4 << 20)
    raw = data.tobytes()
    comp = [gpj.compile(q) for q in QUERIES]
    L = max(c.max_depth for c in comp)
    t, ptr = to_device(data)
    ix = cuda_ctx.build_index(ptr, data.size, L)
    try:
        for c in comp:
            slots = c.num_result_slots
            out = torch.full((max(1, ix.num_lines * slots * 2),), -1, dtype=torch.int32,
                             device="cuda")
            cuda_ctx.query(ix, c, out.data_ptr())
            # capacities far too small at first: the wrapper grows them and repeats
            matches, arena = gpj.compact_results(cuda_ctx, out.data_ptr(), ix.num_lines, slots,
                                                 ptr, data.size, base, match_capacity=3,
                                                 arena_capacity=10)
            res = out.cpu().numpy()[: ix.num_lines * slots * 2]
            line, slot, start, end, length, text, want_arena = _expected(raw, res, ix.num_lines,
                                                                         slots, base)
            assert matches.size == line.size, c.query_text
            np.testing.assert_array_equal(matches["line"], line)
            np.testing.assert_array_equal(matches["slot"], slot)
            np.testing.assert_array_equal(matches["start"], start)
            np.testing.assert_array_equal(matches["end"], end)
            np.testing.assert_array_equal(matches["length"], length)
            np.testing.assert_array_equal(matches["text_offset"], text)
            assert arena == want_arena, c.query_text
    finally:
        cuda_ctx.free_index(ix)


def test_compaction_capacity_and_offsets_only(cuda_ctx, gpj):
    """Beyond the capacities nothing is written but the counts are exact;
    without an arena only offsets are produced."""
    res = np.array([[0, 3], [-1, -1], [5, 9], [10, 10], [-1, 4], [20, 26]], np.int32)
    data = bytes(range(97, 97 + 32))
    t_in, p_in = to_device(np.frombuffer(data, np.uint8).copy())
    d_res = torch.from_numpy(res.reshape(-1)).cuda()
    counts = torch.zeros(3, dtype=torch.int64, device="cuda")
    matches = torch.full((2 * gpj.MATCH_DTYPE.itemsize,), 0xEE, dtype=torch.uint8, device="cuda")
    cuda_ctx.compact(d_res.data_ptr(), 3, 2, p_in, len(data), 7, matches.data_ptr(), 2, 0, 0,
                     counts.data_ptr())
    torch.cuda.synchronize()
    assert counts.cpu().tolist() == [4, 3 + 4 + 0 + 6, 0]
    got = matches.cpu().numpy().view(gpj.MATCH_DTYPE)
    assert got["line"].tolist() == [0, 1] and got["slot"].tolist() == [0, 0]
    assert got["start"].tolist() == [7, 12] and got["end"].tolist() == [10, 16]


@pytest.mark.parametrize("pair", [(9, 5), (3, 40)], ids=["start_after_end", "end_past_input"])
def test_invalid_range_is_an_execution_error(cuda_ctx, gpj, pair):
    res = np.array([0, 2, pair[0], pair[1]], np.int32)
    data = np.frombuffer(b"x" * 32, np.uint8).copy()
    t_in, p_in = to_device(data)
    d_res = torch.from_numpy(res).cuda()
    with pytest.raises(gpj.QueryExecutionError, match="invalid result range"):
        gpj.compact_results(cuda_ctx, d_res.data_ptr(), 2, 1, p_in, data.size)


def test_no_results(cuda_ctx, gpj):
    t_in, p_in = to_device(np.zeros(64, np.uint8))
    matches, arena = gpj.compact_results(cuda_ctx, 0, 0, 3, p_in, 64)
    assert matches.size == 0 and arena == b""
