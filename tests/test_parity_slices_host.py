"""The slice-parallel oracle check used for the full-size parity tests and
the bench's parity gate: on CPU, a whole-partition oracle index passes it
exactly, and a mistake planted in that stand-in (one bit of the string
mask, one leveled bit, one newline offset, one result) is caught."""
import numpy as np
import pytest

import oracle
import parity_slices as ps


@pytest.fixture(scope="module")
def corpus(gpj):
    from gpjson_b200 import datagen
    data = datagen.tweets(17, 3 << 20, deep=True)
    queries = [gpj.compile(q, wildcard_limit=8) for q in
               ["$.user.lang", "$.entities.hashtags[*].text", "$.place.country_code"]]
    L = max(c.max_depth for c in queries)
    whole = oracle.OracleIndex(data, L)
    results = [whole.query(c.ir_bytes, c.num_result_slots) for c in queries]
    return data, queries, L, whole, results


def test_bit_range_realigns_words():
    rng = np.random.default_rng(0)
    words = rng.integers(0, 2**63, 40, dtype=np.uint64) * np.uint64(2) + np.uint64(1)
    bits = np.unpackbits(words.view(np.uint8), bitorder="little")
    for start, nbits in [(0, 64), (3, 100), (64, 1), (127, 600), (5, 0), (1000, 1500)]:
        got = ps.bit_range(words, start, nbits)
        want_bits = np.zeros(((nbits + 63) // 64) * 64, np.uint8)
        seg = bits[start:start + nbits]
        want_bits[:seg.size] = seg
        want = np.packbits(want_bits, bitorder="little").view(np.uint64)
        np.testing.assert_array_equal(got, want)


def test_slices_agree_with_whole_partition(corpus):
    data, queries, L, whole, results = corpus
    info = ps.check_ndjson_partition(data, L, whole.S, whole.LB, whole.NL, queries, results,
                                     slice_bytes=200_000, threads=4)
    assert info["slices"] > 10 and info["lines"] == whole.num_lines


@pytest.mark.parametrize("what", ["S", "LB", "NL", "R"])
def test_planted_mistake_is_caught(corpus, what):
    data, queries, L, whole, results = corpus
    S, LB, NL = whole.S.copy(), whole.LB.copy(), whole.NL.copy()
    R = [r.copy() for r in results]
    if what == "S":
        S[S.size // 2] ^= np.uint64(1 << 17)
    elif what == "LB":
        LB[LB.size // 3] ^= np.uint64(1 << 40)
    elif what == "NL":
        NL[NL.size // 2] += 1
    else:
        hit = np.argwhere(R[0][:, 0, 0] >= 0).ravel()
        R[0][hit[hit.size // 2], 0, 1] += 1
    with pytest.raises(AssertionError):
        ps.check_ndjson_partition(data, L, S, LB, NL, queries, R, slice_bytes=200_000,
                                  threads=4)
