"""Pins the CPU oracle against the reference's own known answers (CPU only).

The vectors in tests/golden/reference_kats.json were extracted from the
reference's unit tests by tests/golden/make_golden.py.
"""
import json
import random
from pathlib import Path

import numpy as np
import pytest

import oracle
import ref_test_oracles as rto

KATS = json.loads((Path(__file__).parent / "golden" / "reference_kats.json").read_text())


def _reference_root() -> Path:
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "_gpjb_build_ref", Path(__file__).resolve().parent.parent / "oracle" / "ref" / "build_ref.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.reference_root()


# the reference's sample datasets, read in place where the reference is present
DATASETS = _reference_root() / "dataset"


def test_newline_kat():
    k = KATS["newline"]
    ix = oracle.OracleIndex(k["data"], 1)
    assert ix.NL.tolist() == k["expected"]


def test_string_kat():
    k = KATS["string"]
    ix = oracle.OracleIndex(k["data"], 1)
    assert ix.S.tolist() == k["expected"]


def test_leveled_kat():
    k = KATS["leveled"]
    ix = oracle.OracleIndex(k["data"], k["num_levels"])
    assert ix.LB.tolist() == k["expected"]


def test_ld_json_fixture_matches_reference_test_oracles():
    k = KATS["ld_json_fixture"]
    data = k["data"].encode()
    ix = oracle.OracleIndex(data, k["max_depth"])
    assert ix.NL.tolist() == rto.expected_newline_index(data)
    assert ix.S.tolist() == rto.expected_string_index(data).tolist()
    assert ix.LB.tolist() == rto.expected_leveled_bitmap_index(data, k["max_depth"]).tolist()


def _values(ix, compiled):
    res = ix.query(compiled.ir_bytes, compiled.num_result_slots)
    out = []
    for line in res:
        vals = [bytes(ix.data[s:e]).decode() for s, e in line if s >= 0 and e >= 0]
        out.append(vals)
    return out


def test_query_executor_kat(gpj):
    k = KATS["query_executor"]
    ix = oracle.OracleIndex(k["json_text"], 4)
    for qi, expected in k["expected"].items():
        c = gpj.compile(k["queries"][int(qi)])
        assert _values(ix, c) == [[expected]]
    c = gpj.compile(k["unmatched_query"])
    assert _values(ix, c) == [[]]


def test_engine_kat(gpj):
    k = KATS["engine"]
    data = k["contents"].encode()
    comp = [gpj.compile(q) for q in k["queries"]]
    ix = oracle.OracleIndex(data, max(c.max_depth for c in comp))
    vals = [_values(ix, c) for c in comp]
    for q, line, expected in k["expected"]:
        assert vals[q][line] == [expected]
    assert vals[0][2] == []  # the empty record after the final newline


def _random_jsonish(rng: random.Random, n: int) -> bytes:
    alphabet = b'{}[]:,"\\\n ab1'
    weights = [4, 4, 3, 3, 5, 5, 8, 3, 1, 6, 10, 10, 4]
    return bytes(rng.choices(alphabet, weights=weights, k=n))


@pytest.mark.parametrize("seed", range(40))
def test_oracle_matches_reference_test_oracles_random(seed):
    rng = random.Random(seed)
    n = rng.choice([0, 1, 7, 63, 64, 65, 127, 128, 129, 300, 1000, 4097])
    data = _random_jsonish(rng, n)
    L = rng.choice([1, 2, 3, 5, 8])
    ix = oracle.OracleIndex(data, L)
    assert ix.NL.tolist() == rto.expected_newline_index(data)
    # the reference test helpers use the unbounded backslash rule; random
    # inputs this short never hold a run of 64 backslashes.  They leave the
    # bits past the end 0, while the builders' shift-xor cascade
    # (sharemem/string-index.cu:16-28) carries the end-of-data string state
    # into them: compare in-range bits, then check the tail separately.
    S = ix.S.copy()
    want = rto.expected_string_index(data)
    if n % 64:
        valid = (1 << (n % 64)) - 1
        tail = int(S[-1]) & ~valid & (2**64 - 1)
        assert tail in (0, (2**64 - 1) & ~valid)
        S[-1] = np.uint64(int(S[-1]) & valid)
    assert S.tolist() == want.tolist()
    assert ix.LB.tolist() == rto.expected_leveled_bitmap_index(data, L).tolist()


def test_word_local_escape_rule():
    """A 64-byte all-backslash word passes carry 0 on (the builders' rule),
    while an unbounded count would escape the quote after it."""
    data = b"a" * 63 + b"\\" + b"\\" * 64 + b'"x"'
    ix = oracle.OracleIndex(data, 1)
    unbounded = oracle.escape_unbounded(data)
    # byte 128 (the quote) is escaped under the unbounded rule ...
    assert int(unbounded[2]) & 1 == 1
    # ... but not under the word-local rule the GPU builders implement
    assert int(ix.E[2]) & 1 == 0
    assert int(ix.Q[2]) & 1 == 1


def test_signed_char_depth_wraps():
    data = b"[" * 200 + b"1" + b"]" * 200
    ix = oracle.OracleIndex(data, 4)
    # depths 0..3 get their bracket, depth 128.. wraps negative and is skipped
    lvl0 = [i for i in range(len(data)) if int(ix.LB[i // 64]) >> (i % 64) & 1]
    assert lvl0 == [0, len(data) - 1]


@pytest.mark.skipif(not DATASETS.exists(), reason="reference sample datasets absent")
@pytest.mark.parametrize("name", ["twitter_sample_small_records.json",
                                  "bestbuy_sample_small_records.json"])
def test_oracle_on_reference_samples(name):
    data = (DATASETS / name).read_bytes()
    ix = oracle.OracleIndex(data, 3)
    assert ix.NL.tolist() == rto.expected_newline_index(data)
    assert ix.S.tolist() == rto.expected_string_index(data).tolist()
    assert ix.LB.tolist() == rto.expected_leveled_bitmap_index(data, 3).tolist()


def test_query_oracle_semantics_on_synthetic_records(gpj):
    """$.user.lang and indexed hashtags agree with a JSON parser."""
    from gpjson_b200 import datagen
    data = bytes(datagen.tweets(5, 200_000))
    recs = [json.loads(line) for line in data.split(b"\n") if line]
    ix = oracle.OracleIndex(data, 4)
    for q, get in [
        ("$.user.lang", lambda r: [r["user"]["lang"]]),
        ("$.entities.hashtags[1].text",
         lambda r: [r["entities"]["hashtags"][1]["text"]] if len(r["entities"]["hashtags"]) > 1 else []),
        ("$.place.country_code",
         lambda r: [r["place"]["country_code"]] if r["place"] else []),
        ("$.retweeted_status.user.id",
         lambda r: [r["retweeted_status"]["user"]["id"]] if "retweeted_status" in r else []),
    ]:
        vals = _values(ix, gpj.compile(q))
        for i, r in enumerate(recs):
            want = [json.dumps(v, ensure_ascii=False, separators=(",", ":")) for v in get(r)]
            assert vals[i] == want, (q, i)


def normalize_array_file(data: bytes):
    """The reference's array-to-NDJSON normalisation
    (tests/benchmark/benchmark_large_output_test.cpp:31-66): drop "[", "]" and
    "," lines and one trailing comma per line.  Returns the normalised bytes
    and, per kept line, (raw start offset, normalised start offset)."""
    out = bytearray()
    kept = []
    pos = 0
    for raw in data.split(b"\n"):
        start = pos
        pos += len(raw) + 1
        line = raw.rstrip(b"\r")
        if line in (b"", b"[", b"]", b","):
            continue
        if line.endswith(b","):
            line = line[:-1]
        kept.append((start, len(out)))
        out += line + b"\n"
    return bytes(out), kept


def test_array_records_match_reference_normalisation(gpj):
    """$[*].X on the raw array file (records = elements, bitmap level 1)
    equals the reference running $.X on its normalised NDJSON copy, shifted by
    each element's byte offset."""
    from gpjson_b200 import datagen
    raw = bytes(datagen.products(9, 400_000))
    norm, kept = normalize_array_file(raw)
    c = gpj.compile("$.categoryPath[1:3].id")
    got = oracle.OracleIndex(raw, c.max_depth + 1).query(c.ir_bytes, c.num_result_slots, 1)
    want = oracle.OracleIndex(norm, c.max_depth).query(c.ir_bytes, c.num_result_slots)
    # raw record r (line r) holds element r-1: line 0 is "["
    assert got[0].tolist() == [[-1, -1]] * c.num_result_slots
    for j, (rs, ns) in enumerate(kept):
        shift = rs - ns
        w = np.where(want[j] >= 0, want[j] + shift, -1)
        assert got[j + 1].tolist() == w.tolist(), j
    assert (got[len(kept) + 1:] == -1).all()
