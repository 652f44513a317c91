"""The reference implementation itself against this engine on the same bytes.

The reference library is compiled from its own sources into oracle/_ref by
oracle/ref/build_ref.py and driven by the harness oracle/ref/ref_dump.cpp;
for each of its four index builders (UNCOMBINED, COMBINED, FUSED, SHAREMEM)
the string mask, leveled bitmaps, newline index and query results must equal
this engine's bit for bit, and the escape and quote bitmaps of its SHAREMEM
kernels (escape_index, quote_index) must equal this engine's E and Q.
Inputs range from the reference's own fixtures to 64 MiB of post records
(the c0 workload).  Inputs are well-formed JSON only: the reference's query
search loops have no bound on malformed input, and its kernels assert on a
few inputs, so every input and query is first checked on the CPU against
those assert conditions (tests/ref_guard.py) and never reaches the reference
if one would fire.  Skipped where oracle/_ref was not built (no reference
sources at build time)."""
import json
import subprocess
from pathlib import Path

import numpy as np
import pytest
import torch

import oracle
import ref_guard
from devmem import to_device, index_arrays

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parent.parent
REF = ROOT / "oracle" / "_ref" / "ref_dump"
KATS = json.loads((Path(__file__).parent / "golden" / "reference_kats.json").read_text())

TWEET_QUERIES = ["$.user.lang", "$.entities.hashtags[0:8].text", "$.place.country_code",
                 "$.retweeted_status.user.id", "$['user']['name']", "$.entities.urls[0,1].url",
                 "$.user", "$.nonexistent.key"]
LINE_QUERIES = ["$.categoryPath[1:3].id", "$.sku", "$.offers[0]", "$.name"]


def _escapes() -> bytes:
    # backslash runs of every length up to 60 inside strings, escaped quotes,
    # runs across 64-byte word edges (each line stays valid JSON)
    lines = []
    for k in range(0, 61):
        esc = "\\\\" * (k // 2) + ('\\"' if k % 2 else "")
        lines.append('{"a":"' + "x" * (k % 61) + esc + '","b":[{"c":"' + esc + '"},[1,2]],"d":' +
                     str(k) + '}')
    return ("\n".join(lines) + "\n").encode()


def _as_ndjson(array_file: bytes) -> bytes:
    lines = array_file.split(b"\n")
    elems = [ln.rstrip(b",") for ln in lines if ln not in (b"[", b"]", b"")]
    return b"\n".join(elems) + b"\n"


def _inputs():
    from gpjson_b200 import datagen
    products = bytes(datagen.products(42, 1 << 20))
    return {
        "ld_fixture": (KATS["ld_json_fixture"]["data"].encode(), ["$.id", "$.name", "$.nested.arr[1].x"]),
        "bookstore": (KATS["query_executor"]["json_text"].encode(),
                      ["$.store.book[0:4].author", "$.store.bicycle.color", "$.store.book[1].price"]),
        "escapes": (_escapes(), ["$.a", "$.b[0].c", "$.d", "$.b[1][1]"]),
        "tweets_2MiB": (bytes(datagen.tweets(41, 2 << 20, deep=True)), TWEET_QUERIES),
        # the array file for the index only (its records sit one level down),
        # and its elements as NDJSON -- the reference's own normalisation
        # (tests/benchmark/benchmark_large_output_test.cpp:31-66) -- for queries
        "products_array_1MiB": (products, []),
        "products_ndjson_1MiB": (_as_ndjson(products), LINE_QUERIES),
        "tweets_64MiB_c0": (bytes(datagen.tweets(0, 64 << 20)),
                            ["$.user.lang", "$.entities.hashtags[0:8].text", "$.place.country_code"]),
    }


def _read(path, dtype=np.int64):
    return np.fromfile(path, dtype=dtype) if Path(path).exists() else np.zeros(0, dtype)


@pytest.fixture(scope="module")
def cases(tmp_path_factory):
    if not REF.exists():
        pytest.skip("oracle/_ref/ref_dump not built")
    if not torch.cuda.is_available():
        pytest.skip("CUDA device required")
    d = tmp_path_factory.mktemp("refparity")
    out = {}
    for name, (data, queries) in _inputs().items():
        p = d / f"{name}.json"
        p.write_bytes(data)
        out[name] = (p, data, queries)
    return d, out


@pytest.mark.parametrize("builder", [0, 1, 2, 3], ids=["UNCOMBINED", "COMBINED", "FUSED", "SHAREMEM"])
def test_reference_outputs_equal_ours(cases, builder, gpj, cuda_ctx):
    d, inputs = cases
    for name, (path, data, queries) in inputs.items():
        comp = [gpj.compile(q) for q in queries]
        levels = max([4] + [c.max_depth for c in comp])
        # nothing reaches the reference's device asserts
        assert ref_guard.problems(data, comp, levels) == [], name
        prefix = d / f"{name}.b{builder}"
        r = subprocess.run([str(REF), str(path), str(builder), str(levels), str(prefix)] + queries,
                           capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        ref_S, ref_LB, ref_NL = (_read(f"{prefix}.{k}") for k in ("S", "LB", "NL"))
        b = oracle.as_bytes(data)
        t, ptr = to_device(b)
        ix = cuda_ctx.build_index(ptr, b.size, levels, gpj.GPJ_INDEX_EMIT_ESCAPE_QUOTE)
        try:
            ours = index_arrays(ix)
            W = (b.size + 63) // 64
            np.testing.assert_array_equal(ours["E"].view(np.int64), _read(f"{prefix}.E")[:W],
                                          err_msg=f"{name} E")
            np.testing.assert_array_equal(ours["Q"].view(np.int64), _read(f"{prefix}.Q")[:W],
                                          err_msg=f"{name} Q")
            np.testing.assert_array_equal(ours["S"].view(np.int64), ref_S[:W], err_msg=f"{name} S")
            np.testing.assert_array_equal(ours["LB"].view(np.int64), ref_LB[:W * levels],
                                          err_msg=f"{name} LB")
            np.testing.assert_array_equal(ours["NL"], ref_NL, err_msg=f"{name} NL")
            for q, c in enumerate(comp):
                out = torch.full((max(1, ix.num_lines * c.num_result_slots * 2),), -7,
                                 dtype=torch.int32, device="cuda")
                cuda_ctx.query(ix, c, out.data_ptr())
                torch.cuda.synchronize()
                got = out.cpu().numpy()[: ix.num_lines * c.num_result_slots * 2].astype(np.int64)
                np.testing.assert_array_equal(got, _read(f"{prefix}.R{q}"),
                                              err_msg=f"{name} {queries[q]}")
        finally:
            cuda_ctx.free_index(ix)
