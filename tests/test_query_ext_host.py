"""Query-language extensions of this build, pinned on CPU: the oracle's
results for numeric filters, "..name" and the "[*]" element-count check
agree with an independent evaluation of the same paths over json.loads of
every record.  The reference's compiler rejects these queries
(src/gpjson/query/query_compiler.cpp:202-204, 287-289, 366-391), so there is
no reference output to compare with; the JSON parser is the second opinion.
"""
import json
from decimal import Decimal

import numpy as np
import pytest

import oracle


def _records(data: bytes):
    return [ln for ln in data.split(b"\n")]


def _loads(b: bytes):
    return json.loads(b, parse_float=Decimal, parse_int=Decimal)


def _descend(v, name, out):
    """Every member `name` below v, pre-order (= by position of its ':')."""
    if isinstance(v, dict):
        for k, x in v.items():
            if k == name:
                out.append(x)
            _descend(x, name, out)
    elif isinstance(v, list):
        for x in v:
            _descend(x, name, out)


def _get(v, path):
    for k in path:
        if isinstance(k, int):
            if not isinstance(v, list) or k >= len(v):
                return None
            v = v[k]
        else:
            if not isinstance(v, dict) or k not in v:
                return None
            v = v[k]
    return v


def _values(data: bytes, res):
    """Parsed values of the (start, end) pairs of every record."""
    return [[_loads(data[s:e]) for s, e in line if s >= 0] for line in res]


@pytest.fixture(scope="module")
def tweets():
    from gpjson_b200 import datagen
    return datagen.tweets(41, 2 << 20, deep=True).tobytes()


@pytest.fixture(scope="module")
def products():
    from gpjson_b200 import datagen
    # one element per line; the lines between the brackets are the records
    lines = datagen.products(42, 1 << 20).tobytes().split(b"\n")
    return b"\n".join(ln.rstrip(b",") for ln in lines if ln.startswith(b"{"))


@pytest.mark.parametrize("name", ["id", "lang", "text", "indices", "country_code"])
def test_descend_matches_json_walk(gpj, tweets, name):
    c = gpj.compile(f"$..{name}", wildcard_limit=64)
    ix = oracle.OracleIndex(tweets, c.max_depth)
    got = _values(tweets, ix.query(c.ir_bytes, c.num_result_slots))
    assert not ix.last_status & oracle.OracleIndex.STATUS_OVERFLOW
    want = []
    for rec in _records(tweets):
        out = []
        if rec:
            _descend(_loads(rec), name, out)
        want.append(out)
    assert got == want
    assert sum(map(len, want)) > 100


def test_descend_below_a_member(gpj, tweets):
    c = gpj.compile("$.user..id", wildcard_limit=4)
    ix = oracle.OracleIndex(tweets, c.max_depth)
    got = _values(tweets, ix.query(c.ir_bytes, c.num_result_slots))
    want = []
    for rec in _records(tweets):
        out = []
        u = _get(_loads(rec), ["user"]) if rec else None
        if u is not None:
            _descend(u, "id", out)
        want.append(out)
    assert got == want


def test_descend_overflow_sets_status(gpj, tweets):
    c = gpj.compile("$..id", wildcard_limit=1)
    ix = oracle.OracleIndex(tweets, c.max_depth)
    res = ix.query(c.ir_bytes, c.num_result_slots)
    assert ix.last_status & oracle.OracleIndex.STATUS_OVERFLOW
    # the first match per record is still the first one in document order
    assert (res[:, 0, 0] >= 0).sum() > 0


@pytest.mark.parametrize("path,op,lit", [
    (["user", "followers_count"], ">", "50000"), (["user", "followers_count"], "<=", "9e3"),
    (["user", "friends_count"], "==", "914"), (["user", "statuses_count"], "!=", "0"),
    (["id"], ">=", "5E17"), (["user", "followers_count"], "<", "-1"),
])
def test_numeric_filter_on_value(gpj, tweets, path, op, lit):
    q = "$." + ".".join(path) + f"[?(@ {op} {lit})]"
    c = gpj.compile(q)
    ix = oracle.OracleIndex(tweets, c.max_depth)
    got = _values(tweets, ix.query(c.ir_bytes, c.num_result_slots))
    L = Decimal(lit)
    cmp = {">": lambda a: a > L, ">=": lambda a: a >= L, "<": lambda a: a < L,
           "<=": lambda a: a <= L, "==": lambda a: a == L, "!=": lambda a: a != L}[op]
    want = []
    for rec in _records(tweets):
        v = _get(_loads(rec), path) if rec else None
        want.append([v] if isinstance(v, Decimal) and cmp(v) else [])
    assert got == want


def test_numeric_filter_on_member_then_path(gpj, tweets):
    c = gpj.compile("$.user[?(@.followers_count >= 10000)].screen_name")
    ix = oracle.OracleIndex(tweets, c.max_depth)
    got = _values(tweets, ix.query(c.ir_bytes, c.num_result_slots))
    want = []
    for rec in _records(tweets):
        u = _get(_loads(rec), ["user"]) if rec else None
        ok = isinstance(u, dict) and isinstance(u.get("followers_count"), Decimal) and \
            u["followers_count"] >= 10000 and "screen_name" in u
        want.append([u["screen_name"]] if ok else [])
    assert got == want
    assert 0 < sum(map(len, want)) < len(want)


@pytest.mark.parametrize("field,op,lit", [("regularPrice", ">", "1000.5"),
                                          ("customerReviewAverage", "==", "2.30"),
                                          ("salePrice", "<", "12.5e1"),
                                          ("onSale", "==", "0")])
def test_numeric_filter_decimals(gpj, products, field, op, lit):
    c = gpj.compile(f"$.{field}[?(@ {op} {lit})]")
    ix = oracle.OracleIndex(products, c.max_depth)
    got = _values(products, ix.query(c.ir_bytes, c.num_result_slots))
    L = Decimal(lit)
    cmp = {">": lambda a: a > L, "<": lambda a: a < L, "==": lambda a: a == L}[op]
    want = []
    for rec in _records(products):
        v = _get(_loads(rec), [field]) if rec else None
        # booleans and strings are not numbers: the filter fails
        want.append([v] if isinstance(v, Decimal) and cmp(v) else [])
    assert got == want


def test_exact_decimal_comparison_edges(gpj):
    """Numbers that floating point would confuse, compared exactly."""
    vals = ["0", "-0", "0.0", "1", "1.0", "10e-1", "100E-2", "0.1", "0.10000000000000000001",
            "123456789012345678901234567890", "123456789012345678901234567891", "-5", "-5.0001",
            "1e400", "2E400", "-1e-400", "3.14159", "31.4159e-1"]
    data = "\n".join('{"v":%s}' % v for v in vals).encode()
    for lit in ["1", "0", "0.1", "-5", "1e400", "123456789012345678901234567890", "3.14159"]:
        for op in ["==", "!=", "<", "<=", ">", ">="]:
            c = gpj.compile(f"$.v[?(@ {op} {lit})]")
            ix = oracle.OracleIndex(data, c.max_depth)
            got = [bool(r[0][0] >= 0) for r in ix.query(c.ir_bytes, 1)]
            L = Decimal(lit)
            want = [{"==": a == L, "!=": a != L, "<": a < L, "<=": a <= L, ">": a > L,
                     ">=": a >= L}[op] for a in map(Decimal, vals)]
            assert got == want, (op, lit)


def test_wildcard_limit_overflow_status(gpj, tweets):
    lengths = [len(_get(_loads(r), ["entities", "hashtags"]) or []) if r else 0
               for r in _records(tweets)]
    assert max(lengths) > 3
    for k, expect in ((3, True), (max(lengths), False)):
        c = gpj.compile("$.entities.hashtags[*].text", wildcard_limit=k)
        ix = oracle.OracleIndex(tweets, c.max_depth)
        res = ix.query(c.ir_bytes, c.num_result_slots)
        assert bool(ix.last_status & oracle.OracleIndex.STATUS_OVERFLOW) == expect
        # the first k elements are returned either way
        want = []
        for rec in _records(tweets):
            h = _get(_loads(rec), ["entities", "hashtags"]) if rec else None
            want.append([x["text"] for x in h[:k]] if h else [])
        got = _values(tweets, res)
        assert got == want


# ---- slices counted from the end, and open slices ----

def array_records(seed: int = 7, count: int = 600) -> bytes:
    """Records with arrays of 0-11 elements (objects and numbers), nested
    pairs, and both compact and spaced separators."""
    rng = np.random.default_rng(seed)
    lines = []
    for i in range(count):
        arr = []
        for _ in range(int(rng.integers(0, 12))):
            if rng.random() < 0.7:
                arr.append({"v": int(rng.integers(-99, 99)), "s": "x" * int(rng.integers(0, 5))})
            else:
                arr.append(int(rng.integers(0, 1000)))
        rec = {"id": i, "a": arr, "b": {"c": [[j, j + 1] for j in range(int(rng.integers(0, 5)))]}}
        seps = (",", ":") if i % 2 else (", ", ": ")
        lines.append(json.dumps(rec, separators=seps))
    return "\n".join(lines).encode()


@pytest.fixture(scope="module")
def arrays():
    return array_records()


def _apply(values, rest):
    """The remaining steps over each selected element; a failed step ends the
    record (the reference abandons its remaining slots)."""
    out = []
    for x in values:
        if rest is None:
            out.append(x)
            continue
        kind, arg = rest
        if kind == "key" and isinstance(x, dict) and arg in x:
            out.append(x[arg])
        elif kind == "index" and isinstance(x, list) and arg < len(x):
            out.append(x[arg])
        else:
            break
    return out


SLICE_CASES = [
    ("$.a[-3:-1]", ["a"], -3, -1, None, 0),
    ("$.a[-5:-2].v", ["a"], -5, -2, ("key", "v"), 0),
    ("$.a[1:]", ["a"], 1, None, None, 4),
    ("$.a[0:]", ["a"], 0, None, None, 3),
    ("$.a[2:-1]", ["a"], 2, -1, None, 3),
    ("$.a[1:-3].v", ["a"], 1, -3, ("key", "v"), 5),
    ("$.a[:-2]", ["a"], 0, -2, None, 6),
    ("$.b.c[:-1][1]", ["b", "c"], 0, -1, ("index", 1), 3),
    ("$.b.c[1:][0]", ["b", "c"], 1, None, ("index", 0), 2),
    ("$.a[*]", ["a"], 0, None, None, 5),
]


@pytest.mark.parametrize("query,path,a,b,rest,k", SLICE_CASES)
def test_slices_from_the_end(gpj, arrays, query, path, a, b, rest, k):
    c = gpj.compile(query, wildcard_limit=k)
    ix = oracle.OracleIndex(arrays, c.max_depth)
    res = ix.query(c.ir_bytes, c.num_result_slots)
    got = _values(arrays, res)
    want, overflow = [], False
    for rec in _records(arrays):
        arr = _get(_loads(rec), path) if rec else None
        if not isinstance(arr, list):
            want.append([])
            continue
        n = len(arr)
        if a < 0:
            # reverse indexes -a .. -b-1: every one must exist
            sel = arr[n + a:n + b] if n >= -a else []
        else:
            end = n + b if b is not None else n
            sel = arr[a:end] if a < n else []
            overflow |= len(sel) > k
            sel = sel[:k]
        want.append(_apply(sel, rest))
    assert got == want
    assert sum(map(len, want)) > 100
    assert bool(ix.last_status & oracle.OracleIndex.STATUS_OVERFLOW) == overflow
