"""JSONPath compiler through the C ABI (host-only, runs without a GPU).

Known answers come from the reference's tests/query/query_compiler_test.cpp
(tests/golden/reference_kats.json); the rest restate the grammar of
src/gpjson/query/query_compiler.cpp.
"""
import json
from pathlib import Path

import pytest

KATS = json.loads((Path(__file__).parent / "golden" / "reference_kats.json").read_text())
OPS = {0: "END", 1: "STORE_RESULT", 2: "MOVE_UP", 3: "MOVE_DOWN", 4: "MOVE_TO_KEY",
       5: "MOVE_TO_INDEX", 6: "MOVE_TO_INDEX_REVERSE", 7: "MARK_POSITION",
       8: "RESET_POSITION", 9: "EXPRESSION_STRING_EQUALS",
       # extensions of this build (the reference rejects these queries)
       10: "NUMBER_COMPARE", 11: "DESCEND_KEY", 12: "EXPECT_AT_MOST", 13: "EXPECT_FOLLOWING"}
CMPS = {0: "==", 1: "!=", 2: "<", 3: "<=", 4: ">", 5: ">="}


def decode(ir: bytes):
    """IRByteInputBuffer restated: opcode, then varint / string operands."""
    out, i = [], 0

    def varint():
        nonlocal i
        v, shift = 0, 0
        while True:
            b = ir[i]
            i += 1
            v |= (b & 0x7F) << shift
            shift += 7
            if not b & 0x80:
                return v

    while i < len(ir):
        op = OPS[ir[i]]
        i += 1
        ins = {"opcode": op}
        if op == "NUMBER_COMPARE":
            ins["cmp"] = CMPS[ir[i]]
            i += 1
        if op in ("MOVE_TO_KEY", "EXPRESSION_STRING_EQUALS", "NUMBER_COMPARE", "DESCEND_KEY"):
            n = varint()
            ins["string"] = ir[i:i + n].decode()
            i += n
        elif op in ("MOVE_TO_INDEX", "MOVE_TO_INDEX_REVERSE", "EXPECT_AT_MOST",
                    "EXPECT_FOLLOWING"):
            ins["integer"] = varint()
        out.append(ins)
        if op == "END":
            break
    return out


@pytest.mark.parametrize("case", [c for c in KATS["compiler"]["cases"] if "query" in c],
                         ids=lambda c: c["name"])
def test_reference_ir_shapes(gpj, case):
    c = gpj.compile(case["query"])
    ins = decode(c.ir_bytes)
    assert c.query_text == case["query"]
    assert c.max_depth == case["max_depth"]
    assert c.num_result_slots == case["num_result_slots"]
    assert len(ins) == case["num_instructions"]
    for idx, want in case["instructions"].items():
        assert ins[int(idx)] == want


ERRS = {"MalformedQueryError": "MalformedQueryError",
        "UnsupportedQueryError": "UnsupportedQueryError"}


@pytest.mark.parametrize("query,err", [tuple(t) for c in KATS["compiler"]["cases"]
                                       for t in c.get("throws", [])])
def test_reference_rejections(gpj, query, err):
    with pytest.raises(getattr(gpj, err)):
        gpj.compile(query)


def test_error_messages_follow_reference_format(gpj):
    # "$." fails in peek() before the empty-property check
    with pytest.raises(gpj.MalformedQueryError, match=r"^Expected character, got EOF at 2$"):
        gpj.compile("$.")
    with pytest.raises(gpj.MalformedQueryError, match=r"^Unexpected empty property at 2 \('\['\)$"):
        gpj.compile("$.[0]")
    with pytest.raises(gpj.UnsupportedQueryError,
                       match=r"^Unsupported recursive descent at 2 \('\.'\)$"):
        gpj.compile("$..name")
    with pytest.raises(gpj.MalformedQueryError, match=r"Expected character '\$', got 'x'"):
        gpj.compile("x.a")
    with pytest.raises(gpj.UnsupportedQueryError, match="Unsupported expression type"):
        gpj.compile("$a")


def test_std_exceptions_for_stoull(gpj):
    with pytest.raises(ValueError):  # std::invalid_argument in the reference
        gpj.compile("$.a[1:]")
    with pytest.raises(OverflowError):  # std::out_of_range
        gpj.compile("$.a[99999999999999999999999]")


def test_bracket_property_and_index(gpj):
    ins = decode(gpj.compile("$['store'][\"book\"][2]").ir_bytes)
    assert ins == [{"opcode": "MOVE_TO_KEY", "string": "store"}, {"opcode": "MOVE_DOWN"},
                   {"opcode": "MOVE_TO_KEY", "string": "book"}, {"opcode": "MOVE_DOWN"},
                   {"opcode": "MOVE_TO_INDEX", "integer": 2}, {"opcode": "MOVE_DOWN"},
                   {"opcode": "STORE_RESULT"}, {"opcode": "END"}]


def test_index_list_and_reverse(gpj):
    c = gpj.compile("$.a[1,3].b")
    assert (c.max_depth, c.num_result_slots) == (3, 2)
    ops = [i["opcode"] for i in decode(c.ir_bytes)]
    assert ops == ["MOVE_TO_KEY", "MOVE_DOWN", "MOVE_TO_INDEX", "MOVE_DOWN", "MOVE_TO_KEY",
                   "MOVE_DOWN", "STORE_RESULT", "MOVE_UP", "MOVE_UP", "MOVE_TO_INDEX",
                   "MOVE_DOWN", "MOVE_TO_KEY", "MOVE_DOWN", "STORE_RESULT", "END"]
    r = gpj.compile("$.a[-2]")
    assert decode(r.ir_bytes)[2] == {"opcode": "MOVE_TO_INDEX_REVERSE", "integer": 2}
    rr = gpj.compile("$.a[-3:]")
    assert rr.num_result_slots == 3
    assert [i["integer"] for i in decode(rr.ir_bytes) if "integer" in i] == [3, 2, 1]
    with pytest.raises(gpj.UnsupportedQueryError):
        gpj.compile("$.a[--1]")


def test_large_varint(gpj):
    ins = decode(gpj.compile("$.a[300]").ir_bytes)
    assert ins[2] == {"opcode": "MOVE_TO_INDEX", "integer": 300}
    assert gpj.compile("$.a[300]").ir_bytes[5:7] == bytes([0xAC, 0x02])


def test_wildcard_extension_is_off_by_default(gpj):
    with pytest.raises(gpj.UnsupportedQueryError, match="Unsupported wildcard expression"):
        gpj.compile("$.entities.hashtags[*].text")
    w = gpj.compile("$.entities.hashtags[*].text", wildcard_limit=8)
    r = gpj.compile("$.entities.hashtags[0:8].text")
    # "[*]" = an element-count check, then the IR of "[0:8]" with an
    # element-exists check after each index step
    wi, ri = decode(w.ir_bytes), decode(r.ir_bytes)
    assert wi[4] == {"opcode": "EXPECT_AT_MOST", "integer": 8}
    checks = [i for i, x in enumerate(wi) if x["opcode"] == "EXPECT_FOLLOWING"]
    assert len(checks) == 8 and all(wi[i - 1]["opcode"] == "MOVE_TO_INDEX" and
                                     wi[i]["integer"] == 0 for i in checks)
    assert [x for i, x in enumerate(wi) if i != 4 and i not in checks] == ri
    assert (w.max_depth, w.num_result_slots) == (r.max_depth, r.num_result_slots)


def test_slices_from_the_end_compile(gpj):
    # "[-a:-b]": the reference's reverse-index IR, no extension opcode
    c = gpj.compile("$.a[-4:-1]")
    ins = decode(c.ir_bytes)
    assert [x["integer"] for x in ins if x["opcode"] == "MOVE_TO_INDEX_REVERSE"] == [4, 3, 2]
    assert (c.max_depth, c.num_result_slots) == (2, 3)
    assert not any(x["opcode"] in ("EXPECT_AT_MOST", "EXPECT_FOLLOWING") for x in ins)
    # open slices need the wildcard limit K: K branches, count check a+K+b
    c = gpj.compile("$.a[2:-3].b", wildcard_limit=4)
    ins = decode(c.ir_bytes)
    assert ins[2] == {"opcode": "EXPECT_AT_MOST", "integer": 9}
    assert [x["integer"] for x in ins if x["opcode"] == "MOVE_TO_INDEX"] == [2, 3, 4, 5]
    assert [x["integer"] for x in ins if x["opcode"] == "EXPECT_FOLLOWING"] == [3] * 4
    assert (c.max_depth, c.num_result_slots) == (3, 4)
    assert gpj.compile("$.a[:-1]", wildcard_limit=2).num_result_slots == 2
    assert gpj.compile("$.a[5:]", wildcard_limit=3).num_result_slots == 3
    # without K the reference's errors stand
    with pytest.raises(ValueError):
        gpj.compile("$.a[5:]")
    with pytest.raises(gpj.MalformedQueryError, match="expected an integer"):
        gpj.compile("$.a[:-1]")
    with pytest.raises(gpj.MalformedQueryError, match="Empty index range"):
        gpj.compile("$.a[-1:-2]")
    with pytest.raises(gpj.MalformedQueryError, match="Invalid reverse index 0"):
        gpj.compile("$.a[1:-0]", wildcard_limit=2)
    with pytest.raises(gpj.MalformedQueryError):
        gpj.compile("$.a[*-1]", wildcard_limit=2)
    with pytest.raises(gpj.UnsupportedQueryError, match="Unsupported last n elements"):
        gpj.compile("$.a[--1]", wildcard_limit=2)


def test_reference_syntax_never_uses_extension_opcodes(gpj):
    for case in KATS["compiler"]["cases"]:
        if "query" in case:
            assert all(ins["opcode"] not in ("NUMBER_COMPARE", "DESCEND_KEY", "EXPECT_AT_MOST",
                                             "EXPECT_FOLLOWING")
                       for ins in decode(gpj.compile(case["query"]).ir_bytes))


def test_recursive_descent_extension(gpj):
    with pytest.raises(gpj.UnsupportedQueryError, match="Unsupported recursive descent at 2"):
        gpj.compile("$..id")  # the reference's error without a slot limit
    c = gpj.compile("$..id", wildcard_limit=5)
    assert decode(c.ir_bytes) == [{"opcode": "DESCEND_KEY", "string": "id"}, {"opcode": "END"}]
    assert (c.num_result_slots, c.max_depth) == (5, 15)
    c = gpj.compile("$.user..id", wildcard_limit=3)
    assert [i["opcode"] for i in decode(c.ir_bytes)] == \
        ["MOVE_TO_KEY", "MOVE_DOWN", "DESCEND_KEY", "END"]
    assert c.num_result_slots == 3
    with pytest.raises(gpj.UnsupportedQueryError, match="after a recursive descent"):
        gpj.compile("$..a.b", wildcard_limit=3)
    with pytest.raises(gpj.MalformedQueryError, match="empty property"):
        gpj.compile("$..", wildcard_limit=3)


@pytest.mark.parametrize("text,cmp,lit", [("@ > 5", ">", "5"), ("@ >= -1.5e3", ">=", "-1.5e3"),
                                          ("@ < 0.25", "<", "0.25"), ("@ <= 0", "<=", "0"),
                                          ("@ != 12", "!=", "12"), ("@ == 7E+2", "==", "7E+2"),
                                          ("@.b > 3", ">", "3")])
def test_numeric_filter_extension(gpj, text, cmp, lit):
    c = gpj.compile(f"$.a[?({text})]")
    ins = decode(c.ir_bytes)
    i = [k for k, x in enumerate(ins) if x["opcode"] == "NUMBER_COMPARE"][0]
    assert ins[i] == {"opcode": "NUMBER_COMPARE", "cmp": cmp, "string": lit}
    assert ins[i + 1] == {"opcode": "RESET_POSITION"}
    assert ins[2] == {"opcode": "MARK_POSITION"}
    assert c.num_result_slots == 1


@pytest.mark.parametrize("query,err,msg", [
    ('$.a[?(@ > "x")]', "UnsupportedQueryError", "comparison of a string"),
    ("$.a[?(@ > 01)]", "MalformedQueryError", "Invalid number"),
    ("$.a[?(@ > 1.)]", "MalformedQueryError", "Invalid number"),
    ("$.a[?(@ > 1e)]", "MalformedQueryError", "Invalid number"),
    ("$.a[?(@ > +1)]", "MalformedQueryError", "Invalid number"),
    ("$.a[?(@ == x)]", "MalformedQueryError", "Invalid quoted string"),
    ("$.a[?(@ ~ 1)]", "UnsupportedQueryError", "Unsupported character for expression"),
])
def test_filter_errors(gpj, query, err, msg):
    with pytest.raises(getattr(gpj, err), match=msg):
        gpj.compile(query)
