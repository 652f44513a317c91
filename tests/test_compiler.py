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
       8: "RESET_POSITION", 9: "EXPRESSION_STRING_EQUALS"}


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
        if op in ("MOVE_TO_KEY", "EXPRESSION_STRING_EQUALS"):
            n = varint()
            ins["string"] = ir[i:i + n].decode()
            i += n
        elif op in ("MOVE_TO_INDEX", "MOVE_TO_INDEX_REVERSE"):
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
    with pytest.raises(gpj.UnsupportedQueryError):
        gpj.compile("$.entities.hashtags[*].text")
    w = gpj.compile("$.entities.hashtags[*].text", wildcard_limit=8)
    r = gpj.compile("$.entities.hashtags[0:8].text")
    assert (w.ir_bytes, w.max_depth, w.num_result_slots) == \
        (r.ir_bytes, r.max_depth, r.num_result_slots)
