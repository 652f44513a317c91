"""Extracts the known-answer vectors of the reference's own tests into
tests/golden/reference_kats.json.

Run in a checkout where the reference project is available (its path is the
first argument, else $GPJSON_REFERENCE_ROOT, else /root/reference).  Only the small literal fixtures and
expected values of the reference's unit tests are extracted:

  tests/index/newline_index_test.cpp        ComputesExpectedNewlineIndex
  tests/index/string_index_test.cpp         ComputesExpectedStringIndex
  tests/index/leveled_bitmap_index_test.cpp ComputesExpectedLeveledBitmapIndex
  tests/index/index_test_utils.hpp          ld_json_fixture, kMaxDepth
  tests/query/query_executor_test.cpp       bookstore record + expected values
  tests/engine_test.cpp                     two-record file + expected values
  tests/query/query_compiler_test.cpp       IR shapes, depths, slot counts,
                                            malformed / unsupported queries

The resulting JSON is committed; tests read it, never the reference.
"""
from __future__ import annotations

import json
import re
import sys
from pathlib import Path

OUT = Path(__file__).resolve().parent / "reference_kats.json"


def cpp_string_literals(src: str) -> str:
    """Concatenates the C++ string literals of `src` (plain and R"(...)")."""
    out = []
    i = 0
    while i < len(src):
        if src.startswith('R"(', i):
            j = src.index(')"', i + 3)
            out.append(src[i + 3:j])
            i = j + 2
        elif src[i] == '"':
            i += 1
            buf = []
            while src[i] != '"':
                c = src[i]
                if c == "\\":
                    n = src[i + 1]
                    buf.append({"n": "\n", "t": "\t", "\\": "\\", '"': '"', "'": "'",
                                "r": "\r", "0": "\0"}[n])
                    i += 2
                else:
                    buf.append(c)
                    i += 1
            out.append("".join(buf))
            i += 1
        else:
            i += 1
    return "".join(out)


def between(text: str, start: str, end: str) -> str:
    i = text.index(start) + len(start)
    return text[i:text.index(end, i)]


def main(ref: Path) -> None:
    t = ref / "tests"
    kats: dict = {"source": "Xinyu-Li-123/15418-project tests"}

    nl = (t / "index/newline_index_test.cpp").read_text()
    body = between(nl, "ComputesExpectedNewlineIndex", "}\n")
    kats["newline"] = {
        "cite": "tests/index/newline_index_test.cpp:64-69",
        "data": cpp_string_literals(between(body, "data =", ";")),
        "expected": [int(x) for x in re.findall(r"-?\d+", between(body, "oracle{", "}"))],
    }

    st = (t / "index/string_index_test.cpp").read_text()
    body = between(st, "ComputesExpectedStringIndex", "\n}\n")
    kats["string"] = {
        "cite": "tests/index/string_index_test.cpp:86-93",
        "data": cpp_string_literals(between(body, "data =", ";")),
        "expected": [int(x, 2) for x in re.findall(r"0b([01]+)", between(body, "oracles{", "}"))],
    }

    lb = (t / "index/leveled_bitmap_index_test.cpp").read_text()
    body = between(lb, "ComputesExpectedLeveledBitmapIndex", "\n}\n")
    words = re.findall(r"word_from_bits\((0b[01]+|\d+)\)", body)
    kats["leveled"] = {
        "cite": "tests/index/leveled_bitmap_index_test.cpp:123-131",
        "data": cpp_string_literals(between(body, "data =", ";")),
        "num_levels": int(re.search(r"expected_leveled_bitmap_index\(data, (\d+)\)", body).group(1)),
        "expected": [int(w, 0) for w in words],
    }

    ut = (t / "index/index_test_utils.hpp").read_text()
    kats["ld_json_fixture"] = {
        "cite": "tests/index/index_test_utils.hpp:80-89",
        "data": cpp_string_literals(between(ut, "return std::string{", "};")),
        "max_depth": int(re.search(r"kMaxDepth = (\d+);", ut).group(1)),
    }

    qe = (t / "query/query_executor_test.cpp").read_text()
    json_text = cpp_string_literals(between(qe, "const std::string json_text =", ";\n"))
    expect = re.findall(r'EXPECT_EQ\(materialized\.queries\(\)\[(\d)\]\.lines\(\)\[0\]\.values\(\)\[0\]\.json_text\(\),\s*"((?:[^"\\]|\\.)*)"\)', qe)
    kats["query_executor"] = {
        "cite": "tests/query/query_executor_test.cpp:155-195,215-245",
        "json_text": json_text,
        "queries": re.findall(r'compiler\.compile\("([^"]+)", options\)', qe),
        "expected": {int(i): cpp_string_literals('"' + v + '"') for i, v in expect},
        "unmatched_query": "$.store.magazine",
    }

    en = (t / "engine_test.cpp").read_text()
    contents = cpp_string_literals(between(en, '"gpjson_engine_partitioned.ldjson",', ");"))
    expect = re.findall(r'EXPECT_EQ\(result\.queries\(\)\[(\d)\]\.lines\(\)\[(\d)\]\.values\(\)\[0\]\.json_text\(\),\s*"((?:[^"\\]|\\.)*)"\)', en)
    kats["engine"] = {
        "cite": "tests/engine_test.cpp:18-58,89-129",
        "contents": contents,
        "queries": re.findall(r'^\s+"(\$[^"]+)",$', en, re.M)[:2],
        "file_partition_size": int(re.search(r"index_builder_type,\s*(\d+),", en).group(1)),
        "expected": [[int(q), int(l), cpp_string_literals('"' + v + '"')] for q, l, v in expect],
    }

    qc = (t / "query/query_compiler_test.cpp").read_text()
    cases = []
    for m in re.finditer(r"TEST\(QueryCompilerTest, (\w+)\) \{(.*?)\n\}", qc, re.S):
        name, body = m.group(1), m.group(2)
        case = {"name": name}
        comp = re.search(r'compiler\.compile\(\s*"((?:[^"\\]|\\.)*)", options\)', body)
        if "EXPECT_THROW" in body:
            case["throws"] = [
                [cpp_string_literals('"' + q + '"'), err]
                for q, err in re.findall(
                    r'EXPECT_THROW\(compiler\.compile\("((?:[^"\\]|\\.)*)", options\),\s*gpjson::error::query::(\w+)\)',
                    body)]
        else:
            case["query"] = cpp_string_literals('"' + comp.group(1) + '"')
            md = re.search(r"max_depth\(\), (\d+)U", body)
            ns = re.search(r"num_result_slots\(\), (\d+)U", body)
            ni = re.search(r"instructions\.size\(\), (\d+)U", body)
            case["max_depth"] = int(md.group(1))
            case["num_result_slots"] = int(ns.group(1))
            case["num_instructions"] = int(ni.group(1))
            ops = {}
            for i, op in re.findall(r"instructions\[(\d+)\]\.opcode, QueryOpcode::(\w+)", body):
                ops.setdefault(int(i), {})["opcode"] = op
            for i, s in re.findall(r'instructions\[(\d+)\]\.string_operand, "((?:[^"\\]|\\.)*)"', body):
                ops.setdefault(int(i), {})["string"] = cpp_string_literals('"' + s + '"')
            for i, v in re.findall(r"instructions\[(\d+)\]\.integer_operand, (\d+)U", body):
                ops.setdefault(int(i), {})["integer"] = int(v)
            case["instructions"] = {str(k): v for k, v in sorted(ops.items())}
        cases.append(case)
    kats["compiler"] = {"cite": "tests/query/query_compiler_test.cpp:58-147", "cases": cases}

    OUT.write_text(json.dumps(kats, indent=1, sort_keys=True) + "\n")
    print(f"wrote {OUT}")


if __name__ == "__main__":
    import os
    main(Path(sys.argv[1] if len(sys.argv) > 1 else
              os.environ.get("GPJSON_REFERENCE_ROOT", "/root/reference")))
