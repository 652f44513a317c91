"""The CPU pre-check of the reference's device asserts (tests/ref_guard.py):
the inputs the reference-GPU parity test uses pass it, and inputs that would
trip each guarded assert are caught on the CPU."""
import numpy as np

import ref_guard


def test_well_formed_inputs_pass(gpj):
    from gpjson_b200 import datagen
    data = datagen.tweets(41, 1 << 20, deep=True)
    comp = [gpj.compile(q) for q in ["$.user.lang", "$.entities.hashtags[0:8].text",
                                     "$.retweeted_status.user.id", "$.user.lang[?(@ == \"en\")]"]]
    assert ref_guard.problems(data, comp, 4) == []


def test_all_backslash_word_is_caught(gpj):
    line = b'{"a":"' + b"x" * 58 + b"\\" * 64 + b'"}\n'  # 64 backslashes from byte 64
    assert not ref_guard.escape_chunks_ok(np.frombuffer(line, np.uint8))
    assert ref_guard.problems(line, [gpj.compile("$.a")], 1)
    ok = b'{"a":"' + b"x" * 59 + b"\\" * 62 + b'"}\n'  # a 62-byte run across two words
    assert ref_guard.escape_chunks_ok(np.frombuffer(ok, np.uint8))


def test_depth_below_top_is_caught():
    assert not ref_guard.depth_ok(np.frombuffer(b'{"a":1}}\n', np.uint8))
    assert ref_guard.depth_ok(np.frombuffer(b'{"a":"}}"}\n', np.uint8))  # inside a string
    deep = b"[" * 130 + b"]" * 130
    assert not ref_guard.depth_ok(np.frombuffer(deep, np.uint8))


def test_query_asserts_are_caught(gpj):
    data = b'{"a":5,"b":[],"c":"x"}\n{"a":"y","b":[1],"c":"z"}\n'
    # a string filter on a number (query.cu:430)
    assert ref_guard.problems(data, [gpj.compile('$.a[?(@ == "y")]')], 2)
    # a key search that lands on neither ':' nor '}' (query.cu:265)
    assert ref_guard.problems(b'{"a" , "b":1}\n', [gpj.compile("$.b")], 1)
    assert ref_guard.problems(data, [gpj.compile("$.c"), gpj.compile("$.b[0]")], 2) == []
