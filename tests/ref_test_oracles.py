"""Python restatements of the expected-value helpers in the reference's own
index tests, used to cross-check the C oracle on many inputs.

  expected_newline_index        tests/index/newline_index_test.cpp:27-35
  is_escaped_quote +
  expected_string_index         tests/index/string_index_test.cpp:28-59
  expected_leveled_bitmap_index tests/index/leveled_bitmap_index_test.cpp:57-92

Note the test helpers count the whole backslash run before a quote, while
the builders carry escape parity only from the previous 64-byte word; the two
agree unless a run of 64 or more backslashes exists.
"""
from __future__ import annotations

import numpy as np


def expected_newline_index(data: bytes) -> list[int]:
    return [0] + [i for i, c in enumerate(data) if c == 0x0A]


def is_escaped_quote(data: bytes, q: int) -> bool:
    k = 0
    i = q
    while i > 0 and data[i - 1] == 0x5C:
        k += 1
        i -= 1
    return k % 2 == 1


def expected_string_index(data: bytes) -> np.ndarray:
    words = np.zeros((len(data) + 63) // 64, np.uint64)
    in_string = False
    for i, c in enumerate(data):
        if c == 0x22 and not is_escaped_quote(data, i):
            if not in_string:
                words[i // 64] |= np.uint64(1 << (i % 64))
                in_string = True
            else:
                in_string = False
        elif in_string:
            words[i // 64] |= np.uint64(1 << (i % 64))
    return words


def expected_leveled_bitmap_index(data: bytes, num_levels: int) -> np.ndarray:
    W = (len(data) + 63) // 64
    s = expected_string_index(data)
    levels = np.zeros(W * num_levels, np.uint64)
    level = -1
    for i, c in enumerate(data):
        if int(s[i // 64]) >> (i % 64) & 1:
            continue
        bit = np.uint64(1 << (i % 64))
        if c in (0x7B, 0x5B):
            level += 1
            if 0 <= level < num_levels:
                levels[W * level + i // 64] |= bit
        elif c in (0x7D, 0x5D):
            if 0 <= level < num_levels:
                levels[W * level + i // 64] |= bit
            level -= 1
        elif c in (0x3A, 0x2C):
            if 0 <= level < num_levels:
                levels[W * level + i // 64] |= bit
    return levels
