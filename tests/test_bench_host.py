"""Host-side helpers of bench.py that shape what is measured: the newline
partitions of inputs of 2 GiB and more (cut as the reference's engine cuts
files, file_reader.cpp:65-66: the separating newline belongs to neither
side), the algorithmic byte count of the index roofline, and the config-3
file sizes."""
import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parent.parent))
import bench  # noqa: E402


def test_newline_partitions_cover_input_without_separators():
    rng = np.random.default_rng(3)
    data = rng.choice(np.frombuffer(b"ab{}\n", np.uint8), size=5000, p=[.3, .3, .15, .15, .1])
    data[::30] = 10  # every window of the limits below holds a newline
    for limit in (40, 100, 777, 5000, 10**6):
        parts = bench.newline_partitions(data, limit)
        assert parts[0][0] == 0 and parts[-1][1] == data.size
        for (a0, a1), (b0, _) in zip(parts, parts[1:]):
            assert data[a1] == 10 and b0 == a1 + 1  # cut at a newline that neither side keeps
        for a0, a1 in parts:
            assert 0 <= a1 - a0 <= limit
        # every line survives: lines of all partitions = lines of the whole input
        lines = sum(int(np.count_nonzero(data[a0:a1] == 10)) + 1 for a0, a1 in parts)
        assert lines == int(np.count_nonzero(data == 10)) + 1


def test_record_longer_than_a_partition_is_an_error():
    data = np.frombuffer(b"x" * 100 + b"\n" + b"y" * 10, np.uint8)
    try:
        bench.newline_partitions(data, 50)
    except ValueError as e:
        assert "no newline" in str(e)
    else:
        raise AssertionError("expected ValueError")


def test_single_partition_below_the_limit():
    data = np.frombuffer(b'{"a":1}\n{"a":2}', np.uint8)
    assert bench.newline_partitions(data, bench.INT32_MAX) == [(0, data.size)]


def test_algorithmic_index_bytes():
    # input once + S + L leveled words + the newline index (int64)
    n, levels, lines = 1000, 4, 7
    W = (n + 63) // 64
    assert bench.algorithmic_index_bytes(n, levels, lines) == n + 8 * W * 5 + 8 * lines


def test_c3_sizes_match_the_spec():
    sizes = bench.c3_sizes(seed=3, total=8 << 30)
    assert sizes.size == 10_000
    assert sizes.min() >= 4 << 10 and sizes.max() <= 64 << 20
    assert abs(int(sizes.sum()) - (8 << 30)) < (64 << 20)


def test_cpu_baseline_parity_gate(gpj):
    """The single-input lines' parity gate: the oracle's results on the
    sample's newline partitions, shifted, equal the whole-input results, and a
    planted difference fails the line."""
    import oracle
    from gpjson_b200 import datagen
    data = datagen.tweets(5, 3 << 20)
    comp = bench.compile_all(gpj, ["$.user.lang", "$.entities.hashtags[*].text"])
    levels = max(c.max_depth + b for c, b in comp)
    ix = oracle.OracleIndex(data, levels)
    whole = [ix.query(c.ir_bytes, c.num_result_slots, b) for c, b in comp]
    base, parity = bench.cpu_baseline(data, comp, "lines", levels, 1.0, threads=3,
                                      results=whole)
    assert parity["mismatches"] == 0 and parity["records_checked"] >= 2 * (ix.num_lines - 1)
    bad = [w.copy() for w in whole]
    hit = np.argwhere(bad[0][:, 0, 0] >= 0).ravel()
    bad[0][hit[len(hit) // 2], 0, 1] += 1
    import pytest
    with pytest.raises(AssertionError, match="parity"):
        bench.cpu_baseline(data, comp, "lines", levels, 1.0, threads=3, results=bad)
