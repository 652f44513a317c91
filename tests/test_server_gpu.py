"""Serving loop (gpj_server): every request's results are the same when it
runs alone on the device and when it runs in a mix of concurrent requests
under a tight HBM budget (admission waits, evictions, resident-index hits,
shared builds), and both equal the CPU oracle bit for bit."""
import random

import numpy as np
import pytest
import torch

import oracle

pytestmark = pytest.mark.gpu

TWEET_QUERIES = ["$.user.lang", "$.entities.hashtags[*].text", "$.place.country_code",
                 "$.retweeted_status.user.id", "$.user"]
ARRAY_QUERIES = ["$[*].categoryPath[1:3].id", "$[*].sku"]


def _need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("CUDA device required")


def _compiled(gpj):
    out = {}
    for q in TWEET_QUERIES:
        c = gpj.compile(q, wildcard_limit=8)
        out[q] = (c, 0, c.max_depth)
    for q in ARRAY_QUERIES:
        c = gpj.compile(q.replace("$[*]", "$"), wildcard_limit=8)
        out[q] = (c, 1, c.max_depth + 1)
    return out


def _files():
    from gpjson_b200 import datagen
    rng = random.Random(7)
    files = [np.zeros(0, np.uint8), np.frombuffer(b"\n", np.uint8).copy()]
    sizes = [100, 4000, 33000, 70000, 300000, 1 << 20, 3 << 20] + [1 << 20] * 6
    for i, size in enumerate(sizes):
        files.append(("t", np.array(datagen.tweets(100 + i, size, deep=(i % 2 == 1)))))
    for i, size in enumerate([5000, 200000]):
        files.append(("a", np.array(datagen.products(200 + i, size))))
    junk = bytes(rng.choices(b'{}[]:,"\\\n ab', k=50000))
    files.append(("t", np.frombuffer(junk, np.uint8).copy()))
    out = []
    for f in files:
        if isinstance(f, tuple):
            out.append(f)
        else:
            out.append(("t", f))
    return out


def _requests(files, compiled, count, seed):
    rng = random.Random(seed)
    reqs = []
    for i in range(count):
        fi = i if i < len(files) else rng.randrange(len(files))
        kind, data = files[fi]
        pool = TWEET_QUERIES if kind == "t" else ARRAY_QUERIES
        qs = rng.sample(pool, rng.randint(1, min(3, len(pool))))
        reqs.append((fi + 1, data, [compiled[q] for q in qs], qs))
    return reqs


def _run(server, reqs, one_at_a_time):
    out = {}
    if one_at_a_time:
        for i, (key, data, qs, _) in enumerate(reqs):
            rid = server.submit(data, qs, file_key=key)
            server.wait(rid)
            out[i] = server.response(rid)
        return out
    order = list(range(len(reqs)))
    random.Random(1).shuffle(order)
    ids = {}
    for i in order:
        key, data, qs, _ = reqs[i]
        ids[server.submit(data, qs, file_key=key)] = i
    pending = set(ids)
    while pending:
        for rid in server.poll(timeout_us=2_000_000):
            pending.discard(rid)
            out[ids[rid]] = server.response(rid)
    return out


def _oracle(data, c, base, levels):
    ix = oracle.OracleIndex(bytes(data), levels)
    return ix.query(c.ir_bytes, c.num_result_slots, base)


def test_results_same_alone_and_in_mix(gpj):
    _need_gpu()
    compiled = _compiled(gpj)
    files = _files()
    reqs = _requests(files, compiled, 60, seed=3)
    with gpj.Server(num_slots=1, hbm_budget_bytes=256 << 20, flags=gpj.GPJ_SERVER_NO_CACHE) as s:
        alone = _run(s, reqs, one_at_a_time=True)
    # 16 MiB of device memory: the largest request (3 MiB file, up to ten
    # result slots) needs about 14 MB on its own, and the resident indexes of
    # all files (every file is requested) need about 19 MB, so admission has to
    # wait for memory and evict resident indexes
    with gpj.Server(num_slots=8, hbm_budget_bytes=16 << 20) as s:
        mixed = _run(s, reqs, one_at_a_time=False)
        st = s.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    checked = set()
    for i, (key, data, qs, names) in enumerate(reqs):
        a, m = alone[i], mixed[i]
        assert a.status == 0 and m.status == 0, (a.message, m.message)
        assert a.num_lines == m.num_lines
        for qa, qm in zip(a.results, m.results):
            np.testing.assert_array_equal(qa, qm, err_msg=f"request {i}")
        for (c, base, lv), name, got in zip(qs, names, a.results):
            if (key, name) in checked:
                continue
            checked.add((key, name))
            np.testing.assert_array_equal(got.astype(np.int64), _oracle(data, c, base, lv),
                                          err_msg=f"file {key} {name}")
        assert m.arrival_ns <= m.admit_ns <= m.index_ready_ns <= m.done_ns
    assert st["cache_hits"] > 0 and st["evictions"] > 0, st


def test_shared_build_and_resident_hits(gpj):
    _need_gpu()
    from gpjson_b200 import datagen
    c = gpj.compile("$.user.lang")
    q = [(c, 0, c.max_depth)]
    data = np.array(datagen.tweets(9, 2 << 20))
    with gpj.Server(num_slots=8, hbm_budget_bytes=256 << 20) as s:
        ids = [s.submit(data, q, file_key=42) for _ in range(6)]
        res = [None] * 6
        for k, rid in enumerate(ids):
            s.wait(rid)
            res[k] = s.response(rid)
        st = s.stats()
        assert st["cache_misses"] == 1 and st["cache_hits"] == 5
        assert st["bytes_indexed"] == data.size and st["resident_indexes"] == 1
        later = s.submit(data, q, file_key=42)
        s.wait(later)
        r = s.response(later)
        assert r.cache_hit and s.stats()["bytes_indexed"] == data.size
        # a deeper query than the resident levels rebuilds that key
        deep = gpj.compile("$.retweeted_status.user.id.a.b")
        rid = s.submit(data, [(deep, 0, deep.max_depth)], file_key=42)
        s.wait(rid)
        assert not s.response(rid).cache_hit
        s.clear_cache()
        assert s.stats()["resident_indexes"] == 0
    want = _oracle(data, c, 0, c.max_depth)
    for x in res + [r]:
        np.testing.assert_array_equal(x.results[0].astype(np.int64), want)


def test_truncated_newline_index_is_rebuilt(gpj):
    _need_gpu()
    data = np.frombuffer(b'{"a":1}\n{}\n' * 20000, np.uint8).copy()
    c = gpj.compile("$.a")
    with gpj.Server(num_slots=2, hbm_budget_bytes=64 << 20) as s:
        rid = s.submit(data, [(c, 0, c.max_depth)], file_key=5)
        s.wait(rid)
        r = s.response(rid)
        assert r.status == 0 and s.stats()["rebuilds"] == 1
    assert r.num_lines == 40001
    np.testing.assert_array_equal(r.results[0].astype(np.int64), _oracle(data, c, 0, 1))


def test_oversized_request_fails_and_others_finish(gpj):
    _need_gpu()
    from gpjson_b200 import datagen
    c = gpj.compile("$.user.lang")
    q = [(c, 0, c.max_depth)]
    big = np.array(datagen.tweets(1, 8 << 20))
    small = np.array(datagen.tweets(2, 64 << 10))
    with gpj.Server(num_slots=4, hbm_budget_bytes=4 << 20) as s:
        a = s.submit(big, q, file_key=1)
        b = s.submit(small, q, file_key=2)
        s.wait(a)
        s.wait(b)
        ra, rb = s.response(a), s.response(b)
    assert ra.status == gpj.GPJ_ERR_OOM and "budget" in ra.message
    assert rb.status == 0
    np.testing.assert_array_equal(rb.results[0].astype(np.int64), _oracle(small, c, 0, 2))


def test_grouped_builds_equal_single_builds(gpj):
    """Cache misses admitted in one scheduler pass are indexed by one
    multi-file launch over the arena: fewer index launches than builds, and
    every result equals a server that builds each file alone (and the
    oracle), including a group whose shared newline block is too small (a
    file of very short lines) and empty files."""
    _need_gpu()
    compiled = _compiled(gpj)
    files = _files()
    files.append(("t", np.frombuffer(b'{"a":1}\n{}\n' * 20000, np.uint8).copy()))
    reqs = _requests(files, compiled, 40, seed=11)

    def run(flags):
        with gpj.Server(num_slots=32, hbm_budget_bytes=512 << 20, flags=flags) as s:
            got = _run(s, reqs, one_at_a_time=False)
            return got, s.stats()

    grouped, st_g = run(0)
    alone, st_a = run(gpj.GPJ_SERVER_NO_GROUPS)
    assert st_g["index_launches"] < st_g["cache_misses"], st_g
    assert st_a["index_launches"] >= st_a["cache_misses"] - 2, st_a  # empty files launch nothing
    assert st_g["failed"] == st_a["failed"]
    for i, (key, data, qs, names) in enumerate(reqs):
        g, a = grouped[i], alone[i]
        # the random-structure file can hold an array longer than the "[*]"
        # limit: that request fails with the same status in both modes
        assert g.status == a.status, (i, g.message, a.message)
        assert g.status in (0, gpj.GPJ_ERR_CAPACITY), g.message
        if g.status:
            continue
        assert g.num_lines == a.num_lines
        for (c, base, lv), qg, qa in zip(qs, g.results, a.results):
            np.testing.assert_array_equal(qg, qa, err_msg=f"request {i}")
    for fi, (kind, data) in enumerate(files):
        for i, (key, d, qs, names) in enumerate(reqs):
            if key == fi + 1 and grouped[i].status == 0:
                c, base, lv = qs[0]
                np.testing.assert_array_equal(grouped[i].results[0].astype(np.int64),
                                              _oracle(data, c, base, lv), err_msg=f"file {fi}")
                break


def test_overflow_status_per_request(gpj):
    """In a batched query launch each (request, query) pair has its own
    status word: only the request whose "[*]" array outgrows its limit fails
    (GPJ_ERR_CAPACITY); the others in the same pass succeed."""
    _need_gpu()
    from gpjson_b200 import datagen
    data = np.array(datagen.tweets(12, 1 << 20))
    short = gpj.compile("$.entities.hashtags[*].text", wildcard_limit=2)
    full = gpj.compile("$.entities.hashtags[*].text", wildcard_limit=8)
    lang = gpj.compile("$.user.lang")
    L = full.max_depth
    with gpj.Server(num_slots=8, hbm_budget_bytes=256 << 20) as s:
        ids = [s.submit(data, [(full, 0, L)], file_key=1),
               s.submit(data, [(lang, 0, L), (short, 0, L)], file_key=1),
               s.submit(data, [(lang, 0, L)], file_key=1)]
        for rid in ids:
            s.wait(rid)
        rs = [s.response(rid) for rid in ids]
    assert rs[0].status == 0 and rs[2].status == 0
    assert rs[1].status == gpj.GPJ_ERR_CAPACITY and "result slots" in rs[1].message
    np.testing.assert_array_equal(rs[0].results[0].astype(np.int64), _oracle(data, full, 0, L))
    np.testing.assert_array_equal(rs[2].results[0].astype(np.int64), _oracle(data, lang, 0, L))


def test_truncated_group_newline_block_rebuilds_members(gpj):
    """A pass whose files together hold more newlines than the group's shared
    newline block (every file made of very short lines) rebuilds each member
    alone with its exact line count; results equal the oracle's."""
    _need_gpu()
    c = gpj.compile("$.a")
    q = [(c, 0, c.max_depth)]
    datas = [np.frombuffer((b'{"a":%d}\n{}\n' % k) * (15000 + 1000 * k), np.uint8).copy()
             for k in range(4)]
    with gpj.Server(num_slots=8, hbm_budget_bytes=256 << 20) as s:
        ids = [s.submit(d, q, file_key=k + 1) for k, d in enumerate(datas)]
        for rid in ids:
            s.wait(rid)
        rs = [s.response(rid) for rid in ids]
        st = s.stats()
    assert st["rebuilds"] >= 1 and st["failed"] == 0, st
    for d, r in zip(datas, rs):
        assert r.status == 0 and r.num_lines == d.tobytes().count(b"\n") + 1
        np.testing.assert_array_equal(r.results[0].astype(np.int64), _oracle(d, c, 0, 1))


def test_submit_many_queues_all_at_once(gpj):
    """gpj_server_submit_many: one call queues a whole request table; every
    result equals the oracle's, and a bad entry queues nothing."""
    _need_gpu()
    compiled = _compiled(gpj)
    files = _files()
    reqs = _requests(files, compiled, 30, seed=5)
    with gpj.Server(num_slots=16, hbm_budget_bytes=256 << 20) as s:
        with pytest.raises(ValueError):  # a request without queries
            s.submit_prepared(s.prepare([(reqs[0][1], [], 1, 0)]))
        assert s.stats()["submitted"] == 0
        ids = s.submit_prepared(s.prepare([(d, qs, key, 0) for key, d, qs, _ in reqs]))
        out = {}
        for i, rid in enumerate(ids):
            s.wait(rid)
            out[i] = s.response(rid)
    for i, (key, data, qs, names) in enumerate(reqs):
        if out[i].status == gpj.GPJ_ERR_CAPACITY:
            continue  # the random-structure file may outgrow a "[*]" limit
        assert out[i].status == 0, out[i].message
        for (c, base, lv), got in zip(qs, out[i].results):
            np.testing.assert_array_equal(got.astype(np.int64), _oracle(data, c, base, lv))
