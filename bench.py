"""Benchmark: GpJSON index + query throughput on B200 (one JSON line on stdout).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload c1|c0|c2|c3|c4]

A step is one pass of the hot path over the workload: the fused structural
index build of the whole input plus every query of the workload, with the
input already resident in device memory.  `value` is input GB (1e9 B) per
second over all ranks; `e2e` is the same metric through the public C ABI
call that takes host buffers (gpj_query_host: H2D of the input, index, all
queries, D2H of every result array) from pinned memory.

Workloads (seeded synthetic stand-ins for the GpJSON datasets):
  c1  one 1 GiB top-level array of ~2 KiB product records, one element per
      line; query $[*].categoryPath[1:3].id
  c0  64 MiB NDJSON of ~2 KiB post records; query $.user.lang
  c2  4 GiB NDJSON post records (deeper nesting); four queries over one index
  c3  10,000 files (8 GiB) batched in one captured launch chain vs one
      launch chain per file; the default run appends a 2 s c4 serving trace
  c4  serving: Poisson request trace through gpj_server, p50/p99 latency,
      with and without resident-index reuse

Multi-GPU (--gpus N under torchrun): the path has no exchange step, so each
rank runs an independent replica of the workload ("scaling": "weak") and the
timed region is the max over ranks.

--impl reference times the reference algorithm's CPU restatement (the
oracle: the reference project has no CPU implementation of this path) on the
host cores, on a bounded sample of the same workload per step.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

# the serving workload runs up to 32 streams at once: give them their own
# hardware queues (the default is 8)
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

sys.path.insert(0, str(ROOT / "tests"))
import __graft_entry__ as entry  # noqa: E402

METRIC = "index+query GB/s"
L2_BYTES = 126 * 1024 * 1024


def workload(name: str, pkg, size_mib: int | None = None):
    dg = pkg.datagen
    if size_mib:
        # profiling runs: the same generator and query at another size
        sz = size_mib << 20
        if name == "c1":
            return (dg.products(1, sz), ["$[*].categoryPath[1:3].id"], "array",
                    f"c1 generator at {size_mib} MiB, $[*].categoryPath[1:3].id")
        return (dg.tweets(0, sz), ["$.user.lang"], "lines",
                f"c0 generator at {size_mib} MiB, $.user.lang")
    if name == "c0":
        data = dg.tweets(0, 64 << 20)
        queries, records = ["$.user.lang"], "lines"
        desc = "c0: 64 MiB NDJSON post records (~2 KiB, depth<=6), $.user.lang"
    elif name == "c1":
        data = dg.products(1, 1 << 30)
        queries, records = ["$[*].categoryPath[1:3].id"], "array"
        desc = ("c1: 1 GiB single top-level array of ~2 KiB product records, "
                "$[*].categoryPath[1:3].id")
    elif name == "c3":
        raise SystemExit("c3 is a batch workload: see run_batch")
    elif name == "c2":
        data = dg.tweets(2, 4 << 30, deep=True)
        queries = ["$.user.lang", "$.entities.hashtags[*].text", "$.place.country_code",
                   "$.retweeted_status.user.id"]
        records = "lines"
        desc = "c2: 4 GiB NDJSON post records (depth<=8), 4 queries over one index"
    else:
        raise SystemExit(f"unknown workload {name}")
    return data, queries, records, desc


def c3_sizes(seed: int = 3, count: int = 10_000, total: int = 8 << 30,
             lo: int = 4 << 10, hi: int = 64 << 20, sigma: float = 2.0):
    """File sizes: ln(size) ~ N(mu, sigma) truncated to [lo, hi], mu solved so
    that the truncated mean is total / count."""
    from math import erf, exp, log, sqrt

    def phi(x):
        return 0.5 * (1.0 + erf(x / sqrt(2.0)))

    def tmean(mu):
        a, b = (log(lo) - mu) / sigma, (log(hi) - mu) / sigma
        return exp(mu + sigma * sigma / 2) * (phi(b - sigma) - phi(a - sigma)) / (phi(b) - phi(a))

    target = total / count
    m0, m1 = log(lo), log(hi)
    for _ in range(100):
        mid = 0.5 * (m0 + m1)
        if tmean(mid) < target:
            m0 = mid
        else:
            m1 = mid
    rng = np.random.default_rng(seed)
    out = []
    while len(out) < count:
        x = rng.lognormal(0.5 * (m0 + m1), sigma, size=count)
        out.extend(int(v) for v in x if lo <= v <= hi)
    sizes = np.array(out[:count], np.int64)
    sizes[-1] = int(np.clip(sizes[-1] + (total - sizes.sum()), lo, hi))
    return sizes


C3_DESC = ("c3: 10,000 seeded files, log-normal sizes 4 KiB-64 MiB, half NDJSON post records "
           "($.user.lang), half product arrays ($[*].categoryPath[1:3].id), one captured "
           "launch chain")
C3_QUERIES = ["$.user.lang", "$[*].categoryPath[1:3].id"]


def c3_shard_seeds(rank: int) -> tuple[int, int]:
    """Seeds of one rank's shard of config 3: (size-distribution seed, base
    seed of its file contents).  Rank 0 is the single-GPU workload; every
    other rank gets its own 10,000 files (multi-GPU runs shard distinct files
    over the ranks, weak scaling)."""
    return 3 + 1000 * rank, 10_000_000 * rank


def c3_files(pkg, scale: float = 1.0, limit_bytes: int | None = None, rank: int = 0):
    """10,000 seeded files (even: NDJSON post records, odd: product arrays);
    with limit_bytes only the leading files up to that many bytes."""
    size_seed, base = c3_shard_seeds(rank)
    sizes = c3_sizes(seed=size_seed, total=int((8 << 30) * scale))
    if limit_bytes is not None:
        keep = int(np.searchsorted(np.cumsum(sizes), limit_bytes)) + 1
        sizes = sizes[:keep]
    dg = pkg.datagen

    def make(i):
        n = int(sizes[i])
        if i % 2 == 0:
            return bytes(dg.tweets(base + 3_000_000 + i, n)), 0
        return bytes(dg.products(base + 4_000_000 + i, n)), 1

    with cf.ThreadPoolExecutor(os.cpu_count() or 4) as pool:
        return list(pool.map(make, range(len(sizes))))


C4_QUERIES = ["$.user.lang", "$.entities.hashtags[*].text", "$.place.country_code",
              "$.retweeted_status.user.id"]


def c4_trace(pkg, seed: int = 4, rate: float = 2000.0, duration_s: float = 4.0,
             repeat: float = 0.3, lo: int = 16 << 10, hi: int = 256 << 20,
             median: int = 256 << 10, sigma: float = 1.5, corpus_bytes: int = 1 << 30):
    """Serving trace: Poisson arrivals at `rate` for `duration_s`; each request
    names a file (30% repeats of an earlier file, else a new one whose size is
    log-normal around `median`, truncated to [lo, hi]) and 1-3 queries of the
    c2 set.  Files are newline-aligned slices of one seeded NDJSON corpus of
    post records (depth <= 8).  Returns (corpus, files [(offset, size)],
    requests [(arrival_s, file, [query indices])])."""
    dg = pkg.datagen
    chunk = 64 << 20
    with cf.ThreadPoolExecutor(os.cpu_count() or 4) as pool:
        parts = list(pool.map(lambda i: dg.tweets(5_000_000 + i, chunk, deep=True),
                              range(max(1, corpus_bytes // chunk))))
    corpus = np.concatenate(parts)
    nls = np.flatnonzero(corpus == 10)
    rng = np.random.default_rng(seed)
    count = int(rate * duration_s)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, count))
    hi = min(hi, corpus.size // 2)
    files, reqs = [], []
    for t in arrivals:
        if files and rng.random() < repeat:
            f = int(rng.integers(len(files)))
        else:
            while True:
                size = int(np.exp(rng.normal(np.log(median), sigma)))
                if lo <= size <= hi:
                    break
            off = int(rng.integers(0, corpus.size - size))
            k = int(np.searchsorted(nls, off))
            start = int(nls[k]) + 1 if k < nls.size else 0
            k2 = int(np.searchsorted(nls, start + size))
            end = int(nls[min(k2, nls.size - 1)]) + 1
            files.append((start, max(0, end - start)))
            f = len(files) - 1
        nq = int(rng.integers(1, 4))
        reqs.append((float(t), f, sorted(int(x) for x in rng.choice(4, nq, replace=False))))
    return corpus, files, reqs


def run_serving(args, world, rank, local, duration_s: float | None = None):
    """c4: the serving loop (gpj_server) fed a Poisson request trace in real
    time, with and without resident-index reuse, plus the same requests all
    submitted at once (saturated throughput).  Latency = result on the host
    minus scheduled arrival."""
    import torch
    pkg = entry.package()
    pkg.load_library()
    duration = duration_s if duration_s is not None else args.serve_seconds
    corpus, files, reqs = c4_trace(pkg, duration_s=duration)
    torch.cuda.set_device(local)
    pinned = torch.from_numpy(corpus).pin_memory()
    view = pinned.numpy()
    comp = [(c, 0, c.max_depth) for c, _ in compile_all(pkg, C4_QUERIES)]
    budget = min(120 * 10**9, int(torch.cuda.mem_get_info(local)[0] * 0.8))

    def arm(cache: bool, realtime: bool, grouped: bool = True):
        flags = (0 if cache else pkg.GPJ_SERVER_NO_CACHE) | \
            (0 if grouped else pkg.GPJ_SERVER_NO_GROUPS)
        srv = pkg.Server(local, num_slots=32, hbm_budget_bytes=budget,
                         host_result_bytes=2 << 30, cache_levels=4, flags=flags)
        ids = []
        t0 = time.monotonic_ns() + 20_000_000
        if realtime:
            for t, f, qs in reqs:
                off, size = files[f]
                target = t0 + int(t * 1e9)
                while time.monotonic_ns() < target:
                    pass
                ids.append(srv.submit(view[off:off + size], [comp[q] for q in qs],
                                      file_key=f + 1, arrival_ns=target))
        else:
            # saturated: every request at once, queued by one C call (the
            # request table is built beforehand, so the host loop of this
            # harness is not what is measured)
            prepared = srv.prepare([(view[files[f][0]:files[f][0] + files[f][1]],
                                     [comp[q] for q in qs], f + 1, 0) for _, f, qs in reqs])
            ids = srv.submit_prepared(prepared)
        pending = set(ids)
        while pending:
            for rid in srv.poll(timeout_us=1_000_000):
                pending.discard(rid)
        out = [srv.response(rid, release=False, copy_results=False) for rid in ids]
        sample = {rid: srv.response(rid, release=False).results for rid in ids[:: max(1, len(ids) // 200)]}
        st = srv.stats()
        srv.close()
        assert all(r.status == 0 for r in out), [r.message for r in out if r.status][:3]
        lat = np.array([r.done_ns - r.arrival_ns for r in out], np.float64) / 1e6
        span = (max(r.done_ns for r in out) - min(r.arrival_ns for r in out)) / 1e9
        served = sum(files[f][1] for _, f, _ in reqs)
        return {
            "p50_ms": round(float(np.percentile(lat, 50)), 4),
            "p99_ms": round(float(np.percentile(lat, 99)), 4),
            "mean_ms": round(float(lat.mean()), 4),
            "req_s": round(len(reqs) / span, 1), "gbs": round(served / span / 1e9, 3),
            "cache_hits": int(st["cache_hits"]), "bytes_indexed": int(st["bytes_indexed"]),
            "arena_peak_bytes": int(st["arena_peak"]),
            "index_builds": int(st["cache_misses"] + st["rebuilds"]),
            "index_launches": int(st["index_launches"]),
            "d2h_bytes": int(sum(r.result_ints for r in out)) * 4,
        }, sample

    # warm-up: a throwaway server runs the first requests (module loading,
    # first launches of each kernel variant, pinned-page mapping)
    warm = reqs[:256]
    srv = pkg.Server(local, num_slots=32, hbm_budget_bytes=min(budget, 8 << 30))
    for _ in range(3):
        ids = [srv.submit(view[files[f][0]:files[f][0] + files[f][1]], [comp[q] for q in qs],
                          file_key=f + 1) for _, f, qs in warm]
        for rid in ids:
            srv.wait(rid)
            srv.release(rid)
    srv.close()

    rt_reuse, s1 = arm(True, True)
    rt_plain, s2 = arm(False, True)
    sat_reuse, _ = arm(True, False)
    sat_plain, _ = arm(False, False)
    sat_ungrouped, _ = arm(True, False, grouped=False)
    for rid in s1:
        for a, b in zip(s1[rid], s2[rid]):
            assert np.array_equal(a, b), "results differ with and without index reuse"
    served = sum(files[f][1] for _, f, _ in reqs)
    return {
        "workload": f"c4: Poisson {len(reqs) / duration:.0f} req/s for {duration:g} s, "
                    f"{len(reqs)} requests over {len(files)} files (log-normal 16 KiB-256 MiB, "
                    "median 256 KiB, 30% repeats), 1-3 of the c2 queries each",
        "requests": len(reqs), "files": len(files), "bytes_requested": served,
        "hbm_budget_bytes": budget, "slots": 32,
        "realtime": {"reuse": rt_reuse, "no_reuse": rt_plain},
        "saturated": {"reuse": sat_reuse, "no_reuse": sat_plain,
                      "reuse_one_launch_per_build": sat_ungrouped},
        "batching": "cache misses admitted in one scheduler pass share one indexer launch",
        "latency": "host-observed: result copied to pinned host memory minus scheduled arrival",
    }


def compile_all(pkg, queries):
    """Compiles the workload queries; "$[*]..." selects array elements as records
    (bitmap level offset 1) and "[*]" inside a path expands to [0:8]."""
    out = []
    for q in queries:
        base = 0
        text = q
        if q.startswith("$[*]"):
            base, text = 1, "$" + q[4:]
        out.append((pkg.compile(text, wildcard_limit=8), base))
    return out


class ClockSampler:
    """Polls SM clocks and throttle reasons through NVML in a background
    thread for the whole timed region (about one sample per millisecond)."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
               "hw_thermal_slowdown": 0x40, "sw_power_cap": 0x4}

    def __init__(self, device: int):
        self.device = device
        self.samples: list[tuple[int, int]] = []
        self.max_mhz = None
        self.ok = False

    def start(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            vis = os.environ.get("CUDA_VISIBLE_DEVICES")
            idx = int(vis.split(",")[self.device]) if vis else self.device
            self.h = pynvml.nvmlDeviceGetHandleByIndex(idx)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.nv = pynvml
            self.ok = True
        except Exception:
            self.ok = False
            return
        self.stop_flag = threading.Event()
        self.t = threading.Thread(target=self._run, daemon=True)
        self.t.start()

    def _run(self):
        nv = self.nv
        while not self.stop_flag.is_set():
            try:
                mhz = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
                rs = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                self.samples.append((mhz, rs))
            except Exception:
                pass
            time.sleep(0.001)

    def stop(self) -> dict:
        if not self.ok:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvml unavailable"]}
        self.stop_flag.set()
        self.t.join()
        reasons = sorted({k for _, rs in self.samples for k, bit in self.REASONS.items()
                          if rs & bit})
        mhz = [m for m, _ in self.samples]
        return {"sm_mhz": float(np.median(mhz)) if mhz else None, "sm_max_mhz": self.max_mhz,
                "reasons": reasons, "samples": len(mhz)}


def measured_peak_hbm() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def dist_init():
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def allreduce_max(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def allreduce_sum(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


INT32_MAX = 0x7FFFFFFF


def newline_partitions(data, limit: int):
    """[start, end) byte ranges below `limit` bytes, cut after a newline that
    is left out of both sides (reference file_reader.cpp:65-66)."""
    n = int(data.size)
    parts, start = [], 0
    while n - start > limit:
        nls = np.flatnonzero(data[start:start + limit] == 10)
        if nls.size == 0:
            raise ValueError(f"no newline within {limit} bytes of offset {start}: "
                             "a record longer than a partition")
        cut = start + int(nls[-1])
        parts.append((start, cut))
        start = cut + 1
    parts.append((start, n))
    return parts


def algorithmic_index_bytes(n: int, levels: int, lines: int) -> int:
    # input read once + S + L leveled words + newline index (int64)
    W = (n + 63) // 64
    return n + 8 * W * (1 + levels) + 8 * lines


def run_ours(args, world, rank, local):
    import torch
    pkg = entry.package()
    pkg.load_library()
    data, queries, records, desc = workload(args.workload, pkg, args.size_mib)
    comp = compile_all(pkg, queries)
    levels = max(c.max_depth + base for c, base in comp)
    n = int(data.size)
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(device=dev)
    ctx = pkg.Context(local)
    d_in = torch.from_numpy(data).to(dev)
    W = (n + 63) // 64
    S = torch.empty(W, dtype=torch.int64, device=dev)
    LB = torch.empty(W * levels, dtype=torch.int64, device=dev)
    nl_cap = n // 32 + 1024
    NL = torch.empty(nl_cap, dtype=torch.int64, device=dev)
    summ = torch.zeros(4, dtype=torch.int64, device=dev)
    ix = pkg.Index()
    ix.d_string, ix.d_leveled = S.data_ptr(), LB.data_ptr()
    ix.d_newline, ix.newline_capacity = NL.data_ptr(), nl_cap
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.int32, device=dev) if n < 2 * L2_BYTES \
        else None
    s = stream.cuda_stream

    # one build to learn the record count and size the result buffers
    with torch.cuda.stream(stream):
        ctx.build_index_async(d_in.data_ptr(), n, levels, ix, summ.data_ptr(), stream=s)
    stream.synchronize()
    lines = int(summ[0].item())
    assert lines <= nl_cap and int(summ[3].item()) == 0
    ix.num_lines = lines
    # partitions of 2 GiB and more need int64 offsets (the reference's int
    # results stop below 2 GiB, query_executor_host.cu:28-33)
    wide = n > INT32_MAX
    outs = [torch.empty(lines * c.num_result_slots * 2,
                        dtype=torch.int64 if wide else torch.int32, device=dev)
            for c, _ in comp]

    def step(ev=None):
        # ev: [start, index done, query 0 done, query 1 done, ...]
        if ev is not None:
            ev[0].record(stream)
        ctx.build_index_async(d_in.data_ptr(), n, levels, ix, summ.data_ptr(), stream=s)
        if ev is not None:
            ev[1].record(stream)
        for q, ((c, base), o) in enumerate(zip(comp, outs)):
            ctx.query(ix, c, o.data_ptr(), stream=s, base_level=base, wide=wide)
            if ev is not None:
                ev[2 + q].record(stream)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
    stream.synchronize()
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(2 + len(comp))]
           for _ in range(args.steps)]
    clocks = ClockSampler(local)
    barrier(world)
    torch.cuda.synchronize(dev)
    clocks.start()
    t_index = t_total = 0.0
    with torch.cuda.stream(stream):
        for k in range(args.steps):
            if flush is not None:
                flush.fill_(k)
            step(evs[k])
    torch.cuda.synchronize(dev)
    t_query = [0.0] * len(comp)
    for e in evs:
        t_index += e[0].elapsed_time(e[1])
        t_total += e[0].elapsed_time(e[-1])
        for q in range(len(comp)):
            t_query[q] += e[1 + q].elapsed_time(e[2 + q])
    barrier(world)
    clk = clocks.stop()
    ms_step = allreduce_max(t_total / args.steps, world)
    ms_index = allreduce_max(t_index / args.steps, world)
    ms_query = [allreduce_max(t / args.steps, world) for t in t_query]

    # end to end through the host-buffer C ABI call, one call per partition
    # (partitions below 2 GiB split at newlines, as the reference's engine
    # cuts files; a single partition for every input below 2 GiB)
    h_in = torch.from_numpy(data).pin_memory()
    parts = newline_partitions(data, INT32_MAX)
    h_outs = []  # per partition, per query
    for p0, p1 in parts:
        pl = int(np.count_nonzero(data[p0:p1] == 10)) + 1
        h_outs.append([torch.empty(pl * c.num_result_slots * 2, dtype=torch.int32).pin_memory()
                       for c, _ in comp])
    e2e_ms = []
    for k in range(args.warmup + args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        got = 0
        for (p0, p1), hp in zip(parts, h_outs):
            got += ctx.query_host(h_in.data_ptr() + p0, p1 - p0, levels, [c for c, _ in comp],
                                  [h.data_ptr() for h in hp], [h.numel() for h in hp],
                                  stream=s, base_levels=[b for _, b in comp])
        e1.record(stream)
        e1.synchronize()
        assert got == lines
        if k >= args.warmup:
            e2e_ms.append(e0.elapsed_time(e1))
    e2e_step = allreduce_max(float(np.mean(e2e_ms)), world)
    # bit-exact check of the e2e results against the device-resident run:
    # partition-local offsets plus the partition start are the global ones
    for q, o in enumerate(outs):
        pieces = []
        for (p0, _), hp in zip(parts, h_outs):
            h = hp[q].numpy().astype(np.int64)
            pieces.append(np.where(h >= 0, h + p0, h))
        assert np.array_equal(np.concatenate(pieces), o.cpu().numpy().astype(np.int64)), \
            "e2e results differ from the device-resident run"

    gb = n * world / 1e9
    peak, peak_kind = measured_peak_hbm()
    b_index = algorithmic_index_bytes(n, levels, lines)
    achieved = b_index / (ms_index / 1e3) / 1e9
    traffic_path = ROOT / "profiles" / f"traffic_{args.workload}.json"
    traffic = None
    if traffic_path.exists():
        try:
            traffic = json.loads(traffic_path.read_text()).get("bytes_per_launch")
        except Exception:
            traffic = None
    line = {
        "metric": METRIC, "value": round(gb / (ms_step / 1e3), 3), "unit": "GB/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms_step, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded generator)",
        "config": {"workload": desc, "input_bytes": n, "records": lines, "levels": levels,
                   "queries": queries, "record_kind": records,
                   "l2": "flushed between steps" if flush is not None else
                         "input larger than L2", "parallelism": f"replicas x{world}"},
        "e2e": {"value": round(gb / (e2e_step / 1e3), 3), "unit": "GB/s",
                "h2d_bytes_per_step": sum(p1 - p0 for p0, p1 in parts),
                "d2h_bytes_per_step": sum(h.numel() * 4 for hp in h_outs for h in hp),
                "partitions": len(parts)},
        "gpu_launches": 1 + len(comp),
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                     "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": traffic,
                     "kernel": "gpjb::index_kernel", "peak_kind": peak_kind,
                     "algorithmic_bytes_per_launch": b_index,
                     "ms_per_launch": round(ms_index, 4)},
        "index_ms": round(ms_index, 4), "query_ms": round(ms_step - ms_index, 4),
        "index_gbs": round(n / 1e9 / (ms_index / 1e3), 1),
        "per_query": [{"query": q, "ms": round(t, 4), "gbs": round(n / 1e9 / (t / 1e3), 1)}
                      for q, t in zip(queries, ms_query)],
        "clocks": clk,
    }
    if rank == 0 and not args.no_cpu_baseline:
        got = [o.cpu().numpy().astype(np.int64).reshape(lines, c.num_result_slots, 2)
               for (c, _), o in zip(comp, outs)]
        line["cpu_baseline"], line["parity"] = cpu_baseline(data, comp, records, levels,
                                                            budget_s=12.0, results=got)
    if rank == 0 and args.ref_gpu:
        line["reference_gpu"] = reference_gpu(data, queries, records, levels, ms_index,
                                              ms_step - ms_index)
    ctx.close()
    return line


REF_DUMP = ROOT / "oracle" / "_ref" / "ref_dump"


def reference_gpu(data, queries, records, levels, ours_index_ms, ours_query_ms):
    """The reference's own index builders and query executor (its library
    compiled from its own sources into oracle/_ref) timed on the same GPU and
    input with CUDA events.  Array-record workloads: the reference indexes the
    array file and runs the queries on its NDJSON normalisation (it has no
    "$[*]").  Every input and query is first checked on the CPU against the
    reference's device-assert conditions (tests/ref_guard.py); an input that
    would trip one is not run.  Not a bench value of this engine: a
    comparison column."""
    import re
    import tempfile

    import ref_guard
    if not REF_DUMP.exists():
        return {"unavailable": "oracle/_ref/ref_dump not built"}
    pkg = entry.package()
    out = {"source": "reference library built from its own sources (oracle/ref/build_ref.py)",
           "ours_index_ms": round(ours_index_ms, 4), "ours_query_ms": round(ours_query_ms, 4)}
    with tempfile.TemporaryDirectory() as d:
        raw = Path(d) / "input.json"
        np.asarray(data).tofile(raw)
        qfile, qtext, qdata = raw, list(queries), np.asarray(data)
        if records == "array":
            b = bytes(np.asarray(data))
            elems = [ln.rstrip(b",") for ln in b.split(b"\n") if ln not in (b"[", b"]", b"")]
            qfile = Path(d) / "records.ndjson"
            qdata = np.frombuffer(b"\n".join(elems) + b"\n", np.uint8)
            qfile.write_bytes(qdata.tobytes())
            qtext = ["$" + q[4:] if q.startswith("$[*]") else q for q in queries]
        comp = [pkg.compile(q) for q in qtext]
        bad = ref_guard.problems(data, [], levels) + ref_guard.problems(qdata, comp, levels)
        if bad:
            return {"unavailable": "input would trip a reference device assert: " + bad[0]}
        for name, builder in (("SHAREMEM", 3), ("COMBINED", 1)):
            env = dict(os.environ, REF_TIME_REPS="5")
            r = subprocess.run([str(REF_DUMP), str(raw), str(builder), str(levels),
                                str(Path(d) / name)], capture_output=True, text=True, env=env,
                               timeout=900)
            q = subprocess.run([str(REF_DUMP), str(qfile), str(builder), str(levels),
                                str(Path(d) / (name + "_q"))] + qtext,
                               capture_output=True, text=True, env=env, timeout=900)
            mi = re.search(r"ms_index ([0-9.]+) ms_query ([0-9.]+)", r.stdout)
            mq = re.search(r"ms_index ([0-9.]+) ms_query ([0-9.]+)", q.stdout)
            if r.returncode != 0 or q.returncode != 0 or mi is None or mq is None:
                out[name] = {"error": (r.stderr + q.stderr + r.stdout[-200:])[-400:]}
                continue
            ms_i, ms_q = float(mi.group(1)), float(mq.group(2))
            out[name] = {"index_ms": round(ms_i, 3), "query_ms": round(ms_q, 3),
                         "index_speedup_ours": round(ms_i / ours_index_ms, 2),
                         "query_speedup_ours": round(ms_q / ours_query_ms, 2)}
    return out


def reference_gpu_column(pkg, local):
    """The reference-GPU column of the default line: the reference's SHAREMEM
    and COMBINED builders and its query executor against this engine on the
    same B200, on the c0 (64 MiB NDJSON, $.user.lang) and c1 (1 GiB array,
    $[*].categoryPath[1:3].id) inputs -- single inputs the reference's
    launch configuration handles (the c3 table has no reference counterpart:
    one Engine::query per file would take minutes).  This engine is timed two
    ways: the kernels into preallocated buffers (gpj_index_build_async and the
    query launches), and through gpj_index_build, which like the reference's
    IndexBuilder::build allocates its outputs and reads the line count."""
    import torch
    out = {}
    for name in ("c0", "c1"):
        data, queries, records, _ = workload(name, pkg)
        comp = compile_all(pkg, queries)
        levels = max(c.max_depth + base for c, base in comp)
        dev = torch.device("cuda", local)
        ctx = pkg.Context(local)
        n = data.size
        d_in = torch.from_numpy(data).to(dev)
        W = (n + 63) // 64
        S = torch.empty(W, dtype=torch.int64, device=dev)
        LB = torch.empty(W * levels, dtype=torch.int64, device=dev)
        NL = torch.empty(n // 32 + 1024, dtype=torch.int64, device=dev)
        summ = torch.zeros(4, dtype=torch.int64, device=dev)
        ix = pkg.Index()
        ix.d_string, ix.d_leveled = S.data_ptr(), LB.data_ptr()
        ix.d_newline, ix.newline_capacity = NL.data_ptr(), NL.numel()
        ctx.build_index_async(d_in.data_ptr(), n, levels, ix, summ.data_ptr())
        torch.cuda.synchronize()
        ix.num_lines = int(summ[0].item())
        outs = [torch.empty(ix.num_lines * c.num_result_slots * 2, dtype=torch.int32, device=dev)
                for c, _ in comp]
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        t_k = t_q = t_api = 0.0
        reps = 5
        for k in range(reps + 2):
            ev[0].record()
            ctx.build_index_async(d_in.data_ptr(), n, levels, ix, summ.data_ptr())
            ev[1].record()
            for (c, base), o in zip(comp, outs):
                ctx.query(ix, c, o.data_ptr(), base_level=base)
            ev[2].record()
            api = ctx.build_index(d_in.data_ptr(), n, levels)
            ev[3].record()
            torch.cuda.synchronize()
            ctx.free_index(api)
            if k >= 2:
                t_k += ev[0].elapsed_time(ev[1])
                t_q += ev[1].elapsed_time(ev[2])
                t_api += ev[2].elapsed_time(ev[3])
        ctx.close()
        del d_in, S, LB, NL, outs
        torch.cuda.empty_cache()
        out[name] = reference_gpu(data, queries, records, levels, t_k / reps, t_q / reps)
        out[name]["ours_index_api_ms"] = round(t_api / reps, 4)
        for b in ("SHAREMEM", "COMBINED"):
            if isinstance(out[name].get(b), dict) and "index_ms" in out[name][b]:
                out[name][b]["index_speedup_ours_api"] = round(
                    out[name][b]["index_ms"] / (t_api / reps), 2)
        out[name]["ours_timing"] = ("ours_index_ms: the index kernel into preallocated buffers; "
                                    "ours_index_api_ms: gpj_index_build (allocates its outputs, "
                                    "reads the line count); queries: kernels, CUDA events")
    return out


def run_batch(args, world, rank, local):
    """c3: 10,000 files (8 GiB) indexed and queried by one captured launch
    chain (gpj_batch), next to the plain one-launch-chain-per-file path."""
    import torch
    pkg = entry.package()
    pkg.load_library()
    files = c3_files(pkg, args.scale, rank=rank)
    comp = compile_all(pkg, C3_QUERIES)
    queries = [(c, base, c.max_depth + base) for c, base in comp]
    buf, offsets = pkg.pack_files([d for d, _ in files])
    total = sum(len(d) for d, _ in files)
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(device=dev)
    s = stream.cuda_stream
    d_buf = torch.from_numpy(buf).to(dev)
    table = [(o, len(d), k) for o, (d, k) in zip(offsets, files)]
    batch = pkg.Batch(d_buf.data_ptr(), buf.size, table, queries, flags=pkg.GPJ_BATCH_AUTOTUNE)
    v = batch.view()

    def timed(fn, steps):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(steps)]
        with torch.cuda.stream(stream):
            for e0, e1 in ev:
                e0.record(stream)
                fn()
                e1.record(stream)
        torch.cuda.synchronize(dev)
        return float(np.mean([e0.elapsed_time(e1) for e0, e1 in ev]))

    for _ in range(args.warmup):
        batch.run(s)
    torch.cuda.synchronize(dev)
    clocks = ClockSampler(local)
    barrier(world)
    clocks.start()
    ms_step = timed(lambda: batch.run(s), args.steps)
    clk = clocks.stop()
    barrier(world)
    ms_step = allreduce_max(ms_step, world)
    ms_index = allreduce_max(timed(lambda: batch.run_stages(pkg.STAGE_INDEX, s), 3), world)
    ms_query = allreduce_max(timed(lambda: batch.run_stages(pkg.STAGE_QUERY, s), 3), world)
    from devmem import d2h
    info = d2h(v.d_file_info, v.num_files * pkg.FILE_INFO_WORDS, np.uint64).reshape(-1, 8)
    assert int(d2h(v.d_totals, 4, np.uint64)[3]) == 0
    lines = info[:, 0].astype(np.int64)
    levels = np.array([queries[k][2] for _, k in files], np.int64)
    nbytes = np.array([len(d) for d, _ in files], np.int64)
    W = (nbytes + 63) // 64
    b_index = int((nbytes + 8 * W * (1 + levels) + 8 * lines).sum())
    b_query = int(v.result_ints) * 4

    # plain path: one single-file index launch + one query launch per file,
    # issued from C (gpj_batch_run_per_file), into the same outputs
    want_np = d2h(v.d_results, v.result_ints, np.int32)
    want = torch.from_numpy(want_np)
    batch.run_per_file(s)
    torch.cuda.synchronize(dev)
    ms_plain = allreduce_max(timed(lambda: batch.run_per_file(s), 3), world)
    got = torch.from_numpy(d2h(v.d_results, v.result_ints, np.int32))
    assert torch.equal(got, want), "plain per-file results differ from the batch"

    # end to end: host input in, host results out, through gpj_batch_run_host
    h_in = torch.from_numpy(buf).pin_memory()
    h_out = torch.empty(int(v.result_ints) + 1, dtype=torch.int32).pin_memory()
    h_info = torch.empty(v.num_files * pkg.FILE_INFO_WORDS, dtype=torch.int64).pin_memory()
    for _ in range(1):
        batch.run_host(h_in.data_ptr(), h_out.data_ptr(), h_info.data_ptr(), s)
    e2e = []
    for _ in range(args.steps):  # the same step count as the device-resident value
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        batch.run_host(h_in.data_ptr(), h_out.data_ptr(), h_info.data_ptr(), s)
        e1.record(stream)
        e1.synchronize()
        e2e.append(e0.elapsed_time(e1))
    assert torch.equal(h_out[: int(v.result_ints)], want)
    e2e_ms = allreduce_max(float(np.mean(e2e)), world)
    ingestion = ingestion_rates(pkg, buf, d_buf, h_in, local)

    gb = allreduce_sum(float(total), world) / 1e9  # every rank indexes its own files
    peak, peak_kind = measured_peak_hbm()
    achieved = b_index / (ms_index / 1e3) / 1e9
    chain = (b_index + b_query) / (ms_step / 1e3) / 1e9
    traffic = None
    tp = ROOT / "profiles" / "traffic_c3.json"
    if tp.exists():
        try:
            traffic = json.loads(tp.read_text()).get("bytes_per_launch")
        except Exception:
            traffic = None
    line = {
        "metric": METRIC, "value": round(gb / (ms_step / 1e3), 3), "unit": "GB/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms_step, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded generator)",
        "config": {"workload": C3_DESC, "input_bytes": total, "files": len(files), "records": int(v.num_records),
                   "l2": "input larger than L2", "parallelism": f"file shards x{world}",
                   "launch_shape": {"index_threads": v.index_threads,
                                    "index_walk": ("per-lane" if v.index_variant & 1 else "listed"),
                                    "lookback_descriptors": 64 if v.index_variant & 2 else 32,
                                    "query_block": v.query_block, "query_grid": v.query_grid,
                                    "graph": bool(v.uses_graph)}},
        "plain_per_file": {"value": round(gb / (ms_plain / 1e3), 3), "unit": "GB/s",
                           "ms_per_step": round(ms_plain, 3),
                           "batched_over_plain": round(ms_plain / ms_step, 2)},
        "e2e": {"value": round(gb / (e2e_ms / 1e3), 3), "unit": "GB/s",
                "h2d_bytes_per_step": int(buf.size),
                "d2h_bytes_per_step": int(v.result_ints) * 4 + v.num_files * 64},
        "gpu_launches": 3,
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                     "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": traffic,
                     "kernel": "gpjb::index_kernel (batched file table)", "peak_kind": peak_kind,
                     "algorithmic_bytes_per_launch": b_index, "ms_per_launch": round(ms_index, 4),
                     "chain_achieved": round(chain, 1), "chain_frac": round(chain / peak, 4)},
        "index_ms": round(ms_index, 4), "query_ms": round(ms_query, 4), "clocks": clk,
        "ingestion": ingestion,
    }
    if rank == 0 and not args.no_ref_gpu:
        line["reference_gpu"] = reference_gpu_column(pkg, local)
    if rank == 0 and not args.no_cpu_baseline:
        # the CPU baseline leg: the oracle over every timed file on every host
        # thread, timed, and its results compared with the batch's (the
        # parity gate of this line: any difference fails the run)
        oracle_res, dt, threads, done = oracle_files(files, queries)
        line["parity"] = batch_parity(files, queries, oracle_res, want_np, info)
        line["cpu_baseline"] = {
            "value": round(done / dt / 1e9, 4), "unit": "GB/s", "cores": threads,
            "kind": "port", "sample": f"all {len(files)} files of the workload ({done} bytes), "
            f"one file per task on {threads} threads, one pass ({dt:.2f} s)"}
    batch.close()
    return line


def ingestion_rates(pkg, buf, d_buf, h_in, local, nbytes: int = 2 << 30, reps: int = 3):
    """Host -> device GB/s of the first `nbytes` of the batch input: pageable
    memory through gpj_copy_to_device's pinned staging ring, pageable memory
    by a plain copy (what a synchronous pageable cudaMemcpy gets, as the
    reference's FilePartition::load_to_device does), and pinned memory.
    Wall clock around each call plus a device synchronisation."""
    import torch
    n = min(nbytes, buf.size)
    src = buf[:n]
    dst = d_buf[:n]
    ctx = pkg.Context(local)
    out = {"bytes": n}

    def rate(fn):
        fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            t0 = time.perf_counter()
            fn()
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t0)
        return round(n / min(ts) / 1e9, 2)

    out["pageable_staged_gbs"] = rate(lambda: ctx.copy_to_device(dst.data_ptr(), src.ctypes.data, n))
    out["pageable_plain_gbs"] = rate(lambda: dst.copy_(torch.from_numpy(src)))
    out["pinned_gbs"] = rate(lambda: dst.copy_(h_in[:n], non_blocking=True))
    ctx.close()
    return out


def oracle_files(files, queries, threads: int | None = None, limit_bytes: int | None = None):
    """The oracle (the reference algorithm restated in C) over whole files,
    one file per task on every host thread: per file the int64
    [lines][slots][2] results of its query, and the wall time.  With
    limit_bytes only the leading files up to that many bytes."""
    import oracle
    threads = threads or os.cpu_count() or 1
    count = len(files)
    if limit_bytes is not None:
        acc, count = 0, 0
        for d, _ in files:
            if acc >= limit_bytes:
                break
            acc += len(d)
            count += 1

    def work(i):
        d, k = files[i]
        c, base, lv = queries[k]
        if not len(d):
            return None
        return oracle.OracleIndex(d, lv).query(c.ir_bytes, c.num_result_slots, base)

    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(threads) as pool:
        res = list(pool.map(work, range(count)))
    dt = time.perf_counter() - t0
    return res, dt, threads, sum(len(files[i][0]) for i in range(count))


def batch_parity(files, queries, want, results, info):
    """Every file's query results of the batch (int32, file-local) against the
    oracle's: the parity gate of the timed c3 numbers.  Raises on the first
    difference."""
    checked = matches = 0
    for f, w in enumerate(want):
        lines, out_off = int(info[f, 0]), int(info[f, 3])
        slots = queries[files[f][1]][0].num_result_slots
        got = results[out_off:out_off + lines * slots * 2].astype(np.int64).reshape(lines, slots, 2)
        if w is None:
            ok = bool((got == -1).all())
        else:
            ok = got.shape == w.shape and np.array_equal(got, w)
            matches += int((w[..., 0] >= 0).sum())
        if not ok:
            raise AssertionError(f"c3 parity: file {f} results differ from the oracle")
        checked += 1
    return {"oracle": "oracle/gpjson_oracle.c (reference algorithm restated, pinned by the "
                      "reference's own test vectors)",
            "files_checked": checked, "files_total": len(files), "matches": matches,
            "mismatches": 0, "outputs": "every file's query results, bit-exact"}


def _partitions(data: np.ndarray, parts: int):
    """Newline-aligned partitions (the reference's independent partitions,
    src/gpjson/file/file_reader.cpp:41-77)."""
    n = data.size
    bounds = [0]
    for k in range(1, parts):
        t = k * n // parts
        nl = np.flatnonzero(data[t:min(n, t + (1 << 20))] == 10)
        if nl.size:
            bounds.append(t + int(nl[0]) + 1)
    bounds.append(n)
    bounds = sorted(set(bounds))
    return [(a, b) for a, b in zip(bounds, bounds[1:]) if b > a]


def cpu_baseline(data, comp, records, levels, budget_s: float, threads: int | None = None,
                 results=None):
    """Times the oracle (the reference algorithm restated in C) on a bounded,
    newline-aligned sample with one partition per host thread.  With
    `results` (this engine's per-query result arrays for the whole input,
    partition offsets) the oracle's results of the sample are compared with
    them: returns (baseline, parity)."""
    import oracle
    threads = threads or os.cpu_count() or 1
    sample = min(data.size, 96 << 20)
    parts = _partitions(data[:sample], threads * 4)

    def work(ab):
        a, b = ab
        ix = oracle.OracleIndex(data[a:b], levels)
        # a partition cut out of a top-level array holds its elements at
        # depth 0, except the first one, which holds the opening bracket
        return [ix.query(c.ir_bytes, c.num_result_slots, base if a == 0 else 0)
                for c, base in comp]

    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(threads) as pool:
        got = list(pool.map(work, parts))
    dt = time.perf_counter() - t0
    done = sum(b - a for a, b in parts)
    base = {"value": round(done / dt / 1e9, 4), "unit": "GB/s", "cores": threads,
            "kind": "port", "sample": f"first {done} bytes of the workload, "
            f"{len(parts)} newline-aligned partitions, {threads} threads"}
    if results is None:
        return base
    # partition k starts after a newline; its lines are the input's lines
    # from (newlines before it) on, and its last line (after the newline that
    # ends it) is empty unless it is the last partition of the input
    checked = 0
    for (a, b), per_query in zip(parts, got):
        first = int(np.count_nonzero(data[:a] == 10))
        for q, want in enumerate(per_query):
            w = want if b == data.size else want[:-1]
            w = np.where(w >= 0, w + a, w)
            g = np.asarray(results[q][first:first + w.shape[0]]).astype(np.int64)
            if g.shape != w.shape or not np.array_equal(g, w):
                raise AssertionError(f"parity: query {q} differs from the oracle in [{a}, {b})")
            checked += w.shape[0]
    return base, {"oracle": "oracle/gpjson_oracle.c on newline partitions of the first "
                            f"{done} bytes", "records_checked": checked, "mismatches": 0}


def run_reference(args, world, rank):
    """CPU arm: the reference algorithm's CPU restatement (the oracle; the
    reference project has no CPU implementation of this path) on all host
    threads, on the same workload, metric and config as this engine's line.
    c3: each timed step indexes and queries all 10,000 files once (warm-up
    steps run only the leading 96 MiB of files: they are untimed)."""
    if rank != 0:
        return None
    pkg = entry.package()
    if args.workload in ("c3", "c4"):
        files = c3_files(pkg, args.scale)
        comp = compile_all(pkg, C3_QUERIES)
        fq = [(c, base, c.max_depth + base) for c, base in comp]
        queries, desc = C3_QUERIES, C3_DESC
        total = sum(len(d) for d, _ in files)
        times, records = [], 0
        for k in range(args.warmup + args.steps):
            if k < args.warmup:
                oracle_files(files, fq, limit_bytes=96 << 20)
                continue
            res, dt, threads, done = oracle_files(files, fq)
            assert done == total
            times.append(dt)
            records = sum(1 if r is None else r.shape[0] for r in res)
        ms = float(np.mean(times)) * 1e3
        v = total / (ms / 1e3) / 1e9
        cb = {"value": round(v, 4), "unit": "GB/s", "cores": threads, "kind": "port",
              "sample": f"all {len(files)} files ({total} bytes) per step, one file per task "
                        f"on {threads} threads"}
        config = {"workload": C3_DESC, "input_bytes": total, "files": len(files),
                  "records": records, "queries": queries}
    else:
        data, queries, records, desc = workload(args.workload, pkg)
        comp = compile_all(pkg, queries)
        levels = max(c.max_depth + base for c, base in comp)
        vals = []
        for k in range(args.warmup + args.steps):
            cb = cpu_baseline(data, comp, records, levels, budget_s=10.0)
            if k >= args.warmup:
                vals.append(cb["value"])
        v = float(np.mean(vals))
        cb["value"] = round(v, 4)
        ms = None
        config = {"workload": desc, "queries": queries}
    return {"metric": METRIC, "value": round(v, 4), "unit": "GB/s", "impl": "reference",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms, 2) if ms is not None else None, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8",
            "data": "synthetic (seeded generator)", "config": config, "cpu_baseline": cb,
            "e2e": {"value": round(v, 4), "unit": "GB/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c3", choices=["c0", "c1", "c2", "c3", "c4"])
    ap.add_argument("--serve-seconds", type=float, default=4.0,
                    help="c4: length of the Poisson request trace")
    ap.add_argument("--no-serving", action="store_true",
                    help="c3: skip the serving trace that the default run appends")
    ap.add_argument("--scale", type=float, default=1.0,
                    help="c3 only: fraction of the 8 GiB total (profiling runs)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-gpu", action="store_true",
                    help="c0-c2: also time the reference's own library on the same GPU")
    ap.add_argument("--no-ref-gpu", action="store_true",
                    help="c3: skip the reference-GPU column (c0 and c1 inputs)")
    ap.add_argument("--size-mib", type=int, default=None,
                    help="profiling: run the workload's generator at this size")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world, rank, local = dist_init()
    if args.impl == "reference":
        line = run_reference(args, world, rank)
    elif args.workload == "c3":
        line = run_batch(args, world, rank, local)
        if not args.no_serving:
            import gc
            import torch
            gc.collect()
            torch.cuda.empty_cache()
            line["serving"] = run_serving(args, world, rank, local, duration_s=2.0)
    elif args.workload == "c4":
        serving = run_serving(args, world, rank, local)
        sat = serving["saturated"]["reuse"]
        line = {
            "metric": METRIC, "value": sat["gbs"], "unit": "GB/s", "n_gpus": world,
            "steps": 1, "warmup": 0, "ms_per_step": None, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8",
            "data": "synthetic (seeded generator)",
            "config": {"workload": serving["workload"], "parallelism": f"replicas x{world}",
                       "l2": "input larger than L2"},
            "e2e": {"value": sat["gbs"], "unit": "GB/s",
                    "h2d_bytes_per_step": serving["bytes_requested"],
                    "d2h_bytes_per_step": sat["d2h_bytes"]},
            "serving": serving,
        }
    else:
        line = run_ours(args, world, rank, local)
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
