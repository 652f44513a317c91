"""gpjson_b200: Python host-side mirror of the reference's engine API.

Thin ctypes bindings over the C ABI in include/gpjson_b200.h.  The names,
argument meaning and errors follow the reference's C++ interface
(Xinyu-Li-123/15418-project):

  compile(query)               query::QueryCompiler::compile
  Context.build_index(...)     index::IndexBuilder::build
  Context.query(...)           query::QueryExecutor::execute_batch (device part)
  Context.query_host(...)      the per-partition body of gpjson::Engine::query

Device memory is passed as integer device pointers (for example
torch.Tensor.data_ptr()); streams as integer cudaStream_t handles.  The native
library is required: there is no CPU path, and loading fails loudly if the
library has not been built.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from pathlib import Path

import numpy as np

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "lib" / "libgpjson_b200.so"

GPJ_OK = 0
GPJ_ERR_CUDA = 1
GPJ_ERR_OOM = 2
GPJ_ERR_MALFORMED_QUERY = 3
GPJ_ERR_UNSUPPORTED_QUERY = 4
GPJ_ERR_EXECUTION = 5
GPJ_ERR_TIMEOUT = 6
GPJ_ERR_INVALID_ARGUMENT = 7
GPJ_ERR_OUT_OF_RANGE = 8
GPJ_ERR_CAPACITY = 9
GPJ_ERR_IMPLEMENTATION = 10

GPJ_INDEX_EMIT_ESCAPE_QUOTE = 1
GPJ_INDEX_NO_TMA = 2
GPJ_INDEX_DIAG_TILE0_UNPUBLISHED = 0x80000000
GPJ_QUERY_OVERFLOW = 0x100  # a record had more results than result slots
MAX_LEVELS = 22
MAX_QUERY_IR = 4096
MAX_QUERY_DEPTH = 16

EXPORTED_SYMBOLS = (
    "gpj_version", "gpj_last_error", "gpj_ctx_create", "gpj_ctx_destroy",
    "gpj_compile", "gpj_index_build", "gpj_index_build_async", "gpj_index_build_noalloc",
    "gpj_index_free",
    "gpj_query_run", "gpj_query_run64", "gpj_query_run_opts", "gpj_query_host",
    "gpj_query_status", "gpj_copy_to_device",
    "gpj_results_compact",
    "gpj_batch_create", "gpj_batch_run", "gpj_batch_run_stages", "gpj_batch_run_per_file",
    "gpj_batch_run_host",
    "gpj_batch_view_get", "gpj_batch_file_layout", "gpj_batch_destroy",
    "gpj_server_create", "gpj_server_submit", "gpj_server_submit_many", "gpj_server_poll",
    "gpj_server_wait",
    "gpj_server_response", "gpj_server_release", "gpj_server_stats_get",
    "gpj_server_clear_cache", "gpj_server_destroy",
)
STAGE_INDEX, STAGE_FINALIZE, STAGE_QUERY = 1, 2, 4

GPJ_BATCH_AUTOTUNE = 4
GPJ_BATCH_NO_GRAPH = 8
GPJ_BATCH_INDEX_LANE_WALK = 16
GPJ_BATCH_INDEX_WIDE_LOOKBACK = 32
FILE_INFO_WORDS = 8  # lines, newline slot, first record, first result int, in-string, depth, bytes, query


# Exception hierarchy of the reference (include/gpjson/error/*.hpp).
class GpJSONError(Exception):
    pass


class CudaError(GpJSONError):
    pass


class MalformedQueryError(GpJSONError):
    pass


class UnsupportedQueryError(GpJSONError):
    pass


class QueryExecutionError(GpJSONError):
    pass


class ImplementationError(GpJSONError):
    pass


class DeviceTimeoutError(GpJSONError):
    """A bounded device-side wait gave up (no reference counterpart)."""


class CapacityError(GpJSONError):
    """A caller-provided buffer is too small (no reference counterpart)."""


_ERRORS = {
    GPJ_ERR_CUDA: CudaError,
    GPJ_ERR_OOM: CudaError,
    GPJ_ERR_MALFORMED_QUERY: MalformedQueryError,
    GPJ_ERR_UNSUPPORTED_QUERY: UnsupportedQueryError,
    GPJ_ERR_EXECUTION: QueryExecutionError,
    GPJ_ERR_TIMEOUT: DeviceTimeoutError,
    GPJ_ERR_INVALID_ARGUMENT: ValueError,
    GPJ_ERR_OUT_OF_RANGE: OverflowError,
    GPJ_ERR_CAPACITY: CapacityError,
    GPJ_ERR_IMPLEMENTATION: ImplementationError,
}


class QueryOpts(C.Structure):
    """gpj_query_opts."""

    _fields_ = [("base_level", C.c_uint32), ("offset_bytes", C.c_uint32),
                ("reserved", C.c_uint32 * 2)]


class Index(C.Structure):
    """gpj_index: device-resident structural indexes of one partition."""

    _fields_ = [
        ("d_input", C.c_void_p),
        ("size_bytes", C.c_uint64),
        ("d_newline", C.c_void_p),
        ("num_lines", C.c_uint64),
        ("newline_capacity", C.c_uint64),
        ("d_string", C.c_void_p),
        ("d_leveled", C.c_void_p),
        ("d_escape", C.c_void_p),
        ("d_quote", C.c_void_p),
        ("num_words", C.c_uint64),
        ("num_levels", C.c_int32),
        ("final_in_string", C.c_int32),
        ("final_depth", C.c_int32),
        ("reserved", C.c_int32),
        ("owner", C.c_void_p),
    ]


class BatchFile(C.Structure):
    _fields_ = [("offset", C.c_uint64), ("size_bytes", C.c_uint64), ("query", C.c_uint32),
                ("reserved", C.c_uint32)]


class BatchQuery(C.Structure):
    _fields_ = [("h_ir", C.c_void_p), ("ir_len", C.c_uint64), ("num_result_slots", C.c_uint32),
                ("base_level", C.c_uint32), ("num_levels", C.c_uint32), ("reserved", C.c_uint32)]


class BatchView(C.Structure):
    _fields_ = [("d_string", C.c_void_p), ("d_leveled", C.c_void_p), ("d_newline", C.c_void_p),
                ("d_results", C.c_void_p), ("d_file_info", C.c_void_p), ("d_totals", C.c_void_p),
                ("num_files", C.c_uint64), ("num_records", C.c_uint64),
                ("result_ints", C.c_uint64), ("newline_slots", C.c_uint64),
                ("string_words", C.c_uint64), ("leveled_words", C.c_uint64),
                ("num_tiles", C.c_uint32), ("index_threads", C.c_uint32),
                ("query_block", C.c_uint32), ("query_grid", C.c_uint32),
                ("uses_graph", C.c_uint32), ("index_variant", C.c_uint32)]


GPJ_SERVER_NO_CACHE = 1
GPJ_SERVER_SLEEP_POLL = 2
GPJ_SERVER_NO_GROUPS = 4
SERVER_MAX_QUERIES = 8


class ServerConfig(C.Structure):
    _fields_ = [("device", C.c_int32), ("num_slots", C.c_int32),
                ("hbm_budget_bytes", C.c_uint64), ("host_result_bytes", C.c_uint64),
                ("cache_levels", C.c_int32), ("flags", C.c_uint32),
                ("reserved", C.c_uint32 * 4)]


class Request(C.Structure):
    _fields_ = [("file_key", C.c_uint64), ("h_input", C.c_void_p), ("size_bytes", C.c_uint64),
                ("queries", C.c_void_p), ("num_queries", C.c_uint32), ("reserved", C.c_uint32),
                ("arrival_ns", C.c_uint64)]


class Response(C.Structure):
    _fields_ = [("status", C.c_int32), ("cache_hit", C.c_int32), ("num_lines", C.c_uint64),
                ("h_results", C.c_void_p), ("result_ints", C.c_uint64),
                ("result_offset", C.c_uint64 * SERVER_MAX_QUERIES),
                ("arrival_ns", C.c_uint64), ("admit_ns", C.c_uint64),
                ("index_ready_ns", C.c_uint64), ("done_ns", C.c_uint64),
                ("message", C.c_char * 128)]


class ServerStats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in (
        "submitted", "completed", "failed", "cache_hits", "cache_misses", "evictions", "rebuilds",
        "bytes_indexed", "bytes_served", "resident_indexes", "resident_bytes", "arena_used",
        "arena_peak", "arena_bytes", "in_flight", "pending", "index_launches")]


_lib = None


def library_path() -> Path:
    return LIB_PATH


def load_library(build_if_missing: bool = False) -> C.CDLL:
    """Loads libgpjson_b200.so; raises if it is missing (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        if not build_if_missing:
            raise RuntimeError(
                f"native library {LIB_PATH} is missing: build it first "
                "(python __graft_entry__.py or 15418-project_b200/build.py)")
        import importlib.util
        spec = importlib.util.spec_from_file_location("_gpjb_build", _PKG / "build.py")
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        mod.build_library()
    lib = C.CDLL(str(LIB_PATH))
    u64, u32, vp, i32 = C.c_uint64, C.c_uint32, C.c_void_p, C.c_int
    P = C.POINTER
    lib.gpj_version.restype = i32
    lib.gpj_last_error.restype = C.c_char_p
    lib.gpj_ctx_create.argtypes = [i32, P(vp)]
    lib.gpj_ctx_destroy.argtypes = [vp]
    lib.gpj_compile.argtypes = [C.c_char_p, u64, vp, u64, P(u64), P(u64), P(u64)]
    lib.gpj_index_build.argtypes = [vp, vp, u64, i32, u32, P(Index), vp]
    lib.gpj_index_build_async.argtypes = [vp, vp, u64, i32, u32, P(Index), vp, vp]
    lib.gpj_index_build_noalloc.argtypes = [vp, u64, i32, u32, P(Index), vp, vp]
    lib.gpj_index_free.argtypes = [vp, P(Index)]
    lib.gpj_query_run.argtypes = [vp, P(Index), vp, u64, u32, vp, vp]
    lib.gpj_query_run64.argtypes = [vp, P(Index), vp, u64, u32, vp, vp]
    lib.gpj_query_run_opts.argtypes = [vp, P(Index), vp, u64, u32, P(QueryOpts), vp, vp]
    lib.gpj_query_host.argtypes = [vp, vp, u64, i32, u32, vp, vp, vp, vp, vp, vp, P(u64), vp]
    lib.gpj_query_status.argtypes = [vp, P(u32), vp]
    lib.gpj_copy_to_device.argtypes = [vp, vp, vp, u64, vp]
    lib.gpj_results_compact.argtypes = [vp, vp, u64, u32, vp, u64, C.c_int64, vp, u64, vp, u64,
                                        vp, vp]
    lib.gpj_batch_create.argtypes = [vp, vp, u64, P(BatchFile), u32, P(BatchQuery), u32, u32,
                                     P(vp), vp]
    lib.gpj_batch_run.argtypes = [vp, vp]
    lib.gpj_batch_run_stages.argtypes = [vp, u32, vp]
    lib.gpj_batch_run_per_file.argtypes = [vp, vp]
    lib.gpj_batch_run_host.argtypes = [vp, vp, vp, vp, vp]
    lib.gpj_batch_view_get.argtypes = [vp, P(BatchView)]
    lib.gpj_batch_file_layout.argtypes = [vp, u32, P(u64), P(u64), P(u32)]
    lib.gpj_batch_destroy.argtypes = [vp]
    lib.gpj_server_create.argtypes = [P(ServerConfig), P(vp)]
    lib.gpj_server_submit.argtypes = [vp, P(Request), P(u64)]
    lib.gpj_server_submit_many.argtypes = [vp, vp, u32, vp]
    lib.gpj_server_poll.argtypes = [vp, P(u64), u32, P(u32), C.c_int64]
    lib.gpj_server_wait.argtypes = [vp, u64, C.c_int64]
    lib.gpj_server_response.argtypes = [vp, u64, P(Response)]
    lib.gpj_server_release.argtypes = [vp, u64]
    lib.gpj_server_stats_get.argtypes = [vp, P(ServerStats)]
    lib.gpj_server_clear_cache.argtypes = [vp]
    lib.gpj_server_destroy.argtypes = [vp]
    for name in EXPORTED_SYMBOLS:
        if name != "gpj_version" and name != "gpj_last_error":
            getattr(lib, name).restype = i32
    _lib = lib
    return lib


def _check(rc: int) -> None:
    if rc != GPJ_OK:
        msg = load_library().gpj_last_error().decode(errors="replace")
        raise _ERRORS.get(rc, GpJSONError)(msg)


@dataclass(frozen=True)
class CompiledQuery:
    """query::CompiledQuery (include/gpjson/query/query.hpp:23-43)."""

    query_text: str
    ir_bytes: bytes
    max_depth: int
    num_result_slots: int


def compile(query: str, wildcard_limit: int = 0) -> CompiledQuery:  # noqa: A001
    """Compiles a JSONPath query (query_compiler.cpp QueryParser::compile)."""
    lib = load_library()
    n, depth, slots = C.c_uint64(), C.c_uint64(), C.c_uint64()
    cap = MAX_QUERY_IR
    while True:
        buf = (C.c_uint8 * cap)()
        rc = lib.gpj_compile(query.encode(), wildcard_limit, buf, cap, C.byref(n),
                             C.byref(depth), C.byref(slots))
        if rc == GPJ_ERR_CAPACITY and n.value > cap:
            cap = n.value
            continue
        _check(rc)
        break
    return CompiledQuery(query, bytes(buf[: n.value]), depth.value, slots.value)


NOALLOC_MAX_BYTES = 4 << 30


def build_index_noalloc(d_input: int, size_bytes: int, num_levels: int, index: Index,
                        d_summary: int, flags: int = 0, stream: int = 0) -> None:
    """gpj_index_build_noalloc: the index build for callers that cannot allocate
    device memory (all buffers are the caller's; scratch is a fixed array in
    the library, inputs up to 4 GiB)."""
    _check(load_library().gpj_index_build_noalloc(
        C.c_void_p(d_input), size_bytes, num_levels, flags, C.byref(index),
        C.c_void_p(d_summary), C.c_void_p(stream)))


class Context:
    """A device binding plus reusable device buffers (gpj_ctx)."""

    def __init__(self, device: int = 0):
        self._lib = load_library()
        h = C.c_void_p()
        _check(self._lib.gpj_ctx_create(device, C.byref(h)))
        self._h = h

    def close(self) -> None:
        if self._h:
            self._lib.gpj_ctx_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def build_index(self, d_input: int, size_bytes: int, num_levels: int,
                    flags: int = 0, stream: int = 0) -> Index:
        ix = Index()
        _check(self._lib.gpj_index_build(self._h, C.c_void_p(d_input), size_bytes,
                                         num_levels, flags, C.byref(ix),
                                         C.c_void_p(stream)))
        return ix

    def build_index_async(self, d_input: int, size_bytes: int, num_levels: int,
                          index: Index, d_summary: int, flags: int = 0,
                          stream: int = 0) -> None:
        _check(self._lib.gpj_index_build_async(self._h, C.c_void_p(d_input), size_bytes,
                                               num_levels, flags, C.byref(index),
                                               C.c_void_p(d_summary), C.c_void_p(stream)))

    def free_index(self, index: Index) -> None:
        _check(self._lib.gpj_index_free(self._h, C.byref(index)))

    def query(self, index: Index, compiled: CompiledQuery, d_out: int, stream: int = 0,
              wide: bool = False, base_level: int = 0) -> None:
        ir = (C.c_uint8 * max(1, len(compiled.ir_bytes))).from_buffer_copy(
            compiled.ir_bytes or b"\0")
        if base_level == 0:
            fn = self._lib.gpj_query_run64 if wide else self._lib.gpj_query_run
            _check(fn(self._h, C.byref(index), ir, len(compiled.ir_bytes),
                      compiled.num_result_slots, C.c_void_p(d_out), C.c_void_p(stream)))
            return
        opts = QueryOpts(base_level, 8 if wide else 4)
        _check(self._lib.gpj_query_run_opts(self._h, C.byref(index), ir, len(compiled.ir_bytes),
                                            compiled.num_result_slots, C.byref(opts),
                                            C.c_void_p(d_out), C.c_void_p(stream)))

    def copy_to_device(self, d_dst: int, h_src: int, size_bytes: int, stream: int = 0) -> None:
        """gpj_copy_to_device: host -> device; pageable sources are staged
        through the context's pinned ring (returns once the source may be
        reused; the copy completes in stream order)."""
        _check(self._lib.gpj_copy_to_device(self._h, C.c_void_p(d_dst), C.c_void_p(h_src),
                                            size_bytes, C.c_void_p(stream)))

    def query_status(self, stream: int = 0) -> int:
        """gpj_query_status: status bits of this context's queries since the
        last call (GPJ_QUERY_OVERFLOW), cleared by the call."""
        flags = C.c_uint32()
        _check(self._lib.gpj_query_status(self._h, C.byref(flags), C.c_void_p(stream)))
        return flags.value

    def compact(self, d_results: int, num_lines: int, num_result_slots: int, d_input: int,
                size_bytes: int, base_offset: int, d_matches: int, match_capacity: int,
                d_arena: int, arena_capacity: int, d_counts: int, stream: int = 0) -> None:
        """gpj_results_compact: device pointers in, asynchronous on `stream`."""
        _check(self._lib.gpj_results_compact(
            self._h, C.c_void_p(d_results), num_lines, num_result_slots, C.c_void_p(d_input),
            size_bytes, base_offset, C.c_void_p(d_matches), match_capacity, C.c_void_p(d_arena),
            arena_capacity, C.c_void_p(d_counts), C.c_void_p(stream)))

    def query_host(self, h_input: int, size_bytes: int, num_levels: int,
                   compiled: list[CompiledQuery], h_outs: list[int],
                   capacities: list[int], stream: int = 0,
                   base_levels: list[int] | None = None) -> int:
        """Host in, host out: returns the number of records."""
        q = len(compiled)
        irs = [(C.c_uint8 * max(1, len(c.ir_bytes))).from_buffer_copy(c.ir_bytes or b"\0")
               for c in compiled]
        ir_ptrs = (C.c_void_p * max(1, q))(*[C.addressof(b) for b in irs])
        ir_lens = (C.c_uint64 * max(1, q))(*[len(c.ir_bytes) for c in compiled])
        slots = (C.c_uint32 * max(1, q))(*[c.num_result_slots for c in compiled])
        outs = (C.c_void_p * max(1, q))(*h_outs)
        caps = (C.c_uint64 * max(1, q))(*capacities)
        bases = (C.c_uint32 * max(1, q))(*(base_levels or [0] * q))
        lines = C.c_uint64()
        _check(self._lib.gpj_query_host(self._h, C.c_void_p(h_input), size_bytes, num_levels,
                                        q, ir_ptrs, ir_lens, slots, bases, outs, caps,
                                        C.byref(lines), C.c_void_p(stream)))
        return lines.value


# gpj_match as a numpy record (40 bytes)
MATCH_DTYPE = np.dtype([("line", "<u8"), ("slot", "<u4"), ("length", "<u4"),
                        ("start", "<i8"), ("end", "<i8"), ("text_offset", "<u8")])


def compact_results(ctx: "Context", d_results: int, num_lines: int, num_result_slots: int,
                    d_input: int, size_bytes: int, base_offset: int = 0,
                    match_capacity: int = 1 << 16, arena_capacity: int = 1 << 20,
                    stream: int = 0):
    """Compacts one query's device result array on the device
    (gpj_results_compact) and copies back only the matches and their bytes.
    Returns (matches as a MATCH_DTYPE array, arena bytes); raises
    QueryExecutionError for an invalid range as the reference does.  Device
    buffers are torch allocations, grown and the call repeated when the
    first guess of the capacities is too small."""
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    counts = torch.zeros(3, dtype=torch.int64, device=dev)
    while True:
        matches = torch.empty(max(1, match_capacity) * MATCH_DTYPE.itemsize, dtype=torch.uint8,
                              device=dev)
        arena = torch.empty(max(1, arena_capacity), dtype=torch.uint8, device=dev)
        ctx.compact(d_results, num_lines, num_result_slots, d_input, size_bytes, base_offset,
                    matches.data_ptr(), match_capacity, arena.data_ptr(), arena_capacity,
                    counts.data_ptr(), stream)
        torch.cuda.synchronize(dev)
        m, nbytes, invalid = (int(x) for x in counts.cpu())
        if invalid:
            raise QueryExecutionError("Query kernel produced an invalid result range")
        if m <= match_capacity and nbytes <= arena_capacity:
            break
        match_capacity, arena_capacity = max(m, 1), max(nbytes, 1)
    out = matches[: m * MATCH_DTYPE.itemsize].cpu().numpy().view(MATCH_DTYPE)
    return out, bytes(arena[:nbytes].cpu().numpy())


def pack_files(files, align: int = 128):
    """Concatenates host byte arrays at `align`-byte offsets (zero padding).
    Returns (buffer, offsets)."""
    import numpy as np
    offsets, pos = [], 0
    for f in files:
        offsets.append(pos)
        pos += (len(f) + align - 1) // align * align
    buf = np.zeros(max(pos, align), np.uint8)
    for f, o in zip(files, offsets):
        buf[o:o + len(f)] = np.frombuffer(bytes(f), np.uint8) if not hasattr(f, "dtype") else f
    return buf, offsets


class Batch:
    """gpj_batch: many files indexed and queried by one captured launch chain.

    files: list of (offset, size_bytes, query_index) in the device buffer;
    queries: list of (CompiledQuery, base_level, num_levels)."""

    def __init__(self, d_input: int, input_bytes: int, files, queries, flags: int = 0,
                 stream: int = 0):
        self._lib = load_library()
        fa = (BatchFile * len(files))(*[BatchFile(o, n, q, 0) for o, n, q in files])
        self._irs = [(C.c_uint8 * max(1, len(c.ir_bytes))).from_buffer_copy(c.ir_bytes or b"\0")
                     for c, _, _ in queries]
        qa = (BatchQuery * len(queries))(*[
            BatchQuery(C.addressof(ir), len(c.ir_bytes), c.num_result_slots, base, lv, 0)
            for (c, base, lv), ir in zip(queries, self._irs)])
        h = C.c_void_p()
        _check(self._lib.gpj_batch_create(None, C.c_void_p(d_input), input_bytes, fa, len(files),
                                          qa, len(queries), flags, C.byref(h),
                                          C.c_void_p(stream)))
        self._h = h

    def run(self, stream: int = 0) -> None:
        _check(self._lib.gpj_batch_run(self._h, C.c_void_p(stream)))

    def run_stages(self, stages: int, stream: int = 0) -> None:
        _check(self._lib.gpj_batch_run_stages(self._h, stages, C.c_void_p(stream)))

    def run_per_file(self, stream: int = 0) -> None:
        _check(self._lib.gpj_batch_run_per_file(self._h, C.c_void_p(stream)))

    def run_host(self, h_input: int, h_results: int = 0, h_file_info: int = 0,
                 stream: int = 0) -> None:
        _check(self._lib.gpj_batch_run_host(self._h, C.c_void_p(h_input), C.c_void_p(h_results),
                                            C.c_void_p(h_file_info), C.c_void_p(stream)))

    def view(self) -> BatchView:
        v = BatchView()
        _check(self._lib.gpj_batch_view_get(self._h, C.byref(v)))
        return v

    def file_layout(self, f: int):
        s, l, lv = C.c_uint64(), C.c_uint64(), C.c_uint32()
        _check(self._lib.gpj_batch_file_layout(self._h, f, C.byref(s), C.byref(l), C.byref(lv)))
        return s.value, l.value, lv.value

    def close(self) -> None:
        if self._h:
            self._lib.gpj_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class ServerResult:
    """A finished request: per-query int32 [lines][slots][2] offset arrays
    (copied out of the server's pinned arena) and its timestamps (ns,
    CLOCK_MONOTONIC)."""

    request_id: int
    status: int
    message: str
    cache_hit: bool
    num_lines: int
    result_ints: int
    results: list
    arrival_ns: int
    admit_ns: int
    index_ready_ns: int
    done_ns: int

    @property
    def latency_ns(self) -> int:
        return self.done_ns - self.arrival_ns


class Server:
    """gpj_server: continuous-batching request loop with resident indexes.

    submit(data, queries, file_key) queues a request; queries are
    (CompiledQuery, base_level, num_levels) triples as for Batch.  `data` is a
    numpy uint8 array (or anything exposing the buffer protocol) that must stay
    alive until the request finishes."""

    def __init__(self, device: int = 0, num_slots: int = 32, hbm_budget_bytes: int = 1 << 30,
                 host_result_bytes: int = 256 << 20, cache_levels: int = 4, flags: int = 0):
        self._lib = load_library()
        cfg = ServerConfig(device, num_slots, hbm_budget_bytes, host_result_bytes, cache_levels,
                           flags)
        h = C.c_void_p()
        _check(self._lib.gpj_server_create(C.byref(cfg), C.byref(h)))
        self._h = h
        self._keep = {}

    def submit(self, data, queries, file_key: int = 0, arrival_ns: int = 0) -> int:
        import numpy as np
        arr = np.frombuffer(data, np.uint8) if not isinstance(data, np.ndarray) else data
        irs = [(C.c_uint8 * max(1, len(c.ir_bytes))).from_buffer_copy(c.ir_bytes or b"\0")
               for c, _, _ in queries]
        qa = (BatchQuery * len(queries))(*[
            BatchQuery(C.addressof(ir), len(c.ir_bytes), c.num_result_slots, base, lv, 0)
            for (c, base, lv), ir in zip(queries, irs)])
        req = Request(file_key, arr.ctypes.data if arr.size else None, arr.size,
                      C.cast(qa, C.c_void_p), len(queries), 0, arrival_ns)
        rid = C.c_uint64()
        _check(self._lib.gpj_server_submit(self._h, C.byref(req), C.byref(rid)))
        self._keep[rid.value] = (arr, [c.num_result_slots for c, _, _ in queries])
        return rid.value

    def prepare(self, items):
        """Builds the request table of gpj_server_submit_many for a list of
        (data, queries, file_key, arrival_ns) items; submit_prepared queues it
        with one call."""
        import numpy as np
        reqs = (Request * max(1, len(items)))()
        keep = []
        for i, (data, queries, key, arrival) in enumerate(items):
            arr = np.frombuffer(data, np.uint8) if not isinstance(data, np.ndarray) else data
            irs = [(C.c_uint8 * max(1, len(c.ir_bytes))).from_buffer_copy(c.ir_bytes or b"\0")
                   for c, _, _ in queries]
            qa = (BatchQuery * len(queries))(*[
                BatchQuery(C.addressof(ir), len(c.ir_bytes), c.num_result_slots, base, lv, 0)
                for (c, base, lv), ir in zip(queries, irs)])
            reqs[i] = Request(key, arr.ctypes.data if arr.size else None, arr.size,
                              C.cast(qa, C.c_void_p), len(queries), 0, arrival)
            keep.append((arr, [c.num_result_slots for c, _, _ in queries], irs, qa))
        return reqs, keep

    def submit_prepared(self, prepared) -> list:
        reqs, keep = prepared
        ids = (C.c_uint64 * max(1, len(keep)))()
        _check(self._lib.gpj_server_submit_many(self._h, C.cast(reqs, C.c_void_p), len(keep), ids))
        for rid, (arr, slots, _, _) in zip(ids[:len(keep)], keep):
            self._keep[rid] = (arr, slots)
        return list(ids[:len(keep)])

    def poll(self, capacity: int = 1024, timeout_us: int = 0) -> list:
        ids = (C.c_uint64 * capacity)()
        n = C.c_uint32()
        _check(self._lib.gpj_server_poll(self._h, ids, capacity, C.byref(n), timeout_us))
        return list(ids[: n.value])

    def wait(self, request_id: int, timeout_us: int = -1) -> None:
        _check(self._lib.gpj_server_wait(self._h, request_id, timeout_us))

    def response(self, request_id: int, release: bool = True,
                 copy_results: bool = True) -> ServerResult:
        import numpy as np
        r = Response()
        _check(self._lib.gpj_server_response(self._h, request_id, C.byref(r)))
        _, slots = self._keep.get(request_id, (None, []))
        results = []
        if r.status == GPJ_OK and copy_results:
            ints = np.ctypeslib.as_array(C.cast(r.h_results, C.POINTER(C.c_int32)),
                                         shape=(max(r.result_ints, 1),))[: r.result_ints]
            for q, s in enumerate(slots):
                off = r.result_offset[q]
                cnt = r.num_lines * s * 2
                results.append(ints[off:off + cnt].copy().reshape(r.num_lines, s, 2))
        out = ServerResult(request_id, r.status, r.message.decode(errors="replace"),
                           bool(r.cache_hit), r.num_lines, r.result_ints, results,
                           r.arrival_ns, r.admit_ns,
                           r.index_ready_ns, r.done_ns)
        if release:
            self.release(request_id)
        return out

    def release(self, request_id: int) -> None:
        _check(self._lib.gpj_server_release(self._h, request_id))
        self._keep.pop(request_id, None)

    def stats(self) -> dict:
        st = ServerStats()
        _check(self._lib.gpj_server_stats_get(self._h, C.byref(st)))
        return {name: getattr(st, name) for name, _ in ServerStats._fields_}

    def clear_cache(self) -> None:
        _check(self._lib.gpj_server_clear_cache(self._h))

    def close(self) -> None:
        if self._h:
            self._lib.gpj_server_destroy(self._h)
            self._h = C.c_void_p()
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
