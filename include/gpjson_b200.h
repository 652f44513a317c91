/*
 * gpjson_b200 -- C ABI of the B200 GpJSON engine.
 *
 * Plain pointers and sizes only.  Device pointers are marked d_, host
 * pointers h_.  Every call returns a status (GPJ_OK = 0); the message of the
 * last failure on the calling thread is gpj_last_error().  Streams are passed
 * as void* (a cudaStream_t; NULL = legacy default stream).
 *
 * Each entry point names the reference interface it replaces
 * (Xinyu-Li-123/15418-project, paths relative to that project).
 */
#ifndef GPJSON_B200_H
#define GPJSON_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The C++ wrapper maps them back onto the reference's
 * exception types (include/gpjson/error/ headers, query/error.hpp, file/error.hpp,
 * cuda/error.hpp). */
#define GPJ_OK 0
#define GPJ_ERR_CUDA 1              /* error::cuda::CudaError */
#define GPJ_ERR_OOM 2               /* error::cuda::CudaError (allocation) */
#define GPJ_ERR_MALFORMED_QUERY 3   /* error::query::MalformedQueryError */
#define GPJ_ERR_UNSUPPORTED_QUERY 4 /* error::query::UnsupportedQueryError */
#define GPJ_ERR_EXECUTION 5         /* error::query::QueryExecutionError */
#define GPJ_ERR_TIMEOUT 6           /* a bounded device wait gave up */
#define GPJ_ERR_INVALID_ARGUMENT 7  /* std::invalid_argument */
#define GPJ_ERR_OUT_OF_RANGE 8      /* std::out_of_range */
#define GPJ_ERR_CAPACITY 9          /* a caller buffer is too small */
#define GPJ_ERR_IMPLEMENTATION 10   /* error::common::ImplementationError */

/* gpj_index_build flags */
#define GPJ_INDEX_EMIT_ESCAPE_QUOTE 1u /* also materialise E and Q */
#define GPJ_INDEX_NO_TMA 2u            /* stage tiles with plain loads */
/* Diagnostic (gpj_index_build and gpj_index_build_async only): the first
 * 32 KiB tile is left out of the launch, so the look-back of every other tile
 * waits for a descriptor that is never published; each wait gives up after
 * about 16 K polls (milliseconds) and the build reports GPJ_ERR_TIMEOUT
 * (d_summary[3] bit 0).  It exercises the bounded-wait error path on a
 * device that stays usable; its outputs are meaningless.  Needs an input of
 * at least two tiles. */
#define GPJ_INDEX_DIAG_TILE0_UNPUBLISHED 0x80000000u

#define GPJ_MAX_LEVELS 22     /* kMaxNumLevels, sharemem/leveled-bitmaps-index.cu */
#define GPJ_MAX_QUERY_IR 4096 /* kMaxQueryIrBytes, query/kernels/orig.hpp:11 */
#define GPJ_MAX_QUERY_DEPTH 16 /* kMaxQueryLevels, query/kernels/orig.hpp:10 */

typedef struct gpj_ctx gpj_ctx;

/* Built structural indexes of one partition (include/gpjson/index/index.hpp:
 * NewlineIndex, StringIndex, LeveledBitmapIndex, BuiltIndices).  Bitmaps use
 * the reference layout: bit b of word w <-> byte 64*w+b, leveled bitmaps
 * level-major d_leveled[level * num_words + w]. */
typedef struct gpj_index {
  const uint8_t *d_input;  /* borrowed partition bytes */
  uint64_t size_bytes;
  int64_t *d_newline;      /* [num_lines]: 0, then every '\n' offset */
  uint64_t num_lines;      /* newline count + 1 */
  uint64_t newline_capacity;
  uint64_t *d_string;      /* [num_words] in-string mask */
  uint64_t *d_leveled;     /* [num_levels * num_words] */
  uint64_t *d_escape;      /* [num_words] or NULL */
  uint64_t *d_quote;       /* [num_words] or NULL */
  uint64_t num_words;      /* ceil(size_bytes / 64) */
  int32_t num_levels;
  int32_t final_in_string; /* string state after the last byte */
  int32_t final_depth;     /* signed-char depth after the last byte */
  int32_t reserved;
  void *owner;             /* library-owned allocation (NULL: caller-owned) */
} gpj_index;

/* Library version, major*10000 + minor*100 + patch. */
int gpj_version(void);

/* Message of the last failed call on this thread ("" if none). */
const char *gpj_last_error(void);

/* Context: device binding plus reusable device buffers.  Replaces the
 * reference's per-call cudaMalloc/cudaFree (src/gpjson/cuda/cuda.cpp:33-47).
 * A context may be used from one host thread at a time. */
int gpj_ctx_create(int device, gpj_ctx **out);
int gpj_ctx_destroy(gpj_ctx *ctx);

/* Compiles a JSONPath query into the byte IR.
 * Replaces query::QueryCompiler::compile / QueryParser::compile
 * (include/gpjson/query/query_compiler.hpp:110-116, 86-92).  Same grammar,
 * IR, max_depth and result-slot count for every query in the reference's
 * syntax.  wildcard_limit = 0 rejects "[*]" and ".." as the reference does
 * (query_compiler.cpp:202-204, 287-289).  Extensions the reference rejects:
 *  - K > 0: "[*]" compiles as "[0:K]" preceded by an element-count check
 *    that raises GPJ_QUERY_OVERFLOW for an array of more than K elements;
 *  - K > 0: "..name" as the last step returns every member named `name`
 *    inside the current value at any indexed level, in document order, in K
 *    result slots (max_depth 15: index that many levels to reach them all);
 *  - numeric filters "[?(@<path> <op> <number>)]", op one of == != < <= > >=,
 *    an exact decimal comparison with a JSON number (a value that is not a
 *    number fails the filter; query_compiler.cpp:366-391 takes only
 *    == "string");
 *  - "[-a:-b]" (a > b >= 1): the reverse indexes a .. b+1, in the
 *    reference's own IR (its parser accepts only "[-a:]",
 *    query_compiler.cpp:256-286);
 *  - K > 0: the open slices "[a:]", "[a:-b]" and "[:-b]": elements a ..
 *    a+K-1 that are not among the last b, in K result slots; an array whose
 *    slice holds more than K elements raises GPJ_QUERY_OVERFLOW.
 * "[--" stays rejected with the reference's message. */
int gpj_compile(const char *query, uint64_t wildcard_limit, uint8_t *h_ir,
                uint64_t ir_capacity, uint64_t *ir_len, uint64_t *max_depth,
                uint64_t *num_result_slots);

/* Builds the newline index, string mask and leveled bitmaps (and, with
 * GPJ_INDEX_EMIT_ESCAPE_QUOTE, the escape and quote bitmaps) of one
 * device-resident partition in one fused launch; the library allocates the
 * outputs (free with gpj_index_free).  Returns once num_lines is known.
 * Replaces index::IndexBuilder::build
 * (include/gpjson/index/index_builder.hpp:55-63; builders at
 * src/gpjson/index/{orig,fuse,sharemem}_index_builder.cu). */
int gpj_index_build(gpj_ctx *ctx, const uint8_t *d_input, uint64_t size_bytes,
                    int num_levels, uint32_t flags, gpj_index *out,
                    void *stream);

/* Same build into caller-owned buffers (index->d_string, d_leveled,
 * d_newline with newline_capacity entries, optional d_escape/d_quote).
 * Asynchronous: d_summary must hold 4 x uint64 in device memory and receives
 * d_summary[0] = line count, [1] = final string state, [2] = final depth
 * (sign-extended signed char), [3] = error bits (nonzero: a bounded device
 * wait gave up; bit 0 look-back, bit 1 tile copy, bit 2 pipeline).  Scratch
 * comes from the context.  If the newline count exceeds newline_capacity - 1
 * the extra offsets are dropped; d_summary[0] still holds the true line
 * count.  Replaces the same builders as gpj_index_build. */
int gpj_index_build_async(gpj_ctx *ctx, const uint8_t *d_input,
                          uint64_t size_bytes, int num_levels, uint32_t flags,
                          gpj_index *index, uint64_t *d_summary, void *stream);

/* Index build that allocates nothing, for callers that cannot call
 * cudaMalloc: hosts that reserve all device memory up front and hand out
 * pieces themselves (a database or serving engine that owns the GPU's memory
 * pool), and latency-critical loops that avoid cudaMalloc/cudaFree because
 * those calls can synchronize the device.  No counterpart in the reference.
 * Same inputs, outputs and results as gpj_index_build_async (caller-owned
 * index buffers and d_summary[0..3]: lines, in-string, depth, error bits);
 * no context is needed.  Its scratch is a fixed 1 MiB device array inside the
 * library, so size_bytes is limited to 4 GiB (GPJ_ERR_CAPACITY beyond).  The
 * first call on a device looks up that array's device address (make it
 * before any stream capture) and keeps it for the process: do not use this
 * entry point across a cudaDeviceReset of that device.  CUDA loads modules
 * lazily by default, so the first call (or the first launch of each index
 * kernel variant) is also when the driver places the array and the kernel
 * code in device memory: a host that reserves all device memory up front
 * should make one call per device with its level count before reserving, or
 * run with CUDA_MODULE_LOADING=EAGER.  All calls on a device share the
 * array: calls whose work overlaps on the GPU race.  Unaligned inputs use
 * plain loads instead of TMA. */
#define GPJ_NOALLOC_MAX_BYTES 4294967296ull
int gpj_index_build_noalloc(const uint8_t *d_input, uint64_t size_bytes,
                            int num_levels, uint32_t flags, gpj_index *index,
                            uint64_t *d_summary, void *stream);

/* Copies size_bytes of host memory to device memory on `stream`.  A pinned
 * (page-locked or registered) source is one cudaMemcpyAsync.  A pageable or
 * mmap'd source goes through the context's ring of three 32 MiB pinned
 * chunks: host threads copy chunk k+1 into the ring while chunk k crosses
 * PCIe, one cudaMemcpyAsync per chunk; the call returns once every chunk is
 * staged (the source may then be reused) and the device copy completes in
 * `stream` order.  gpj_query_host stages its pageable inputs the same way,
 * piece by piece, overlapped with the indexing of the pieces before.
 * Replaces the synchronous pageable copy of FilePartition::load_to_device
 * (src/gpjson/file/file.cpp:30-36, src/gpjson/cuda/cuda.cpp:79-87). */
int gpj_copy_to_device(gpj_ctx *ctx, void *d_dst, const void *h_src, uint64_t size_bytes,
                       void *stream);

/* Releases what gpj_index_build allocated.  Like cudaFree it waits for the
 * device to finish the work already queued.  The context keeps up to four
 * released blocks for later builds of a similar size (no cudaMalloc then);
 * gpj_ctx_destroy frees them.  Free an index with the context that built it,
 * before that context is destroyed, or with ctx = NULL (plain cudaFree). */
int gpj_index_free(gpj_ctx *ctx, gpj_index *index);

/* Runs one compiled query over every record of an indexed partition and
 * writes int32 (start, end) pairs, partition-local, -1 = no match, into
 * d_out[num_lines][num_result_slots][2].  Asynchronous on `stream`.
 * Replaces the per-query launch of query::kernels::orig::execute_batch
 * (src/gpjson/query/kernels/orig/query_executor_host.cu:179-237) and the
 * query kernel (src/gpjson/query/kernels/orig/query.cu:144-454). */
int gpj_query_run(gpj_ctx *ctx, const gpj_index *index, const uint8_t *h_ir,
                  uint64_t ir_len, uint32_t num_result_slots, int32_t *d_out,
                  void *stream);

/* As gpj_query_run with int64 offsets, for partitions of 2 GiB and more
 * (the reference narrows sizes to int, query_executor_host.cu:28-33). */
int gpj_query_run64(gpj_ctx *ctx, const gpj_index *index, const uint8_t *h_ir,
                    uint64_t ir_len, uint32_t num_result_slots, int64_t *d_out,
                    void *stream);

/* Status of the queries run on a context: waits for `stream`, returns in
 * *flags the bits raised by the context's query launches since the last call,
 * and clears them.  GPJ_QUERY_OVERFLOW: a record had more results than the
 * query has result slots, so some were dropped -- only the extensions can:
 * a "[*]" array longer than the wildcard limit, or more "..name" matches.
 * The reference compiles neither, so it has no counterpart. */
#define GPJ_QUERY_OVERFLOW 0x100u
int gpj_query_status(gpj_ctx *ctx, uint32_t *flags, void *stream);

/* Options of gpj_query_run_opts; all-zero means the reference behaviour
 * (int32 offsets, records are lines, query level 0 = bitmap level 0). */
typedef struct gpj_query_opts {
  uint32_t base_level;   /* bitmap level that query level 0 maps to: 1 makes
                            the elements of a top-level array the records
                            ("$[*]..." queries) */
  uint32_t offset_bytes; /* 4 (int32, default when 0) or 8 (int64) */
  uint32_t reserved[2];
} gpj_query_opts;

/* gpj_query_run with options (record level, offset width).  Same kernel and
 * replaced interface as gpj_query_run; the array-element records extend the
 * reference, whose compiler rejects "[*]" (query_compiler.cpp:287-289). */
int gpj_query_run_opts(gpj_ctx *ctx, const gpj_index *index, const uint8_t *h_ir,
                       uint64_t ir_len, uint32_t num_result_slots,
                       const gpj_query_opts *opts, void *d_out, void *stream);

/* End to end from host memory: copies h_input to the device, builds the
 * index with num_levels levels, runs the queries and copies the int32 result
 * arrays back.  Inputs above 32 MiB are copied in pieces on a second stream
 * and each piece is indexed as soon as it is on the device (pinned host
 * memory makes the copies overlap the indexing).  h_out[q] must hold
 * out_capacity[q] int32; *num_lines gets the record count (0 for an empty
 * input).  base_levels may be NULL (all 0).  GPJ_ERR_CAPACITY (nothing
 * copied back) if a result does not fit; GPJ_ERR_CAPACITY after the copies
 * if a record had more results than result slots (GPJ_QUERY_OVERFLOW).  Replaces the per-partition body
 * of gpjson::Engine::query (src/gpjson/engine.cpp:131-166: load_to_device,
 * build, execute_batch). */
int gpj_query_host(gpj_ctx *ctx, const uint8_t *h_input, uint64_t size_bytes,
                   int num_levels, uint32_t num_queries,
                   const uint8_t *const *h_irs, const uint64_t *ir_lens,
                   const uint32_t *num_result_slots, const uint32_t *base_levels,
                   int32_t *const *h_out, const uint64_t *out_capacity,
                   uint64_t *num_lines, void *stream);

/* One match of a compacted result array (gpj_results_compact). */
typedef struct gpj_match {
  uint64_t line;         /* record (line) index */
  uint32_t slot;         /* result slot of the query */
  uint32_t length;       /* end - start */
  int64_t start;         /* global byte offset: base_offset + partition-local start */
  int64_t end;           /* global end offset, exclusive */
  uint64_t text_offset;  /* first byte of the match in the arena */
} gpj_match;

/* Compacts one query's int32 result array d_results[num_lines][slots][2]
 * (partition-local, -1 = no match) on the device: the matches in (line,
 * slot) order with global offsets into d_matches, and the matched bytes of
 * d_input, concatenated in the same order, into d_arena.  d_counts (3
 * words, device) receives the number of matches, the arena bytes they need
 * and the number of invalid ranges (start > end or end > size_bytes, which
 * the reference reports as "Query kernel produced an invalid result range").
 * Matches and bytes beyond match_capacity / arena_capacity are counted but
 * not written: call again with larger buffers.  d_arena or d_input may be
 * NULL (offsets only).  Asynchronous on `stream`.  Replaces the host loop of
 * append_query_line_results (src/gpjson/query/kernels/orig/
 * query_executor_host.cu:80-119): only the matches and their bytes need to
 * be copied to the host. */
int gpj_results_compact(gpj_ctx *ctx, const int32_t *d_results, uint64_t num_lines,
                        uint32_t num_result_slots, const uint8_t *d_input,
                        uint64_t size_bytes, int64_t base_offset, gpj_match *d_matches,
                        uint64_t match_capacity, uint8_t *d_arena, uint64_t arena_capacity,
                        uint64_t *d_counts, void *stream);

/* ------------------------------------------------------------------------ */
/* Batched path: many files indexed and queried by one launch chain         */
/* ------------------------------------------------------------------------ */

#define GPJ_BATCH_AUTOTUNE 4u /* time the launch shapes at creation, keep the fastest: indexer
                                 tile size and variant, then query block and grid */
#define GPJ_BATCH_NO_GRAPH 8u /* launch the kernels directly instead of a CUDA graph */
/* Indexer variant without GPJ_BATCH_AUTOTUNE (gpj_batch_view.index_variant;
 * indexes of up to 4 levels, same outputs): */
#define GPJ_BATCH_INDEX_LANE_WALK 16u      /* each lane walks its own leveled quarters */
#define GPJ_BATCH_INDEX_WIDE_LOOKBACK 32u  /* look-back rounds of 64 descriptors */

/* One file of a batch: `offset` (a multiple of 128) and `size_bytes` inside
 * the batch's device buffer; `query` indexes the batch's query table. */
typedef struct gpj_batch_file {
  uint64_t offset;
  uint64_t size_bytes;
  uint32_t query;
  uint32_t reserved;
} gpj_batch_file;

/* A compiled query applied to every record of the files that name it.
 * num_levels = bitmap levels indexed for those files; base_level as in
 * gpj_query_opts. */
typedef struct gpj_batch_query {
  const uint8_t *h_ir;
  uint64_t ir_len;
  uint32_t num_result_slots;
  uint32_t base_level;
  uint32_t num_levels;
  uint32_t reserved;
} gpj_batch_query;

/* Device-resident outputs of a batch (owned by the batch).
 * d_file_info: 8 uint64 per file: lines, first newline-index slot, first
 * record, first result int, final in-string state, final depth, size, query.
 * d_newline: every file's newline index packed (file f at its slot);
 * d_results: int32 [lines][slots][2] per file at its first result int, with
 * file-local offsets; d_string/d_leveled: per-file words at the offsets of
 * gpj_batch_file_layout.  d_totals: records, result ints, newline slots,
 * error bits (nonzero: a bounded device wait gave up). */
typedef struct gpj_batch_view {
  uint64_t *d_string;
  uint64_t *d_leveled;
  int64_t *d_newline;
  int32_t *d_results;
  uint64_t *d_file_info;
  uint64_t *d_totals;
  uint64_t num_files;
  uint64_t num_records;
  uint64_t result_ints;
  uint64_t newline_slots;
  uint64_t string_words;
  uint64_t leveled_words;
  uint32_t num_tiles;
  uint32_t index_threads; /* indexer CTA size: tiles of index_threads * 128 B */
  uint32_t query_block;
  uint32_t query_grid;
  uint32_t uses_graph;
  uint32_t index_variant; /* indexer variant bits for up to 4 levels: 1 = each lane walks its
                             own leveled quarters (no per-warp list), 2 = look-back rounds of
                             64 descriptors (else 32); the outputs are the same for all */
} gpj_batch_view;

typedef struct gpj_batch gpj_batch;

/* Plans a batch over a 16-byte aligned device buffer: sizes every output
 * with one run (the only host round trip), optionally autotunes the launch
 * shapes, and captures index -> per-file finalize -> query in a CUDA graph.
 * Replaces the per-partition loop of gpjson::Engine::query
 * (src/gpjson/engine.cpp:131-166) run once per file, for many files at once;
 * the batching itself has no counterpart in the reference. */
int gpj_batch_create(gpj_ctx *ctx, const uint8_t *d_input, uint64_t input_bytes,
                     const gpj_batch_file *files, uint32_t num_files,
                     const gpj_batch_query *queries, uint32_t num_queries,
                     uint32_t flags, gpj_batch **out, void *stream);

/* Replays the batch on `stream` (asynchronous). */
int gpj_batch_run(gpj_batch *batch, void *stream);

/* Runs only some stages of the batch, directly (no graph), in the order
 * index, finalize, query: for timing and profiling one kernel. */
#define GPJ_BATCH_STAGE_INDEX 1u
#define GPJ_BATCH_STAGE_FINALIZE 2u
#define GPJ_BATCH_STAGE_QUERY 4u
int gpj_batch_run_stages(gpj_batch *batch, uint32_t stages, void *stream);

/* The same work as gpj_batch_run, issued the plain way: one single-file
 * index launch and one query launch per file, into the same outputs (the
 * comparison point of the batched path; no host round trips). */
int gpj_batch_run_per_file(gpj_batch *batch, void *stream);

/* End to end from host memory: copies h_input (input_bytes, the batch's
 * layout) into the batch's device input buffer, runs the batch, copies the
 * result ints (view.result_ints) and the per-file info (8 uint64 per file)
 * back, and waits.  Either output pointer may be NULL.  Above 32 MiB, with
 * the files in table order and not overlapping, the input is copied in
 * groups of whole files and each group is indexed as soon as it lands; the
 * finalize and the queries follow the last group. */
int gpj_batch_run_host(gpj_batch *batch, const uint8_t *h_input, int32_t *h_results,
                       uint64_t *h_file_info, void *stream);

/* Device pointers and sizes of the batch outputs. */
int gpj_batch_view_get(const gpj_batch *batch, gpj_batch_view *view);

/* Word offsets of one file's string-mask and leveled-bitmap words
 * (leveled words are level-major with the file's own word count). */
int gpj_batch_file_layout(const gpj_batch *batch, uint32_t file,
                          uint64_t *string_off, uint64_t *leveled_off,
                          uint32_t *num_levels);

int gpj_batch_destroy(gpj_batch *batch);

/* ---- Serving: continuous batching with resident indexes ------------------
 *
 * A server owns one device arena (the HBM budget), one pinned host arena for
 * results, and num_slots CUDA streams.  The cache misses admitted in one
 * scheduler pass are indexed by ONE launch of the multi-file indexer over the
 * arena (then each request's queries run on its own stream);
 * GPJ_SERVER_NO_GROUPS builds each with its own launch instead.  A scheduler thread admits submitted
 * requests in arrival order whenever a slot is free and the request's device
 * footprint (input copy, bitmaps, newline index, scratch, results) fits the
 * arena, evicting idle resident indexes least-recently-used first.  Admitted
 * requests run concurrently, one per stream: H2D copy -> index build ->
 * queries -> D2H of the results.  Indexes of requests with a nonzero file_key
 * stay resident after completion, so later requests for the same key and size
 * skip the copy and the build; a request whose key is being built by another
 * request waits for that build instead of repeating it.
 *
 * The reference answers one Engine::query call at a time and rebuilds every
 * index (src/gpjson/engine.cpp:131-166); the server has no counterpart there
 * and runs the same index and query kernels as gpj_index_build_async and
 * gpj_query_run, so each request's results equal those of that plain path. */
typedef struct gpj_server gpj_server;

#define GPJ_SERVER_NO_CACHE 1u /* never keep indexes resident */
#define GPJ_SERVER_SLEEP_POLL 2u /* scheduler sleeps between event polls */
#define GPJ_SERVER_NO_GROUPS 4u  /* build each cache miss with its own launch */
#define GPJ_SERVER_MAX_QUERIES 8

typedef struct gpj_server_config {
  int32_t device;
  int32_t num_slots;           /* requests on the device at once; 0 = 32 */
  uint64_t hbm_budget_bytes;   /* device arena; 0 = 1 GiB */
  uint64_t host_result_bytes;  /* pinned result arena; 0 = 256 MiB */
  int32_t cache_levels;        /* levels built for resident indexes (at least
                                  each request's own need); 0 = 4 */
  uint32_t flags;              /* GPJ_SERVER_* */
  uint32_t reserved[4];
} gpj_server_config;

/* One request: a file and 1..GPJ_SERVER_MAX_QUERIES compiled queries (the
 * gpj_batch_query fields: IR, result slots, base level, levels needed).
 * h_input must stay valid until the request completes; pinned host memory
 * makes the copy asynchronous.  arrival_ns: the caller's arrival time on
 * CLOCK_MONOTONIC (0 = the time of submission), the start of the measured
 * latency.  Files are limited to 2^31 - 1 bytes (int32 offsets). */
typedef struct gpj_request {
  uint64_t file_key;           /* resident-index identity; 0 = do not cache */
  const uint8_t *h_input;
  uint64_t size_bytes;
  const gpj_batch_query *queries;
  uint32_t num_queries;
  uint32_t reserved;
  uint64_t arrival_ns;
} gpj_request;

/* A finished request.  h_results points into the server's pinned arena and
 * stays valid until gpj_server_release: query q's block starts at int
 * result_offset[q] and holds int32 [num_lines][slots_q][2] partition-local
 * [start, end) pairs, -1 where a slot matched nothing (the layout of
 * gpj_query_run). */
typedef struct gpj_response {
  int32_t status;              /* GPJ_OK or the failure's code */
  int32_t cache_hit;           /* 1: the index was resident (or being built) */
  uint64_t num_lines;
  const int32_t *h_results;
  uint64_t result_ints;
  uint64_t result_offset[GPJ_SERVER_MAX_QUERIES];
  uint64_t arrival_ns;
  uint64_t admit_ns;           /* slot and memory granted */
  uint64_t index_ready_ns;     /* index available (build done, or cached) */
  uint64_t done_ns;            /* results on the host */
  char message[128];           /* failure message, "" on success */
} gpj_response;

typedef struct gpj_server_stats {
  uint64_t submitted, completed, failed;
  uint64_t cache_hits, cache_misses, evictions, rebuilds;
  uint64_t bytes_indexed;      /* input bytes copied and indexed */
  uint64_t bytes_served;       /* input bytes of completed requests */
  uint64_t resident_indexes, resident_bytes;
  uint64_t arena_used, arena_peak, arena_bytes;
  uint64_t in_flight, pending;
  uint64_t index_launches;     /* indexer launches (a grouped build is one) */
} gpj_server_stats;

int gpj_server_create(const gpj_server_config *config, gpj_server **out);

/* Queues a request (copies the request and its IRs); returns its id. */
int gpj_server_submit(gpj_server *server, const gpj_request *request, uint64_t *request_id);

/* Queues `count` requests at once (one lock, one wake-up of the scheduler);
 * request_ids[i] gets the id of requests[i].  All are checked first: on an
 * error nothing is queued. */
int gpj_server_submit_many(gpj_server *server, const gpj_request *requests, uint32_t count,
                           uint64_t *request_ids);

/* Waits up to timeout_us (negative: forever) for finished requests not yet
 * reported by this call and returns up to capacity of their ids. */
int gpj_server_poll(gpj_server *server, uint64_t *ids, uint32_t capacity, uint32_t *count,
                    int64_t timeout_us);

/* Waits up to timeout_us (negative: forever) for one request; GPJ_ERR_TIMEOUT
 * if it is still running. */
int gpj_server_wait(gpj_server *server, uint64_t request_id, int64_t timeout_us);

/* Response of a finished request (GPJ_ERR_OUT_OF_RANGE if unknown or
 * released, GPJ_ERR_TIMEOUT if not finished). */
int gpj_server_response(gpj_server *server, uint64_t request_id, gpj_response *out);

/* Frees a finished request's host results. */
int gpj_server_release(gpj_server *server, uint64_t request_id);

int gpj_server_stats_get(gpj_server *server, gpj_server_stats *out);

/* Drops every idle resident index. */
int gpj_server_clear_cache(gpj_server *server);

/* Finishes the requests on the device, fails the queued ones, frees all. */
int gpj_server_destroy(gpj_server *server);

#ifdef __cplusplus
}
#endif

#endif /* GPJSON_B200_H */
