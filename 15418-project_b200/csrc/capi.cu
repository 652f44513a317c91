// C ABI of the engine (include/gpjson_b200.h): argument checks, device
// buffer reuse, launches and error reporting.  No CPU fallback: every entry
// point that computes needs a CUDA device and fails with GPJ_ERR_CUDA
// otherwise.
#include "compact.cuh"
#include "compiler.hpp"
#include "indexer.cuh"
#include "query.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <utility>
#include <vector>

struct gpj_ctx {
  int device = 0;
  // grow-only device buffers
  void *scratch = nullptr;
  uint64_t scratch_bytes = 0;
  void *staging = nullptr;  // aligned copy of unaligned inputs / host inputs
  uint64_t staging_bytes = 0;
  // host_query(): index + results kept between calls
  void *host_index = nullptr;
  uint64_t host_index_bytes = 0;
  void *host_results = nullptr;
  uint64_t host_results_bytes = 0;
  unsigned long long *pinned = nullptr;  // 8 words of pinned host memory
  void *compact_scratch = nullptr;  // per-block counts of gpj_results_compact
  uint64_t compact_scratch_bytes = 0;
  // host inputs arrive in pieces on a copy stream (created on first use)
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t piece_ready = nullptr;
  // status bits the context's query launches raise (GPJ_QUERY_OVERFLOW)
  unsigned int *d_status = nullptr;
  // pinned staging ring for pageable or mmap'd host inputs (created on first
  // use): a slot is refilled once the copy that last read it has finished
  void *stage = nullptr;
  cudaEvent_t stage_done[3] = {nullptr, nullptr, nullptr};
  int stage_next = 0;
  // gpj_index_build allocations: sizes of the live ones, and the ones
  // gpj_index_free released, kept for the next build of a similar size (a
  // cudaMalloc/cudaFree pair of tens of MB costs milliseconds)
  std::unordered_map<void *, uint64_t> index_live;
  std::vector<std::pair<void *, uint64_t>> index_spare;
};

namespace {

thread_local std::string g_error;

int fail(int code, const std::string &msg) {
  g_error = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char *what) {
  (void)cudaGetLastError();
  const int code = (e == cudaErrorMemoryAllocation) ? GPJ_ERR_OOM : GPJ_ERR_CUDA;
  return fail(code, std::string(what) + ": " + cudaGetErrorString(e));
}

#define GPJ_CUDA(call, what)                      \
  do {                                            \
    const cudaError_t e_ = (call);                \
    if (e_ != cudaSuccess) return cuda_fail(e_, what); \
  } while (0)

int ensure(void *&buf, uint64_t &have, uint64_t need) {
  if (need <= have && buf != nullptr) return GPJ_OK;
  if (buf != nullptr) {
    cudaFree(buf);
    buf = nullptr;
    have = 0;
  }
  if (need == 0) need = 256;
  GPJ_CUDA(cudaMalloc(&buf, need), "cudaMalloc");
  have = need;
  return GPJ_OK;
}

int bind_device(gpj_ctx *ctx) {
  if (ctx == nullptr) return fail(GPJ_ERR_INVALID_ARGUMENT, "null context");
  GPJ_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
  return GPJ_OK;
}

uint64_t round256(uint64_t x) { return (x + 255u) & ~uint64_t(255); }

// Newline-index capacity guess for a fresh build: one record per 32 bytes
// covers every realistic JSON-lines file; a build that finds more newlines
// is repeated with the exact size.
uint64_t nl_capacity_guess(uint64_t n) { return n / 32u + 1024u; }

// Enqueues the fused indexer.  `in` may be unaligned: it is then copied into
// the context's staging buffer first (TMA needs 16-byte aligned rows).
int enqueue_index(gpj_ctx *ctx, const uint8_t *in, uint64_t n, int levels,
                  uint32_t flags, const gpj_index &out, cudaStream_t stream) {
  gpjb::IndexLaunch L;
  L.single.n = n;
  L.single.levels = levels;
  L.num_levels = levels;
  L.full_rows = n / 128u;
  L.S = out.d_string;
  L.LB = out.d_leveled;
  L.E = (flags & GPJ_INDEX_EMIT_ESCAPE_QUOTE) ? out.d_escape : nullptr;
  L.Q = (flags & GPJ_INDEX_EMIT_ESCAPE_QUOTE) ? out.d_quote : nullptr;
  L.NL = out.d_newline;
  L.nl_cap = out.newline_capacity;
  L.num_tiles = uint32_t(gpjb::index_num_tiles(n));

  const uint8_t *src = in;
  if (n > 0 && (reinterpret_cast<uintptr_t>(in) & 15u) != 0) {
    int rc = ensure(ctx->staging, ctx->staging_bytes, round256(n));
    if (rc != GPJ_OK) return rc;
    GPJ_CUDA(cudaMemcpyAsync(ctx->staging, in, n, cudaMemcpyDeviceToDevice, stream),
             "copy unaligned input");
    src = static_cast<const uint8_t *>(ctx->staging);
  }
  L.in = src;

  int rc = ensure(ctx->scratch, ctx->scratch_bytes, gpjb::index_scratch_bytes(n));
  if (rc != GPJ_OK) return rc;
  gpjb::index_bind_scratch(L, ctx->scratch);

  CUtensorMap map;
  bool tma = false;
  if ((flags & GPJ_INDEX_NO_TMA) == 0) tma = gpjb::index_make_tensor_map(&map, src, n);
  if (n == 0) {
    // no tiles: NL = [0], one line, empty bitmaps; the summary is written
    // here because no kernel runs
    const unsigned long long summary[4] = {1ull, 0ull, ~0ull, 0ull};
    GPJ_CUDA(cudaMemsetAsync(ctx->scratch, 0, 64, stream), "cudaMemsetAsync");
    GPJ_CUDA(cudaMemcpyAsync(L.summary, summary, sizeof(summary), cudaMemcpyHostToDevice,
                             stream),
             "summary");
    if (out.newline_capacity > 0)
      GPJ_CUDA(cudaMemsetAsync(out.d_newline, 0, sizeof(int64_t), stream), "cudaMemsetAsync");
    return GPJ_OK;
  }
  if (flags & GPJ_INDEX_DIAG_TILE0_UNPUBLISHED) {
    if (L.num_tiles < 2)
      return fail(GPJ_ERR_INVALID_ARGUMENT,
                  "GPJ_INDEX_DIAG_TILE0_UNPUBLISHED needs an input of at least two tiles");
    L.lookback_spin_limit = 1u << 14;
    GPJ_CUDA(gpjb::index_clear_scratch(L, stream), "cudaMemsetAsync");
    GPJ_CUDA(gpjb::index_launch_range(L, tma ? &map : nullptr, tma, stream, 1u, L.num_tiles),
             "index kernel launch");
    return GPJ_OK;
  }
  GPJ_CUDA(gpjb::index_launch(L, tma ? &map : nullptr, tma, stream), "index kernel launch");
  return GPJ_OK;
}

// ---- Host -> device copies -------------------------------------------------
//
// A pinned (page-locked or registered) source is copied by the DMA engines
// directly.  A pageable or mmap'd source would make every cudaMemcpyAsync
// synchronous and staged through the driver's small bounce buffer; instead it
// goes through a ring of pinned chunks: host threads copy chunk k+1 into the
// ring while chunk k crosses PCIe, one cudaMemcpyAsync per chunk.
constexpr uint64_t kStageChunk = 32ull << 20;
constexpr int kStageSlots = 3;
constexpr int kStageThreads = 4;

bool host_is_pinned(const void *p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

// memcpy split over a few host threads (one thread copies ~10 GB/s, PCIe
// Gen5 takes ~55)
void parallel_memcpy(uint8_t *dst, const uint8_t *src, uint64_t n) {
  if (n < (4ull << 20)) {
    std::memcpy(dst, src, n);
    return;
  }
  const uint64_t part = ((n + kStageThreads - 1) / kStageThreads + 4095u) & ~uint64_t(4095);
  std::thread workers[kStageThreads - 1];
  for (int t = 1; t < kStageThreads; ++t) {
    const uint64_t off = uint64_t(t) * part;
    if (off < n)
      workers[t - 1] = std::thread(
          [=] { std::memcpy(dst + off, src + off, std::min<uint64_t>(part, n - off)); });
  }
  std::memcpy(dst, src, std::min<uint64_t>(part, n));
  for (auto &w : workers)
    if (w.joinable()) w.join();
}

// Enqueues the copy of [h, h + n) to d on `stream`.  Pageable sources are
// staged; when this returns, the source may be reused.
int stage_copy(gpj_ctx *ctx, uint8_t *d, const uint8_t *h, uint64_t n, cudaStream_t stream,
               bool pinned) {
  if (n == 0) return GPJ_OK;
  if (pinned) {
    GPJ_CUDA(cudaMemcpyAsync(d, h, n, cudaMemcpyHostToDevice, stream), "copy input");
    return GPJ_OK;
  }
  if (ctx->stage == nullptr) {
    GPJ_CUDA(cudaMallocHost(&ctx->stage, kStageChunk * kStageSlots), "cudaMallocHost");
    for (auto &e : ctx->stage_done)
      GPJ_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
  }
  auto *ring = static_cast<uint8_t *>(ctx->stage);
  for (uint64_t off = 0; off < n; off += kStageChunk) {
    const uint64_t len = std::min(kStageChunk, n - off);
    const int slot = ctx->stage_next;
    ctx->stage_next = (slot + 1) % kStageSlots;
    GPJ_CUDA(cudaEventSynchronize(ctx->stage_done[slot]), "cudaEventSynchronize");
    uint8_t *chunk = ring + uint64_t(slot) * kStageChunk;
    parallel_memcpy(chunk, h + off, len);
    GPJ_CUDA(cudaMemcpyAsync(d + off, chunk, len, cudaMemcpyHostToDevice, stream),
             "copy staged input");
    GPJ_CUDA(cudaEventRecord(ctx->stage_done[slot], stream), "cudaEventRecord");
  }
  return GPJ_OK;
}

// Pieces of a host input: copied in this many tiles at a time on the copy
// stream, each piece indexed as soon as it has arrived, so the index of one
// piece overlaps the copy of the next.
constexpr uint32_t kIngestPieceTiles = 1024;  // 32 MiB

// Copies n host bytes to d_in (256-byte aligned) and indexes them on
// `stream`: inputs of more than one piece are copied piece by piece on the
// context's copy stream, and one indexer launch per piece claims its tiles
// once the piece is on the device (the look-back reads the finished
// descriptors of the pieces before it).
int enqueue_index_from_host(gpj_ctx *ctx, const uint8_t *h_in, uint8_t *d_in, uint64_t n,
                            int levels, const gpj_index &out, cudaStream_t stream) {
  const uint64_t piece = uint64_t(kIngestPieceTiles) * gpjb::kTileBytes;
  const bool pinned = n > 0 && host_is_pinned(h_in);
  if (n <= piece) {
    const int rc = stage_copy(ctx, d_in, h_in, n, stream, pinned);
    if (rc != GPJ_OK) return rc;
    return enqueue_index(ctx, d_in, n, levels, 0u, out, stream);
  }
  if (ctx->copy_stream == nullptr)
    GPJ_CUDA(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking),
             "cudaStreamCreate");
  if (ctx->piece_ready == nullptr)
    GPJ_CUDA(cudaEventCreateWithFlags(&ctx->piece_ready, cudaEventDisableTiming),
             "cudaEventCreate");
  gpjb::IndexLaunch L;
  L.in = d_in;
  L.single.n = n;
  L.single.levels = levels;
  L.num_levels = levels;
  L.full_rows = n / 128u;
  L.S = out.d_string;
  L.LB = out.d_leveled;
  L.NL = out.d_newline;
  L.nl_cap = out.newline_capacity;
  L.num_tiles = uint32_t(gpjb::index_num_tiles(n));
  int rc = ensure(ctx->scratch, ctx->scratch_bytes, gpjb::index_scratch_bytes(n));
  if (rc != GPJ_OK) return rc;
  gpjb::index_bind_scratch(L, ctx->scratch);
  CUtensorMap map;
  const bool tma = gpjb::index_make_tensor_map(&map, d_in, n);
  GPJ_CUDA(gpjb::index_clear_scratch(L, stream), "cudaMemsetAsync");
  // the copies start after the work already queued on `stream`
  GPJ_CUDA(cudaEventRecord(ctx->piece_ready, stream), "cudaEventRecord");
  GPJ_CUDA(cudaStreamWaitEvent(ctx->copy_stream, ctx->piece_ready, 0), "cudaStreamWaitEvent");
  for (uint32_t t0 = 0; t0 < L.num_tiles; t0 += kIngestPieceTiles) {
    const uint32_t t1 = t0 + kIngestPieceTiles < L.num_tiles ? t0 + kIngestPieceTiles : L.num_tiles;
    const uint64_t b0 = uint64_t(t0) * gpjb::kTileBytes;
    const uint64_t b1 = uint64_t(t1) * gpjb::kTileBytes < n ? uint64_t(t1) * gpjb::kTileBytes : n;
    const int rc = stage_copy(ctx, d_in + b0, h_in + b0, b1 - b0, ctx->copy_stream, pinned);
    if (rc != GPJ_OK) return rc;
    GPJ_CUDA(cudaEventRecord(ctx->piece_ready, ctx->copy_stream), "cudaEventRecord");
    GPJ_CUDA(cudaStreamWaitEvent(stream, ctx->piece_ready, 0), "cudaStreamWaitEvent");
    GPJ_CUDA(gpjb::index_clear_counter(L, stream), "cudaMemsetAsync");
    GPJ_CUDA(gpjb::index_launch_range(L, tma ? &map : nullptr, tma, stream, t0, t1),
             "index kernel launch");
  }
  return GPJ_OK;
}

// summary words in the context scratch: [lines, in_string, depth, pad] then
// the error word
const unsigned long long *summary_ptr(gpj_ctx *ctx, uint64_t n) {
  gpjb::IndexLaunch L;
  L.num_tiles = uint32_t(gpjb::index_num_tiles(n));
  gpjb::index_bind_scratch(L, ctx->scratch);
  return L.summary;
}
const unsigned int *error_ptr(gpj_ctx *ctx, uint64_t n) {
  gpjb::IndexLaunch L;
  L.num_tiles = uint32_t(gpjb::index_num_tiles(n));
  gpjb::index_bind_scratch(L, ctx->scratch);
  return L.error;
}

// Copies the summary and error word to pinned memory and waits.
int read_summary(gpj_ctx *ctx, uint64_t n, cudaStream_t stream, uint64_t *lines,
                 int *in_string, int *depth) {
  GPJ_CUDA(cudaMemcpyAsync(ctx->pinned, summary_ptr(ctx, n), 32, cudaMemcpyDeviceToHost,
                           stream),
           "read index summary");
  GPJ_CUDA(cudaMemcpyAsync(ctx->pinned + 4, error_ptr(ctx, n), 4, cudaMemcpyDeviceToHost,
                           stream),
           "read index error word");
  GPJ_CUDA(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
  const unsigned int err = reinterpret_cast<const unsigned int *>(ctx->pinned + 4)[0];
  if (n > 0 && err != 0)
    return fail(GPJ_ERR_TIMEOUT, "index kernel: a bounded wait gave up (error bits " +
                                     std::to_string(err) + ")");
  *lines = ctx->pinned[0];
  *in_string = int(ctx->pinned[1]);
  *depth = int(int64_t(ctx->pinned[2]));
  return GPJ_OK;
}

constexpr size_t kSpareIndexBlocks = 4;

// Releases an index allocation.  With its context the block is kept for
// reuse after a device synchronisation (what cudaFree implies: work still
// reading the index has finished); the largest spare goes once more than
// kSpareIndexBlocks are kept.
void release_index(gpj_ctx *ctx, gpj_index *ix) {
  void *mem = ix->owner;
  std::memset(ix, 0, sizeof(*ix));
  if (mem == nullptr) return;
  auto it = ctx != nullptr ? ctx->index_live.find(mem) : decltype(ctx->index_live)::iterator{};
  if (ctx == nullptr || it == ctx->index_live.end() || cudaSetDevice(ctx->device) != cudaSuccess ||
      cudaDeviceSynchronize() != cudaSuccess) {
    if (ctx != nullptr && it != ctx->index_live.end()) ctx->index_live.erase(it);
    cudaFree(mem);
    return;
  }
  ctx->index_spare.emplace_back(mem, it->second);
  ctx->index_live.erase(it);
  if (ctx->index_spare.size() > kSpareIndexBlocks) {
    auto big = std::max_element(ctx->index_spare.begin(), ctx->index_spare.end(),
                                [](const auto &a, const auto &b) { return a.second < b.second; });
    cudaFree(big->first);
    ctx->index_spare.erase(big);
  }
}

// One device block of at least `bytes`: the smallest spare that is not more
// than 1.5x (+ 16 MiB) larger, else a new cudaMalloc.
int take_index_block(gpj_ctx *ctx, uint64_t bytes, void **mem) {
  *mem = nullptr;
  auto best = ctx->index_spare.end();
  for (auto it = ctx->index_spare.begin(); it != ctx->index_spare.end(); ++it) {
    if (it->second >= bytes && it->second <= bytes + bytes / 2 + (16u << 20) &&
        (best == ctx->index_spare.end() || it->second < best->second))
      best = it;
  }
  uint64_t got = bytes;
  if (best != ctx->index_spare.end()) {
    *mem = best->first;
    got = best->second;
    ctx->index_spare.erase(best);
  } else {
    cudaError_t e = cudaMalloc(mem, bytes);
    if (e == cudaErrorMemoryAllocation && !ctx->index_spare.empty()) {
      // the spares may be what stands in the way
      (void)cudaGetLastError();
      for (auto &b : ctx->index_spare) cudaFree(b.first);
      ctx->index_spare.clear();
      e = cudaMalloc(mem, bytes);
    }
    GPJ_CUDA(e, "cudaMalloc index");
  }
  ctx->index_live[*mem] = got;
  return GPJ_OK;
}

// Carves one allocation into the index arrays.
int alloc_index(gpj_ctx *ctx, gpj_index *ix, uint64_t n, int levels, bool eq, uint64_t nl_cap) {
  const uint64_t W = (n + 63u) / 64u;
  const uint64_t s_bytes = round256(W * 8u);
  const uint64_t lb_bytes = round256(W * 8u * uint64_t(levels));
  const uint64_t nl_bytes = round256(nl_cap * 8u);
  const uint64_t eq_bytes = eq ? 2u * s_bytes : 0u;
  void *mem = nullptr;
  const int rc = take_index_block(ctx, s_bytes + lb_bytes + nl_bytes + eq_bytes + 256u, &mem);
  if (rc != GPJ_OK) return rc;
  auto *p = static_cast<unsigned char *>(mem);
  ix->owner = mem;
  ix->d_string = reinterpret_cast<uint64_t *>(p);
  ix->d_leveled = reinterpret_cast<uint64_t *>(p + s_bytes);
  ix->d_newline = reinterpret_cast<int64_t *>(p + s_bytes + lb_bytes);
  ix->newline_capacity = nl_cap;
  if (eq) {
    ix->d_escape = reinterpret_cast<uint64_t *>(p + s_bytes + lb_bytes + nl_bytes);
    ix->d_quote = reinterpret_cast<uint64_t *>(p + s_bytes + lb_bytes + nl_bytes + s_bytes);
  } else {
    ix->d_escape = nullptr;
    ix->d_quote = nullptr;
  }
  ix->num_words = W;
  ix->num_levels = levels;
  return GPJ_OK;
}

int check_levels(int levels) {
  if (levels < 0 || levels > GPJ_MAX_LEVELS)
    return fail(GPJ_ERR_INVALID_ARGUMENT,
                "num_levels must be in [0, " + std::to_string(GPJ_MAX_LEVELS) + "]");
  return GPJ_OK;
}

template <typename OutT>
int run_query(gpj_ctx *ctx, const gpj_index *ix, const uint8_t *h_ir, uint64_t ir_len,
              uint32_t slots, OutT *d_out, cudaStream_t stream, uint32_t base_level = 0) {
  if (ix == nullptr || d_out == nullptr || h_ir == nullptr)
    return fail(GPJ_ERR_INVALID_ARGUMENT, "null argument");
  if (ir_len > uint64_t(GPJ_MAX_QUERY_IR))
    return fail(GPJ_ERR_EXECUTION, "Compiled query IR exceeds constant memory buffer");
  if (ix->num_lines == 0 || ix->size_bytes == 0) return GPJ_OK;
  if (ix->num_lines > ix->newline_capacity)
    return fail(GPJ_ERR_CAPACITY, "newline index was truncated: rebuild with capacity >= " +
                                      std::to_string(ix->num_lines));
  if (base_level > 0 && int64_t(base_level) >= int64_t(ix->num_levels))
    return fail(GPJ_ERR_EXECUTION, "Query requires more bitmap levels than the index provides");
  if (sizeof(OutT) == 4 && ix->size_bytes > 0x7FFFFFFFull)
    return fail(GPJ_ERR_EXECUTION, "partition size exceeds CUDA int range");
  int rc = bind_device(ctx);
  if (rc != GPJ_OK) return rc;
  gpjb::QueryLaunch q;
  q.in = ix->d_input;
  q.n = int64_t(ix->size_bytes);
  q.NL = ix->d_newline;
  q.num_lines = int64_t(ix->num_lines);
  q.S = ix->d_string;
  q.LB = ix->d_leveled;
  q.W = int64_t(ix->num_words);
  q.ir_len = int(ir_len);
  q.num_results = int(slots);
  q.base_level = int(base_level);
  q.num_levels = ix->num_levels;
  if constexpr (sizeof(OutT) == 8) q.out64 = reinterpret_cast<int64_t *>(d_out);
  else q.out32 = reinterpret_cast<int32_t *>(d_out);
  q.status = ctx->d_status;
  gpjb::IrBlob blob;
  std::memset(blob.bytes, 0, sizeof(blob.bytes));
  std::memcpy(blob.bytes, h_ir, size_t(ir_len));
  GPJ_CUDA(gpjb::query_launch(q, blob, 0, 256, stream), "query kernel launch");
  return GPJ_OK;
}

}  // namespace

namespace gpjb {
// Records the last-error message for entry points defined in other files.
int report_error(int code, const char *message) { return fail(code, message); }
}  // namespace gpjb

extern "C" {

int gpj_version(void) { return 100; }

const char *gpj_last_error(void) { return g_error.c_str(); }

int gpj_ctx_create(int device, gpj_ctx **out) {
  if (out == nullptr) return fail(GPJ_ERR_INVALID_ARGUMENT, "null output");
  *out = nullptr;
  int count = 0;
  const cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0)
    return fail(GPJ_ERR_CUDA, "no CUDA device: the B200 engine has no CPU path");
  if (device < 0 || device >= count) return fail(GPJ_ERR_INVALID_ARGUMENT, "bad device");
  GPJ_CUDA(cudaSetDevice(device), "cudaSetDevice");
  gpj_ctx *ctx = new (std::nothrow) gpj_ctx;
  if (ctx == nullptr) return fail(GPJ_ERR_OOM, "host allocation");
  ctx->device = device;
  void *pinned = nullptr;
  const cudaError_t pe = cudaMallocHost(&pinned, 64);
  if (pe != cudaSuccess) {
    delete ctx;
    return cuda_fail(pe, "cudaMallocHost");
  }
  ctx->pinned = static_cast<unsigned long long *>(pinned);
  void *status = nullptr;
  cudaError_t se = cudaMalloc(&status, 256);
  if (se == cudaSuccess) se = cudaMemset(status, 0, 256);
  if (se != cudaSuccess) {
    cudaFree(status);
    cudaFreeHost(pinned);
    delete ctx;
    return cuda_fail(se, "cudaMalloc");
  }
  ctx->d_status = static_cast<unsigned int *>(status);
  *out = ctx;
  return GPJ_OK;
}

int gpj_copy_to_device(gpj_ctx *ctx, void *d_dst, const void *h_src, uint64_t size_bytes,
                       void *stream_) {
  int rc = bind_device(ctx);
  if (rc != GPJ_OK) return rc;
  if (size_bytes > 0 && (d_dst == nullptr || h_src == nullptr))
    return fail(GPJ_ERR_INVALID_ARGUMENT, "null buffer with nonzero size");
  if (size_bytes == 0) return GPJ_OK;
  return stage_copy(ctx, static_cast<uint8_t *>(d_dst), static_cast<const uint8_t *>(h_src),
                    size_bytes, static_cast<cudaStream_t>(stream_), host_is_pinned(h_src));
}

int gpj_query_status(gpj_ctx *ctx, uint32_t *flags, void *stream_) {
  if (flags == nullptr) return fail(GPJ_ERR_INVALID_ARGUMENT, "null flags");
  int rc = bind_device(ctx);
  if (rc != GPJ_OK) return rc;
  auto stream = static_cast<cudaStream_t>(stream_);
  auto *h = reinterpret_cast<unsigned int *>(ctx->pinned + 6);
  GPJ_CUDA(cudaMemcpyAsync(h, ctx->d_status, 4, cudaMemcpyDeviceToHost, stream), "read status");
  GPJ_CUDA(cudaMemsetAsync(ctx->d_status, 0, 4, stream), "clear status");
  GPJ_CUDA(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
  *flags = *h;
  return GPJ_OK;
}

int gpj_ctx_destroy(gpj_ctx *ctx) {
  if (ctx == nullptr) return GPJ_OK;
  cudaSetDevice(ctx->device);
  cudaFree(ctx->scratch);
  cudaFree(ctx->staging);
  cudaFree(ctx->host_index);
  cudaFree(ctx->host_results);
  cudaFree(ctx->compact_scratch);
  cudaFree(ctx->d_status);
  cudaFreeHost(ctx->pinned);
  for (auto &b : ctx->index_spare) cudaFree(b.first);
  if (ctx->piece_ready) cudaEventDestroy(ctx->piece_ready);
  for (auto &e : ctx->stage_done)
    if (e) cudaEventDestroy(e);
  if (ctx->stage) cudaFreeHost(ctx->stage);
  if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
  delete ctx;
  return GPJ_OK;
}

int gpj_compile(const char *query, uint64_t wildcard_limit, uint8_t *h_ir,
                uint64_t ir_capacity, uint64_t *ir_len, uint64_t *max_depth,
                uint64_t *num_result_slots) {
  if (query == nullptr) return fail(GPJ_ERR_INVALID_ARGUMENT, "null query");
  try {
    const gpjb::CompiledIr c = gpjb::compile_query(query, wildcard_limit);
    if (ir_len) *ir_len = c.ir.size();
    if (max_depth) *max_depth = c.max_depth;
    if (num_result_slots) *num_result_slots = c.num_result_slots;
    if (c.ir.size() > ir_capacity || (h_ir == nullptr && !c.ir.empty()))
      return fail(GPJ_ERR_CAPACITY, "IR buffer too small: need " + std::to_string(c.ir.size()));
    std::memcpy(h_ir, c.ir.data(), c.ir.size());
    return GPJ_OK;
  } catch (const gpjb::CompileError &e) {
    return fail(e.code, e.message);
  } catch (const std::exception &e) {
    return fail(GPJ_ERR_IMPLEMENTATION, e.what());
  }
}

int gpj_index_build(gpj_ctx *ctx, const uint8_t *d_input, uint64_t size_bytes,
                    int num_levels, uint32_t flags, gpj_index *out, void *stream_) {
  if (out == nullptr) return fail(GPJ_ERR_INVALID_ARGUMENT, "null output");
  std::memset(out, 0, sizeof(*out));
  int rc = check_levels(num_levels);
  if (rc == GPJ_OK) rc = bind_device(ctx);
  if (rc != GPJ_OK) return rc;
  if (size_bytes > 0 && d_input == nullptr)
    return fail(GPJ_ERR_INVALID_ARGUMENT, "null input with nonzero size");
  auto stream = static_cast<cudaStream_t>(stream_);
  const bool eq = (flags & GPJ_INDEX_EMIT_ESCAPE_QUOTE) != 0;
  uint64_t cap = nl_capacity_guess(size_bytes);
  for (int attempt = 0; attempt < 2; ++attempt) {
    rc = alloc_index(ctx, out, size_bytes, num_levels, eq, cap);
    if (rc != GPJ_OK) return rc;
    out->d_input = d_input;
    out->size_bytes = size_bytes;
    rc = enqueue_index(ctx, d_input, size_bytes, num_levels, flags, *out, stream);
    uint64_t lines = 0;
    int in_string = 0, depth = -1;
    if (rc == GPJ_OK) rc = read_summary(ctx, size_bytes, stream, &lines, &in_string, &depth);
    if (rc != GPJ_OK) {
      release_index(ctx, out);
      return rc;
    }
    out->num_lines = lines;
    out->final_in_string = in_string;
    out->final_depth = depth;
    if (lines <= cap) return GPJ_OK;
    release_index(ctx, out);
    cap = lines;  // exact size, second pass
  }
  return fail(GPJ_ERR_IMPLEMENTATION, "newline capacity retry failed");
}

int gpj_index_build_async(gpj_ctx *ctx, const uint8_t *d_input, uint64_t size_bytes,
                          int num_levels, uint32_t flags, gpj_index *index,
                          uint64_t *d_summary, void *stream_) {
  if (index == nullptr) return fail(GPJ_ERR_INVALID_ARGUMENT, "null index");
  int rc = check_levels(num_levels);
  if (rc == GPJ_OK) rc = bind_device(ctx);
  if (rc != GPJ_OK) return rc;
  const uint64_t W = (size_bytes + 63u) / 64u;
  if (W > 0 && (index->d_string == nullptr || (num_levels > 0 && index->d_leveled == nullptr)))
    return fail(GPJ_ERR_INVALID_ARGUMENT, "missing output buffers");
  if ((flags & GPJ_INDEX_EMIT_ESCAPE_QUOTE) && W > 0 &&
      (index->d_escape == nullptr || index->d_quote == nullptr))
    return fail(GPJ_ERR_INVALID_ARGUMENT, "escape/quote buffers required");
  auto stream = static_cast<cudaStream_t>(stream_);
  index->d_input = d_input;
  index->size_bytes = size_bytes;
  index->num_words = W;
  index->num_levels = num_levels;
  rc = enqueue_index(ctx, d_input, size_bytes, num_levels, flags, *index, stream);
  if (rc != GPJ_OK) return rc;
  if (d_summary != nullptr) {
    GPJ_CUDA(cudaMemcpyAsync(d_summary, summary_ptr(ctx, size_bytes), 24,
                             cudaMemcpyDeviceToDevice, stream),
             "copy summary");
    GPJ_CUDA(cudaMemsetAsync(d_summary + 3, 0, 8, stream), "cudaMemsetAsync");
    if (size_bytes > 0)
      GPJ_CUDA(cudaMemcpyAsync(d_summary + 3, error_ptr(ctx, size_bytes), 4,
                               cudaMemcpyDeviceToDevice, stream),
               "copy error word");
  }
  return GPJ_OK;
}

int gpj_index_free(gpj_ctx *ctx, gpj_index *index) {
  if (index != nullptr) release_index(ctx, index);
  return GPJ_OK;
}

int gpj_query_run(gpj_ctx *ctx, const gpj_index *index, const uint8_t *h_ir,
                  uint64_t ir_len, uint32_t num_result_slots, int32_t *d_out, void *stream) {
  return run_query<int32_t>(ctx, index, h_ir, ir_len, num_result_slots, d_out,
                            static_cast<cudaStream_t>(stream));
}

int gpj_query_run64(gpj_ctx *ctx, const gpj_index *index, const uint8_t *h_ir,
                    uint64_t ir_len, uint32_t num_result_slots, int64_t *d_out, void *stream) {
  return run_query<int64_t>(ctx, index, h_ir, ir_len, num_result_slots, d_out,
                            static_cast<cudaStream_t>(stream));
}

int gpj_query_run_opts(gpj_ctx *ctx, const gpj_index *index, const uint8_t *h_ir,
                       uint64_t ir_len, uint32_t num_result_slots, const gpj_query_opts *opts,
                       void *d_out, void *stream) {
  const uint32_t base = opts ? opts->base_level : 0u;
  const uint32_t width = opts && opts->offset_bytes ? opts->offset_bytes : 4u;
  if (width == 8)
    return run_query<int64_t>(ctx, index, h_ir, ir_len, num_result_slots,
                              static_cast<int64_t *>(d_out), static_cast<cudaStream_t>(stream),
                              base);
  if (width != 4) return fail(GPJ_ERR_INVALID_ARGUMENT, "offset_bytes must be 4 or 8");
  return run_query<int32_t>(ctx, index, h_ir, ir_len, num_result_slots,
                            static_cast<int32_t *>(d_out), static_cast<cudaStream_t>(stream),
                            base);
}

int gpj_query_host(gpj_ctx *ctx, const uint8_t *h_input, uint64_t size_bytes, int num_levels,
                   uint32_t num_queries, const uint8_t *const *h_irs, const uint64_t *ir_lens,
                   const uint32_t *num_result_slots, const uint32_t *base_levels,
                   int32_t *const *h_out, const uint64_t *out_capacity, uint64_t *num_lines,
                   void *stream_) {
  int rc = check_levels(num_levels);
  if (rc == GPJ_OK) rc = bind_device(ctx);
  if (rc != GPJ_OK) return rc;
  if (size_bytes > 0 && h_input == nullptr) return fail(GPJ_ERR_INVALID_ARGUMENT, "null input");
  if (num_queries > 0 && (h_irs == nullptr || ir_lens == nullptr || num_result_slots == nullptr ||
                          h_out == nullptr || out_capacity == nullptr))
    return fail(GPJ_ERR_INVALID_ARGUMENT, "null query arrays");
  auto stream = static_cast<cudaStream_t>(stream_);
  const uint64_t n = size_bytes;
  const uint64_t W = (n + 63u) / 64u;
  // one device region: input | S | LB | NL
  const uint64_t in_bytes = round256(n);
  const uint64_t s_bytes = round256(W * 8u);
  const uint64_t lb_bytes = round256(W * 8u * uint64_t(num_levels));
  uint64_t cap = nl_capacity_guess(n);
  for (int attempt = 0; attempt < 2; ++attempt) {
    const uint64_t nl_bytes = round256(cap * 8u);
    rc = ensure(ctx->host_index, ctx->host_index_bytes, in_bytes + s_bytes + lb_bytes + nl_bytes);
    if (rc != GPJ_OK) return rc;
    auto *base = static_cast<unsigned char *>(ctx->host_index);
    gpj_index ix;
    std::memset(&ix, 0, sizeof(ix));
    auto *d_in = reinterpret_cast<uint8_t *>(base);
    ix.d_input = d_in;
    ix.size_bytes = n;
    ix.d_string = reinterpret_cast<uint64_t *>(base + in_bytes);
    ix.d_leveled = reinterpret_cast<uint64_t *>(base + in_bytes + s_bytes);
    ix.d_newline = reinterpret_cast<int64_t *>(base + in_bytes + s_bytes + lb_bytes);
    ix.newline_capacity = cap;
    ix.num_words = W;
    ix.num_levels = num_levels;
    rc = enqueue_index_from_host(ctx, h_input, d_in, n, num_levels, ix, stream);
    uint64_t lines = 0;
    int in_string = 0, depth = -1;
    if (rc == GPJ_OK) rc = read_summary(ctx, n, stream, &lines, &in_string, &depth);
    if (rc != GPJ_OK) return rc;
    if (n == 0) {
      if (num_lines) *num_lines = 0;  // the reference executes nothing for an empty partition
      return GPJ_OK;
    }
    if (num_lines) *num_lines = lines;
    if (lines > cap) {
      cap = lines;
      continue;
    }
    ix.num_lines = lines;
    // results: one device region, one slice per query
    uint64_t total = 0;
    for (uint32_t q = 0; q < num_queries; ++q) {
      const uint64_t need = lines * uint64_t(num_result_slots[q]) * 2u;
      if (need > out_capacity[q])
        return fail(GPJ_ERR_CAPACITY, "result buffer of query " + std::to_string(q) +
                                          " needs " + std::to_string(need) + " int32");
      total += round256(need * 4u);
    }
    rc = ensure(ctx->host_results, ctx->host_results_bytes, total);
    if (rc != GPJ_OK) return rc;
    GPJ_CUDA(cudaMemsetAsync(ctx->d_status, 0, 4, stream), "clear status");
    uint64_t off = 0;
    for (uint32_t q = 0; q < num_queries; ++q) {
      auto *d_out = reinterpret_cast<int32_t *>(static_cast<unsigned char *>(ctx->host_results) + off);
      rc = run_query<int32_t>(ctx, &ix, h_irs[q], ir_lens[q], num_result_slots[q], d_out, stream,
                              base_levels ? base_levels[q] : 0u);
      if (rc != GPJ_OK) return rc;
      const uint64_t need = lines * uint64_t(num_result_slots[q]) * 2u;
      if (need > 0)
        GPJ_CUDA(cudaMemcpyAsync(h_out[q], d_out, need * 4u, cudaMemcpyDeviceToHost, stream),
                 "copy results");
      off += round256(need * 4u);
    }
    auto *h_status = reinterpret_cast<unsigned int *>(ctx->pinned + 6);
    GPJ_CUDA(cudaMemcpyAsync(h_status, ctx->d_status, 4, cudaMemcpyDeviceToHost, stream),
             "read status");
    GPJ_CUDA(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
    if (*h_status & GPJ_QUERY_OVERFLOW)
      return fail(GPJ_ERR_CAPACITY,
                  "a record has more results than result slots (a \"[*]\" array longer than "
                  "the wildcard limit, or more \"..\" matches); the results are truncated");
    return GPJ_OK;
  }
  return fail(GPJ_ERR_IMPLEMENTATION, "newline capacity retry failed");
}

int gpj_results_compact(gpj_ctx *ctx, const int32_t *d_results, uint64_t num_lines,
                        uint32_t num_result_slots, const uint8_t *d_input, uint64_t size_bytes,
                        int64_t base_offset, gpj_match *d_matches, uint64_t match_capacity,
                        uint8_t *d_arena, uint64_t arena_capacity, uint64_t *d_counts,
                        void *stream_) {
  int rc = bind_device(ctx);
  if (rc != GPJ_OK) return rc;
  if (d_counts == nullptr) return fail(GPJ_ERR_INVALID_ARGUMENT, "null counts");
  const uint64_t items = num_lines * uint64_t(num_result_slots);
  if (items > 0 && d_results == nullptr) return fail(GPJ_ERR_INVALID_ARGUMENT, "null results");
  if (match_capacity > 0 && d_matches == nullptr)
    return fail(GPJ_ERR_INVALID_ARGUMENT, "null match buffer");
  if (num_result_slots > 0 && num_lines > UINT64_MAX / num_result_slots / 2u)
    return fail(GPJ_ERR_OUT_OF_RANGE, "result array too large");
  rc = ensure(ctx->compact_scratch, ctx->compact_scratch_bytes,
              gpjb::compact_scratch_bytes(num_lines, num_result_slots));
  if (rc != GPJ_OK) return rc;
  GPJ_CUDA(gpjb::compact_launch(d_results, num_lines, num_result_slots, d_input, size_bytes,
                                base_offset, d_matches, match_capacity, d_arena,
                                arena_capacity,
                                reinterpret_cast<unsigned long long *>(d_counts),
                                ctx->compact_scratch, static_cast<cudaStream_t>(stream_)),
           "result compaction launch");
  return GPJ_OK;
}

}  // extern "C"
