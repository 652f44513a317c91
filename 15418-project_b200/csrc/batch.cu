// Batched path: many files of uneven sizes indexed and queried by one launch
// chain (fused indexer over a file table -> per-file finalize -> batched
// query), captured once in a CUDA graph and replayed.  A plan is built for one
// device buffer holding every file at a 128-byte aligned offset.
//
// Creation runs the chain once to size the packed newline index and the
// result arrays exactly (the only host round trip), optionally times the
// candidate launch shapes (tile size of the indexer, block and grid of the
// query kernel) and keeps the fastest, then captures the graph.
#include "indexer.cuh"
#include "query.cuh"

#include "gpjson_b200.h"

#include <cuda_runtime.h>

#include <cstring>
#include <string>
#include <vector>

namespace gpjb {
int report_error(int code, const char *message);  // capi.cu
}

struct gpj_batch {
  int device = 0;
  const uint8_t *d_input = nullptr;
  uint64_t input_bytes = 0;
  uint32_t num_files = 0;
  uint32_t flags = 0;
  // host copies
  std::vector<gpjb::IndexFile> files;
  std::vector<uint32_t> query_of_file;
  std::vector<gpjb::BatchQueryGroup> groups;
  gpjb::IrBlob blob{};
  int max_levels = 0;
  // device state
  gpjb::IndexFile *d_files = nullptr;
  uint32_t *d_tile_file = nullptr;
  uint32_t *d_tile_row = nullptr;
  std::vector<uint64_t> host_lines;  // per-file line counts (sizing pass)
  std::vector<uint64_t> host_info;   // file info rows of the sizing pass
  uint32_t *d_query_of_file = nullptr;
  uint32_t *d_slots = nullptr;
  uint64_t *d_S = nullptr, *d_LB = nullptr;
  int64_t *d_NL = nullptr;
  int32_t *d_out = nullptr;
  uint64_t *d_info = nullptr, *d_totals = nullptr;
  void *d_scratch = nullptr;
  uint64_t s_words = 0, lb_words = 0, nl_slots = 0, result_ints = 0, records = 0;
  // launch shape
  int index_threads = gpjb::kIndexThreads;
  int query_block = 256;
  int query_grid = 0;
  CUtensorMap map{};
  bool tma = false;
  gpjb::IndexLaunch L;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t stream = nullptr;
  // gpj_batch_run_host: the input arrives in pieces on a copy stream
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t piece_ready = nullptr;
};

namespace {

int fail_cuda(cudaError_t e, const char *what) {
  (void)cudaGetLastError();
  std::string m = std::string(what) + ": " + cudaGetErrorString(e);
  return gpjb::report_error(e == cudaErrorMemoryAllocation ? GPJ_ERR_OOM : GPJ_ERR_CUDA,
                            m.c_str());
}

#define BCUDA(call, what)                          \
  do {                                             \
    const cudaError_t e_ = (call);                 \
    if (e_ != cudaSuccess) return fail_cuda(e_, what); \
  } while (0)

// Lays out the tiles, words and leveled words of every file for a tile size.
void layout(gpj_batch *b, int threads) {
  uint64_t tiles = 0, s = 0, lb = 0;
  for (uint32_t f = 0; f < b->num_files; ++f) {
    gpjb::IndexFile &F = b->files[f];
    const uint64_t W = (F.n + 63u) / 64u;
    F.first_tile = uint32_t(tiles);
    F.s_off = s;
    F.lb_off = lb;
    tiles += gpjb::tiles_for(F.n, threads);
    s += W;
    lb += W * uint64_t(F.levels);
  }
  b->s_words = s;
  b->lb_words = lb;
  b->L.num_tiles = uint32_t(tiles);
}

int bind_launch(gpj_batch *b) {
  gpjb::IndexLaunch &L = b->L;
  L.in = b->d_input;
  L.full_rows = b->input_bytes / 128u;
  L.files = b->d_files;
  L.tile_file = b->d_tile_file;
  L.tile_row = b->d_tile_row;
  L.num_files = b->num_files;
  L.num_levels = b->max_levels;
  L.S = b->d_S;
  L.LB = b->d_LB;
  L.E = nullptr;
  L.Q = nullptr;
  L.NL = b->d_NL;
  L.nl_cap = b->d_NL ? b->nl_slots : 0;
  gpjb::index_bind_scratch(L, b->d_scratch);
  b->tma = (b->flags & GPJ_INDEX_NO_TMA) == 0 &&
           gpjb::index_make_tensor_map(&b->map, b->d_input, b->input_bytes, b->index_threads);
  return GPJ_OK;
}

gpjb::BatchQueryLaunch query_launch_of(const gpj_batch *b) {
  gpjb::BatchQueryLaunch q;
  q.in = b->d_input;
  q.S = b->d_S;
  q.LB = b->d_LB;
  q.NL = b->d_NL;
  q.files = b->d_files;
  q.num_files = b->num_files;
  q.file_info = b->d_info;
  q.totals = b->d_totals;
  q.out = b->d_out;
  // overflow of extension queries lands in the error word of the totals
  // (written by the finalize kernel just before the query launch)
  q.status = reinterpret_cast<unsigned int *>(b->d_totals + gpjb::kTotError);
  q.record_counter = reinterpret_cast<unsigned long long *>(b->d_totals + gpjb::kTotRecordCounter);
  q.num_groups = int(b->groups.size());
  for (size_t g = 0; g < b->groups.size(); ++g) q.groups[g] = b->groups[g];
  return q;
}

// The whole chain on `stream`; `with_query` = false for the sizing pass.
cudaError_t enqueue(gpj_batch *b, cudaStream_t stream, bool with_query) {
  cudaError_t e = gpjb::index_launch(b->L, b->tma ? &b->map : nullptr, b->tma, stream,
                                     b->index_threads);
  if (e != cudaSuccess) return e;
  e = gpjb::index_finalize_files(b->L, b->d_query_of_file, b->d_slots, b->d_info, b->d_totals,
                                 stream);
  if (e != cudaSuccess || !with_query) return e;
  return gpjb::batch_query_launch(query_launch_of(b), b->blob, b->query_grid, b->query_block,
                                  stream);
}

void release(gpj_batch *b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->stream) cudaStreamDestroy(b->stream);
  if (b->piece_ready) cudaEventDestroy(b->piece_ready);
  if (b->copy_stream) cudaStreamDestroy(b->copy_stream);
  cudaFree(b->d_files);
  cudaFree(b->d_tile_file);
  cudaFree(b->d_tile_row);
  cudaFree(b->d_query_of_file);
  cudaFree(b->d_slots);
  cudaFree(b->d_S);
  cudaFree(b->d_LB);
  cudaFree(b->d_NL);
  cudaFree(b->d_out);
  cudaFree(b->d_info);
  cudaFree(b->d_totals);
  cudaFree(b->d_scratch);
}

int alloc_layout_buffers(gpj_batch *b) {
  cudaFree(b->d_S);
  cudaFree(b->d_LB);
  cudaFree(b->d_scratch);
  cudaFree(b->d_files);
  cudaFree(b->d_tile_file);
  cudaFree(b->d_tile_row);
  b->d_S = b->d_LB = nullptr;
  b->d_scratch = nullptr;
  b->d_files = nullptr;
  b->d_tile_file = nullptr;
  b->d_tile_row = nullptr;
  BCUDA(cudaMalloc(&b->d_S, (b->s_words + 2) * 8u), "cudaMalloc S");
  BCUDA(cudaMalloc(&b->d_LB, (b->lb_words + 2) * 8u), "cudaMalloc LB");
  BCUDA(cudaMalloc(&b->d_scratch, (uint64_t(b->L.num_tiles) * 8u + 64u + 255u) & ~uint64_t(255)),
        "cudaMalloc scratch");
  BCUDA(cudaMalloc(&b->d_files, b->files.size() * sizeof(gpjb::IndexFile)), "cudaMalloc files");
  BCUDA(cudaMemcpy(b->d_files, b->files.data(), b->files.size() * sizeof(gpjb::IndexFile),
                   cudaMemcpyHostToDevice),
        "copy file table");
  // per tile: its file, and its first 128-byte input row (bit 31: the file's
  // first tile), so the indexer can start a tile's copy after one load
  std::vector<uint32_t> tile_file(b->L.num_tiles), tile_row(b->L.num_tiles);
  for (uint32_t f = 0; f < b->num_files; ++f) {
    const uint32_t end = (f + 1 < b->num_files) ? b->files[f + 1].first_tile : b->L.num_tiles;
    const uint64_t row = b->files[f].in_off / 128u;
    for (uint32_t t = b->files[f].first_tile; t < end; ++t) {
      tile_file[t] = f;
      tile_row[t] = uint32_t(row + uint64_t(t - b->files[f].first_tile) * b->index_threads) |
                    (t == b->files[f].first_tile ? 0x80000000u : 0u);
    }
  }
  BCUDA(cudaMalloc(&b->d_tile_file, (tile_file.size() + 1) * 4u), "cudaMalloc tile map");
  BCUDA(cudaMemcpy(b->d_tile_file, tile_file.data(), tile_file.size() * 4u,
                   cudaMemcpyHostToDevice),
        "copy tile map");
  // row numbers take 31 bits (inputs below 256 GiB); beyond that the
  // indexer finds a tile's row through the file table
  if (b->input_bytes / 128u + uint64_t(b->index_threads) < 0x80000000ull) {
    BCUDA(cudaMalloc(&b->d_tile_row, (tile_row.size() + 1) * 4u), "cudaMalloc tile rows");
    BCUDA(cudaMemcpy(b->d_tile_row, tile_row.data(), tile_row.size() * 4u,
                     cudaMemcpyHostToDevice),
          "copy tile rows");
  }
  return bind_launch(b);
}

float time_chain(gpj_batch *b, cudaStream_t stream, int reps) {
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  enqueue(b, stream, true);  // warm
  cudaEventRecord(e0, stream);
  for (int i = 0; i < reps; ++i) enqueue(b, stream, true);
  cudaEventRecord(e1, stream);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return ms / float(reps);
}

}  // namespace

extern "C" {

int gpj_batch_create(gpj_ctx *ctx, const uint8_t *d_input, uint64_t input_bytes,
                     const gpj_batch_file *files, uint32_t num_files,
                     const gpj_batch_query *queries, uint32_t num_queries, uint32_t flags,
                     gpj_batch **out, void *stream_) {
  (void)ctx;
  if (out == nullptr || files == nullptr || queries == nullptr || num_files == 0)
    return gpjb::report_error(GPJ_ERR_INVALID_ARGUMENT, "gpj_batch_create: empty batch");
  *out = nullptr;
  if (num_queries == 0 || num_queries > uint32_t(gpjb::kMaxBatchGroups))
    return gpjb::report_error(GPJ_ERR_INVALID_ARGUMENT,
                              "gpj_batch_create: 1 to 8 queries per batch");
  if ((reinterpret_cast<uintptr_t>(d_input) & 15u) != 0 || d_input == nullptr)
    return gpjb::report_error(GPJ_ERR_INVALID_ARGUMENT,
                              "gpj_batch_create: the input buffer must be 16-byte aligned");
  gpj_batch *b = new gpj_batch;
  BCUDA(cudaGetDevice(&b->device), "cudaGetDevice");
  b->d_input = d_input;
  b->input_bytes = input_bytes;
  b->num_files = num_files;
  b->flags = flags;
  b->L.variant = ((flags & GPJ_BATCH_INDEX_LANE_WALK) ? gpjb::kIndexVariantLaneWalk : 0u) |
                 ((flags & GPJ_BATCH_INDEX_WIDE_LOOKBACK) ? gpjb::kIndexVariantWideLookback : 0u);
  // query groups: IR packed into one 4 KiB blob
  int ir_off = 0;
  std::vector<uint32_t> slots(num_queries);
  for (uint32_t g = 0; g < num_queries; ++g) {
    const gpj_batch_query &Qg = queries[g];
    if (Qg.h_ir == nullptr || ir_off + int(Qg.ir_len) > gpjb::kMaxQueryIrBytes ||
        Qg.num_levels > uint32_t(GPJ_MAX_LEVELS) || Qg.base_level >= Qg.num_levels) {
      delete b;
      return gpjb::report_error(GPJ_ERR_INVALID_ARGUMENT,
                                "gpj_batch_create: bad query (IR over 4 KiB in total, or "
                                "base_level >= num_levels)");
    }
    gpjb::BatchQueryGroup G;
    G.ir_off = ir_off;
    G.ir_len = int(Qg.ir_len);
    G.num_results = int(Qg.num_result_slots);
    G.base_level = int(Qg.base_level);
    std::memcpy(b->blob.bytes + ir_off, Qg.h_ir, Qg.ir_len);
    ir_off += int(Qg.ir_len);
    b->groups.push_back(G);
    slots[g] = Qg.num_result_slots;
  }
  b->files.resize(num_files);
  b->query_of_file.resize(num_files);
  for (uint32_t f = 0; f < num_files; ++f) {
    const gpj_batch_file &bf = files[f];
    if (bf.offset % 128u != 0 || bf.offset + bf.size_bytes > input_bytes ||
        bf.query >= num_queries) {
      delete b;
      return gpjb::report_error(GPJ_ERR_INVALID_ARGUMENT,
                                "gpj_batch_create: file offsets must be multiples of 128 "
                                "inside the input, with a valid query index");
    }
    b->files[f].in_off = bf.offset;
    b->files[f].n = bf.size_bytes;
    b->files[f].levels = int32_t(queries[bf.query].num_levels);
    b->query_of_file[f] = bf.query;
    if (int(queries[bf.query].num_levels) > b->max_levels)
      b->max_levels = int(queries[bf.query].num_levels);
  }
  int rc;
  auto bail = [&](int code) {
    release(b);
    delete b;
    return code;
  };
  if (cudaMalloc(&b->d_query_of_file, num_files * 4u) != cudaSuccess ||
      cudaMalloc(&b->d_slots, num_queries * 4u) != cudaSuccess ||
      cudaMalloc(&b->d_info, uint64_t(num_files) * gpjb::kFileInfoWords * 8u) != cudaSuccess ||
      cudaMalloc(&b->d_totals, 64) != cudaSuccess)
    return bail(fail_cuda(cudaErrorMemoryAllocation, "cudaMalloc batch tables"));
  cudaMemcpy(b->d_query_of_file, b->query_of_file.data(), num_files * 4u, cudaMemcpyHostToDevice);
  cudaMemcpy(b->d_slots, slots.data(), num_queries * 4u, cudaMemcpyHostToDevice);
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess)
    return bail(fail_cuda(cudaErrorUnknown, "cudaStreamCreate"));
  cudaStream_t s = b->stream;

  // sizing pass: newline slots and result ints (no newline index written)
  layout(b, b->index_threads);
  if ((rc = alloc_layout_buffers(b)) != GPJ_OK) return bail(rc);
  {
    cudaError_t e = enqueue(b, s, false);
    uint64_t totals[4] = {0, 0, 0, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(totals, b->d_totals, 32, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return bail(fail_cuda(e, "batch sizing pass"));
    if (totals[gpjb::kTotError] != 0)
      return bail(gpjb::report_error(GPJ_ERR_TIMEOUT, "batch sizing pass: bounded wait gave up"));
    b->records = totals[gpjb::kTotRecords];
    b->result_ints = totals[gpjb::kTotResultInts];
    b->nl_slots = totals[gpjb::kTotNlSlots];
    std::vector<uint64_t> info(uint64_t(num_files) * gpjb::kFileInfoWords);
    if (cudaMemcpy(info.data(), b->d_info, info.size() * 8u, cudaMemcpyDeviceToHost) != cudaSuccess)
      return bail(fail_cuda(cudaErrorUnknown, "read file info"));
    b->host_lines.resize(num_files);
    b->host_info = info;
  }
  if (cudaMalloc(&b->d_NL, (b->nl_slots + 1) * 8u) != cudaSuccess ||
      cudaMalloc(&b->d_out, (b->result_ints + 1) * 4u) != cudaSuccess)
    return bail(fail_cuda(cudaErrorMemoryAllocation, "cudaMalloc batch outputs"));
  if ((rc = bind_launch(b)) != GPJ_OK) return bail(rc);
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
  b->query_grid = sms * 8;

  if (flags & GPJ_BATCH_AUTOTUNE) {
    // Two stages, each candidate timed over a few runs of the whole chain.
    // First the indexer: tile size (128 or 256 threads x 128 B) and kernel
    // variant (listed or per-lane leveled walk, look-back rounds of 32 or
    // 64 descriptors), with the default query shape.  Then the query block
    // and persistent grid for that indexer.
    float best = 1e30f;
    int best_t = b->index_threads;
    uint32_t best_v = b->L.variant;
    for (int threads : {256, 128}) {
      layout(b, threads);
      b->index_threads = threads;
      if ((rc = alloc_layout_buffers(b)) != GPJ_OK) return bail(rc);
      const uint32_t variants[] = {0u, uint32_t(gpjb::kIndexVariantLaneWalk),
                                   uint32_t(gpjb::kIndexVariantWideLookback),
                                   uint32_t(gpjb::kIndexVariantLaneWalk) |
                                       uint32_t(gpjb::kIndexVariantWideLookback)};
      for (uint32_t variant : variants) {
        b->L.variant = variant;
        const float ms = time_chain(b, s, 3);
        if (ms < best) {
          best = ms;
          best_t = threads;
          best_v = variant;
        }
      }
    }
    if (best_t != b->index_threads) {
      layout(b, best_t);
      b->index_threads = best_t;
      if ((rc = alloc_layout_buffers(b)) != GPJ_OK) return bail(rc);
    }
    b->L.variant = best_v;
    best = 1e30f;
    int best_b = b->query_block, best_g = b->query_grid;
    for (int block : {128, 256}) {
      for (int gm : {4, 5, 8, 16}) {
        b->query_block = block;
        b->query_grid = sms * gm * (256 / block);
        const float ms = time_chain(b, s, 3);
        if (ms < best) {
          best = ms;
          best_b = block;
          best_g = b->query_grid;
        }
      }
    }
    b->query_block = best_b;
    b->query_grid = best_g;
  }

  if ((flags & GPJ_BATCH_NO_GRAPH) == 0) {
    cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      const cudaError_t le = enqueue(b, s, true);
      e = cudaStreamEndCapture(s, &b->graph);
      if (le != cudaSuccess) e = le;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, b->graph, 0);
    if (e != cudaSuccess) return bail(fail_cuda(e, "batch graph capture"));
  }
  const cudaError_t se = cudaStreamSynchronize(s);
  if (se != cudaSuccess) return bail(fail_cuda(se, "batch create"));
  (void)stream_;
  *out = b;
  return GPJ_OK;
}

int gpj_batch_run(gpj_batch *b, void *stream_) {
  if (b == nullptr) return gpjb::report_error(GPJ_ERR_INVALID_ARGUMENT, "null batch");
  auto stream = static_cast<cudaStream_t>(stream_);
  BCUDA(cudaSetDevice(b->device), "cudaSetDevice");
  if (b->exec != nullptr) {
    BCUDA(cudaGraphLaunch(b->exec, stream), "cudaGraphLaunch");
  } else {
    BCUDA(enqueue(b, stream, true), "batch launch");
  }
  return GPJ_OK;
}

int gpj_batch_run_stages(gpj_batch *b, uint32_t stages, void *stream_) {
  if (b == nullptr) return gpjb::report_error(GPJ_ERR_INVALID_ARGUMENT, "null batch");
  auto stream = static_cast<cudaStream_t>(stream_);
  BCUDA(cudaSetDevice(b->device), "cudaSetDevice");
  if (stages & GPJ_BATCH_STAGE_INDEX)
    BCUDA(gpjb::index_launch(b->L, b->tma ? &b->map : nullptr, b->tma, stream, b->index_threads),
          "batch index launch");
  if (stages & GPJ_BATCH_STAGE_FINALIZE)
    BCUDA(gpjb::index_finalize_files(b->L, b->d_query_of_file, b->d_slots, b->d_info,
                                     b->d_totals, stream),
          "batch finalize launch");
  if (stages & GPJ_BATCH_STAGE_QUERY)
    BCUDA(gpjb::batch_query_launch(query_launch_of(b), b->blob, b->query_grid, b->query_block,
                                   stream),
          "batch query launch");
  return GPJ_OK;
}

int gpj_batch_run_per_file(gpj_batch *b, void *stream_) {
  if (b == nullptr) return gpjb::report_error(GPJ_ERR_INVALID_ARGUMENT, "null batch");
  auto stream = static_cast<cudaStream_t>(stream_);
  BCUDA(cudaSetDevice(b->device), "cudaSetDevice");
  // one single-file launch chain per file (the per-partition loop of a
  // plain caller), writing the same outputs at the same places
  for (uint32_t f = 0; f < b->num_files; ++f) {
    const gpjb::IndexFile &F = b->files[f];
    const uint64_t *row = b->host_info.data() + uint64_t(f) * gpjb::kFileInfoWords;
    const gpjb::BatchQueryGroup &G = b->groups[b->query_of_file[f]];
    gpjb::IndexLaunch L;
    L.in = b->d_input + F.in_off;
    L.single.n = F.n;
    L.single.levels = F.levels;
    L.num_levels = F.levels;
    L.full_rows = F.n / 128u;
    L.S = b->d_S + F.s_off;
    L.LB = b->d_LB + F.lb_off;
    L.NL = b->d_NL + row[gpjb::kFiNlOff];
    L.nl_cap = row[gpjb::kFiLines];
    L.num_tiles = uint32_t(gpjb::index_num_tiles(F.n));
    gpjb::index_bind_scratch(L, b->d_scratch);
    if (F.n == 0) {  // one empty record: NL = [0], every slot -1
      BCUDA(cudaMemsetAsync(L.NL, 0, 8, stream), "cudaMemsetAsync");
      BCUDA(cudaMemsetAsync(b->d_out + row[gpjb::kFiOutOff], 0xFF,
                            size_t(G.num_results) * 8u, stream),
            "cudaMemsetAsync");
      continue;
    }
    CUtensorMap map;
    const bool tma = (b->flags & GPJ_INDEX_NO_TMA) == 0 &&
                     gpjb::index_make_tensor_map(&map, L.in, F.n);
    BCUDA(gpjb::index_launch(L, tma ? &map : nullptr, tma, stream), "per-file index launch");
    gpjb::QueryLaunch q;
    q.in = L.in;
    q.n = int64_t(F.n);
    q.NL = L.NL;
    q.num_lines = int64_t(row[gpjb::kFiLines]);
    q.S = L.S;
    q.LB = L.LB;
    q.W = int64_t((F.n + 63u) / 64u);
    q.ir_len = G.ir_len;
    q.num_results = G.num_results;
    q.num_levels = F.levels;
    q.base_level = G.base_level;
    q.out32 = b->d_out + row[gpjb::kFiOutOff];
    q.status = reinterpret_cast<unsigned int *>(b->d_totals + gpjb::kTotError);
    gpjb::IrBlob blob;
    std::memcpy(blob.bytes, b->blob.bytes + G.ir_off, size_t(G.ir_len));
    BCUDA(gpjb::query_launch(q, blob, 0, 256, stream), "per-file query launch");
  }
  return GPJ_OK;
}

namespace {

// Host input of a batch: copied in pieces of whole files of about this many
// bytes; the tiles of each piece are indexed as soon as it is on the device,
// so indexing overlaps the copy of the next piece.  Finalize and queries run
// once every piece is indexed.
constexpr uint64_t kPieceBytes = uint64_t(32) << 20;

// Pieces are byte ranges between file starts: the files must lie in table
// order without overlapping (as gpjson_b200.pack_files lays them out).
bool files_in_order(const gpj_batch *b) {
  for (uint32_t f = 0; f + 1 < b->num_files; ++f)
    if (b->files[f].in_off + b->files[f].n > b->files[f + 1].in_off) return false;
  return true;
}

int run_in_pieces(gpj_batch *b, const uint8_t *h_input, cudaStream_t stream) {
  if (b->copy_stream == nullptr)
    BCUDA(cudaStreamCreateWithFlags(&b->copy_stream, cudaStreamNonBlocking), "cudaStreamCreate");
  if (b->piece_ready == nullptr)
    BCUDA(cudaEventCreateWithFlags(&b->piece_ready, cudaEventDisableTiming), "cudaEventCreate");
  auto *d_in = const_cast<uint8_t *>(b->d_input);
  const CUtensorMap *map = b->tma ? &b->map : nullptr;
  BCUDA(gpjb::index_clear_scratch(b->L, stream), "cudaMemsetAsync");
  // the copies start after the work already queued on `stream`
  BCUDA(cudaEventRecord(b->piece_ready, stream), "cudaEventRecord");
  BCUDA(cudaStreamWaitEvent(b->copy_stream, b->piece_ready, 0), "cudaStreamWaitEvent");
  uint32_t f = 0;
  while (f < b->num_files) {
    // files [f, g): at least one, then more while the piece stays small
    const uint64_t start = f == 0 ? 0u : b->files[f].in_off;
    uint32_t g = f + 1;
    while (g < b->num_files && b->files[g].in_off + b->files[g].n - start <= kPieceBytes) ++g;
    const uint64_t end = g < b->num_files ? b->files[g].in_off : b->input_bytes;
    const uint32_t t0 = b->files[f].first_tile;
    const uint32_t t1 = g < b->num_files ? b->files[g].first_tile : b->L.num_tiles;
    if (end > start)
      BCUDA(cudaMemcpyAsync(d_in + start, h_input + start, end - start, cudaMemcpyHostToDevice,
                            b->copy_stream),
            "copy batch input piece");
    BCUDA(cudaEventRecord(b->piece_ready, b->copy_stream), "cudaEventRecord");
    BCUDA(cudaStreamWaitEvent(stream, b->piece_ready, 0), "cudaStreamWaitEvent");
    if (t1 > t0) {
      BCUDA(gpjb::index_clear_counter(b->L, stream), "cudaMemsetAsync");
      BCUDA(gpjb::index_launch_range(b->L, map, b->tma, stream, t0, t1, b->index_threads),
            "index kernel launch");
    }
    f = g;
  }
  BCUDA(gpjb::index_finalize_files(b->L, b->d_query_of_file, b->d_slots, b->d_info,
                                   b->d_totals, stream),
        "finalize launch");
  BCUDA(gpjb::batch_query_launch(query_launch_of(b), b->blob, b->query_grid, b->query_block,
                                 stream),
        "batch query launch");
  return GPJ_OK;
}

}  // namespace

int gpj_batch_run_host(gpj_batch *b, const uint8_t *h_input, int32_t *h_results,
                       uint64_t *h_file_info, void *stream_) {
  if (b == nullptr || h_input == nullptr)
    return gpjb::report_error(GPJ_ERR_INVALID_ARGUMENT, "null batch or input");
  auto stream = static_cast<cudaStream_t>(stream_);
  BCUDA(cudaSetDevice(b->device), "cudaSetDevice");
  if (b->input_bytes <= kPieceBytes || b->L.num_tiles == 0 || !files_in_order(b)) {
    BCUDA(cudaMemcpyAsync(const_cast<uint8_t *>(b->d_input), h_input, b->input_bytes,
                          cudaMemcpyHostToDevice, stream),
          "copy batch input");
    const int rc = gpj_batch_run(b, stream_);
    if (rc != GPJ_OK) return rc;
  } else {
    const int rc = run_in_pieces(b, h_input, stream);
    if (rc != GPJ_OK) return rc;
  }
  if (h_results != nullptr && b->result_ints > 0)
    BCUDA(cudaMemcpyAsync(h_results, b->d_out, b->result_ints * 4u, cudaMemcpyDeviceToHost,
                          stream),
          "copy batch results");
  if (h_file_info != nullptr)
    BCUDA(cudaMemcpyAsync(h_file_info, b->d_info, uint64_t(b->num_files) * 64u,
                          cudaMemcpyDeviceToHost, stream),
          "copy batch file info");
  uint64_t err = 0;
  BCUDA(cudaMemcpyAsync(&err, b->d_totals + gpjb::kTotError, 8, cudaMemcpyDeviceToHost, stream),
        "copy batch error word");
  BCUDA(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
  if (err & (gpjb::kErrLookbackTimeout | gpjb::kErrTmaTimeout | gpjb::kErrPipelineTimeout))
    return gpjb::report_error(GPJ_ERR_TIMEOUT, "batch index: a bounded device wait gave up");
  if (err & gpjb::kQueryStatusOverflow)
    return gpjb::report_error(GPJ_ERR_CAPACITY,
                              "batch query: a record has more results than result slots; the "
                              "results are truncated");
  return GPJ_OK;
}

int gpj_batch_view_get(const gpj_batch *b, gpj_batch_view *v) {
  if (b == nullptr || v == nullptr)
    return gpjb::report_error(GPJ_ERR_INVALID_ARGUMENT, "null batch");
  std::memset(v, 0, sizeof(*v));
  v->d_string = b->d_S;
  v->d_leveled = b->d_LB;
  v->d_newline = b->d_NL;
  v->d_results = b->d_out;
  v->d_file_info = b->d_info;
  v->d_totals = b->d_totals;
  v->num_files = b->num_files;
  v->num_records = b->records;
  v->result_ints = b->result_ints;
  v->newline_slots = b->nl_slots;
  v->string_words = b->s_words;
  v->leveled_words = b->lb_words;
  v->num_tiles = b->L.num_tiles;
  v->index_threads = uint32_t(b->index_threads);
  v->query_block = uint32_t(b->query_block);
  v->query_grid = uint32_t(b->query_grid);
  v->uses_graph = b->exec != nullptr ? 1u : 0u;
  v->index_variant = b->L.variant;
  return GPJ_OK;
}

int gpj_batch_file_layout(const gpj_batch *b, uint32_t file, uint64_t *string_off,
                          uint64_t *leveled_off, uint32_t *num_levels) {
  if (b == nullptr || file >= b->num_files)
    return gpjb::report_error(GPJ_ERR_INVALID_ARGUMENT, "bad batch or file index");
  if (string_off) *string_off = b->files[file].s_off;
  if (leveled_off) *leveled_off = b->files[file].lb_off;
  if (num_levels) *num_levels = uint32_t(b->files[file].levels);
  return GPJ_OK;
}

int gpj_batch_destroy(gpj_batch *b) {
  if (b == nullptr) return GPJ_OK;
  cudaSetDevice(b->device);
  release(b);
  delete b;
  return GPJ_OK;
}

}  // extern "C"
