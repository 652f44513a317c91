// Host-side interface of the fused structural indexer (internal to the
// library; the public surface is the C ABI in include/gpjson_b200.h).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>

namespace gpjb {

constexpr int kIndexThreads = 256;
constexpr int kIndexWordsPerThread = 2;
constexpr int kTileWords = kIndexThreads * kIndexWordsPerThread;  // 512
constexpr uint64_t kTileBytes = uint64_t(kTileWords) * 64u;       // 32 KiB
constexpr int kTileRows = int(kTileBytes / 128u);                 // 256 rows of 128 B
constexpr int kMaxLevels = 22;  // kMaxNumLevels, sharemem/leveled-bitmaps-index.cu

// One file (partition) of an indexed buffer.  Offsets are relative to the
// IndexLaunch pointers.  Tiles never cross files; string state and depth
// restart at each file, newline counting runs on across files so that every
// file's newline index lands in one packed array.
struct IndexFile {
  uint64_t in_off = 0;     // byte offset in `in` (a multiple of 128 when TMA loads it)
  uint64_t n = 0;          // bytes
  uint64_t s_off = 0;      // first word of its S (and E, Q) words
  uint64_t lb_off = 0;     // first word of its L * W leveled words (level-major)
  uint32_t first_tile = 0; // index of its first tile
  int32_t levels = 0;      // L of this file
};

// Everything one launch of the indexer reads and writes.  Device pointers.
struct IndexLaunch {
  const uint8_t *in = nullptr;  // input bytes
  uint64_t full_rows = 0;       // whole 128-byte rows of `in` the TMA descriptor covers
  IndexFile single;             // the file when `files` is null (one partition)
  const IndexFile *files = nullptr;  // device table, num_files entries, or null
  const uint32_t *tile_file = nullptr;  // file of each tile (optional; else binary search)
  const uint32_t *tile_row = nullptr;   // with tile_file: first 128-byte input row of each
                                        // tile, bit 31 set on a file's first tile (optional)
  uint32_t num_files = 1;
  int num_levels = 0;           // max L over the files (selects the kernel)
  uint64_t *S = nullptr;        // string mask words
  uint64_t *LB = nullptr;       // leveled bitmaps
  uint64_t *E = nullptr;        // escape bitmap words (verify mode) or null
  uint64_t *Q = nullptr;        // quote bitmap words (verify mode) or null
  int64_t *NL = nullptr;        // newline indexes of all files, packed: file f
                                // starts at (newlines before f) + f
  uint64_t nl_cap = 0;
  // scratch: one 64-bit look-back descriptor per tile, a tile ticket counter,
  // an error word and a 4-word summary (one-file launches)
  unsigned long long *tile_state = nullptr;
  unsigned int *tile_counter = nullptr;
  unsigned int *error = nullptr;
  unsigned long long *summary = nullptr;  // [0] lines [1] in-string [2] depth
  uint32_t num_tiles = 0;
  // tiles this launch claims: [tile_begin, tile_end); set by the launchers
  uint32_t tile_begin = 0, tile_end = 0;
  // polls after which a look-back gives up on an unpublished predecessor
  uint32_t lookback_spin_limit = 1u << 22;
  // kernel variant (kIndexVariant* bits; 0 = default), chosen by the batch
  // autotuner; the outputs are the same for every variant
  uint32_t variant = 0;
};

// Index kernel variants for indexes of up to four levels.
enum : uint32_t {
  kIndexVariantLaneWalk = 1u,      // every lane walks its own quarters (no list)
  kIndexVariantWideLookback = 2u,  // look-back rounds of 64 descriptors instead of 32
};

// Error bits the kernels raise in IndexLaunch::error.
enum : unsigned int {
  kErrLookbackTimeout = 1u,
  kErrTmaTimeout = 2u,
  kErrPipelineTimeout = 4u,  // a wait between the control and compute warps
};

inline uint64_t index_num_tiles(uint64_t n) {
  return (n + kTileBytes - 1) / kTileBytes;
}

// Bytes of scratch the indexer needs for n input bytes: descriptors + 64 B of
// counters/summary, rounded to 256 B.
inline uint64_t index_scratch_bytes(uint64_t n) {
  const uint64_t tiles = index_num_tiles(n);
  return ((tiles * 8u + 64u) + 255u) & ~uint64_t(255);
}

// Lays the scratch fields of `L` over a caller-provided region of
// index_scratch_bytes(n) bytes (256-byte aligned).
void index_bind_scratch(IndexLaunch &L, void *scratch);

// Encodes the TMA descriptor for `in` (2-D view: rows of 128 B, 128-byte
// swizzle, boxes of `threads` rows = one tile).  Returns false when the TMA
// path cannot be used (n < 128 or the pointer is not 16-byte aligned); the
// launcher then uses plain loads.
bool index_make_tensor_map(CUtensorMap *map, const uint8_t *in, uint64_t n,
                           int threads = kIndexThreads);

// Zeroes the scratch and launches the indexer on `stream` with `threads`
// (128 or 256) threads per CTA: tiles of threads * 128 bytes, so num_tiles
// and the files' first tiles must be counted with that tile size.
cudaError_t index_launch(const IndexLaunch &L, const CUtensorMap *map,
                         bool use_tma, cudaStream_t stream,
                         int threads = kIndexThreads);

// Launches the indexer for tiles [t0, t1) only, without touching the
// scratch: the look-back descriptors of the tiles before t0 must already be
// final (an earlier launch on the same stream), the ticket counter zero and
// the rest of the descriptors clear (index_clear_scratch).  A file read in
// pieces is indexed by one launch per piece as the pieces arrive.
cudaError_t index_launch_range(const IndexLaunch &L, const CUtensorMap *map, bool use_tma,
                               cudaStream_t stream, uint32_t t0, uint32_t t1,
                               int threads = kIndexThreads);
cudaError_t index_clear_scratch(const IndexLaunch &L, cudaStream_t stream);
cudaError_t index_clear_counter(const IndexLaunch &L, cudaStream_t stream);

inline uint64_t tiles_for(uint64_t n, int threads) {
  const uint64_t tb = uint64_t(threads) * 128u;
  return (n + tb - 1) / tb;
}

}  // namespace gpjb

namespace gpjb {

// Per-file results of a multi-file index build (one row of 8 words per file).
enum FileInfoField : int {
  kFiLines = 0,     // newline count + 1
  kFiNlOff = 1,     // first slot of its newline index in the packed array
  kFiRecOff = 2,    // first record of the file in the batch record numbering
  kFiOutOff = 3,    // first int of its result block
  kFiInString = 4,  // string state after its last byte
  kFiDepth = 5,     // signed-char depth after its last byte (as int64)
  kFiBytes = 6,     // file size
  kFiQuery = 7,     // query group
  kFileInfoWords = 8,
};

// Totals of a multi-file build: [records, result ints, newline slots, error].
enum TotalField : int {
  kTotRecords = 0,
  kTotResultInts = 1,
  kTotNlSlots = 2,
  kTotError = 3,
  kTotRecordCounter = 4,  // the batch query's record counter (not a total)
};

// After index_launch on a file table: derives every file's line count,
// newline-index slot, record and result offsets (exclusive scans over the
// files) from the tiles' inclusive look-back descriptors, writes the leading
// 0 of each empty file's newline index, and the totals.  One CTA.
cudaError_t index_finalize_files(const IndexLaunch &L, const uint32_t *query_of_file,
                                 const uint32_t *slots_of_query, uint64_t *file_info,
                                 uint64_t *totals, cudaStream_t stream);

}  // namespace gpjb
