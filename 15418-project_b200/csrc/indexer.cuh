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

// Everything one launch of the indexer reads and writes.  Device pointers.
struct IndexLaunch {
  const uint8_t *in = nullptr;  // partition bytes
  uint64_t n = 0;               // partition size
  uint64_t W = 0;               // ceil(n / 64)
  int num_levels = 0;           // L, 0..kMaxLevels
  uint64_t full_rows = 0;       // n / 128: rows the TMA descriptor covers
  uint64_t *S = nullptr;        // [W]   string mask
  uint64_t *LB = nullptr;       // [L*W] leveled bitmaps, level-major
  uint64_t *E = nullptr;        // [W]   escape bitmap (verify mode) or null
  uint64_t *Q = nullptr;        // [W]   quote bitmap (verify mode) or null
  int64_t *NL = nullptr;        // newline index, nl_cap entries
  uint64_t nl_cap = 0;
  // scratch: one 64-bit look-back descriptor per tile, a tile ticket counter,
  // an error word and a 4-word summary
  unsigned long long *tile_state = nullptr;
  unsigned int *tile_counter = nullptr;
  unsigned int *error = nullptr;
  unsigned long long *summary = nullptr;  // [0] lines [1] in-string [2] depth
  uint32_t num_tiles = 0;
};

// Error bits the kernels raise in IndexLaunch::error.
enum : unsigned int {
  kErrLookbackTimeout = 1u,
  kErrTmaTimeout = 2u,
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
// swizzle).  Returns false when the TMA path cannot be used (n < 128 or the
// pointer is not 16-byte aligned); the launcher then uses plain loads.
bool index_make_tensor_map(CUtensorMap *map, const uint8_t *in, uint64_t n);

// Zeroes the scratch and launches the indexer on `stream`.  No host sync.
cudaError_t index_launch(const IndexLaunch &L, const CUtensorMap *map,
                         bool use_tma, cudaStream_t stream);

}  // namespace gpjb
