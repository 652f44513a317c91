// Device-side materialisation of query results: the int32 result array
// [lines][slots][2] of one query (partition-local offsets, -1 = no match)
// becomes a dense list of matches in (line, slot) order with global offsets,
// and the bytes of each match are gathered into one contiguous arena.  The
// reference does this on the host for every line and slot, building one
// std::string per match from the host copy of the partition
// (src/gpjson/query/kernels/orig/query_executor_host.cu:80-119); here only
// the matches and their bytes cross PCIe.
//
// Three launches, deterministic order: per-block counts of matches and
// bytes, one block scanning those counts, then every block writing its
// matches at its scanned offsets.
#include "compact.cuh"

namespace gpjb {
namespace {

constexpr int kThreads = 256;
constexpr int kItemsPerThread = 4;
constexpr uint64_t kItemsPerBlock = uint64_t(kThreads) * kItemsPerThread;

struct Item {
  uint64_t match;  // 1 when the (start, end) pair is a valid match
  uint64_t bytes;  // end - start of a valid match
};

// One (line, slot) pair: -1 on either side is "no match", as in the
// reference; a pair with start > end or end beyond the partition is an
// invalid range (the reference raises an execution error for it).
__device__ __forceinline__ Item classify(const int32_t *res, uint64_t i, uint64_t n,
                                         unsigned long long *invalid) {
  const int32_t a = res[2 * i], b = res[2 * i + 1];
  if (a < 0 || b < 0) return {0, 0};
  if (a > b || uint64_t(b) > n) {
    atomicAdd(invalid, 1ull);
    return {0, 0};
  }
  return {1, uint64_t(b - a)};
}

// Block-wide exclusive scan of two 64-bit counters; returns the totals.
__device__ __forceinline__ void block_scan2(uint64_t &m, uint64_t &b, uint64_t &tm, uint64_t &tb) {
  __shared__ unsigned long long s_m[kThreads / 32], s_b[kThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint64_t im = m, ib = b;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const uint64_t xm = __shfl_up_sync(0xFFFFFFFFu, im, off);
    const uint64_t xb = __shfl_up_sync(0xFFFFFFFFu, ib, off);
    if (lane >= off) {
      im += xm;
      ib += xb;
    }
  }
  if (lane == 31) {
    s_m[warp] = im;
    s_b[warp] = ib;
  }
  __syncthreads();
  uint64_t wm = 0, wb = 0;
  tm = 0;
  tb = 0;
#pragma unroll
  for (int w = 0; w < kThreads / 32; ++w) {
    if (w < warp) {
      wm += s_m[w];
      wb += s_b[w];
    }
    tm += s_m[w];
    tb += s_b[w];
  }
  m = wm + im - m;
  b = wb + ib - b;
  __syncthreads();
}

__global__ void __launch_bounds__(kThreads)
    count_kernel(const int32_t *res, uint64_t items, uint64_t n, unsigned long long *block_counts,
                 unsigned long long *counts) {
  const uint64_t first = uint64_t(blockIdx.x) * kItemsPerBlock + uint64_t(threadIdx.x) * kItemsPerThread;
  uint64_t m = 0, b = 0;
#pragma unroll
  for (int k = 0; k < kItemsPerThread; ++k) {
    if (first + k < items) {
      const Item it = classify(res, first + k, n, &counts[2]);
      m += it.match;
      b += it.bytes;
    }
  }
  uint64_t tm, tb;
  block_scan2(m, b, tm, tb);
  if (threadIdx.x == 0) {
    block_counts[2 * blockIdx.x] = tm;
    block_counts[2 * blockIdx.x + 1] = tb;
  }
}

// One block: exclusive scan of the per-block counts in place, totals into
// counts[0] (matches) and counts[1] (arena bytes).
__global__ void __launch_bounds__(kThreads)
    scan_kernel(unsigned long long *block_counts, uint64_t blocks, unsigned long long *counts) {
  uint64_t carry_m = 0, carry_b = 0;
  for (uint64_t base = 0; base < blocks; base += kThreads) {
    const uint64_t i = base + threadIdx.x;
    uint64_t m = i < blocks ? block_counts[2 * i] : 0, b = i < blocks ? block_counts[2 * i + 1] : 0;
    uint64_t tm, tb;
    block_scan2(m, b, tm, tb);
    if (i < blocks) {
      block_counts[2 * i] = carry_m + m;
      block_counts[2 * i + 1] = carry_b + b;
    }
    carry_m += tm;
    carry_b += tb;
  }
  if (threadIdx.x == 0) {
    counts[0] = carry_m;
    counts[1] = carry_b;
  }
}

__global__ void __launch_bounds__(kThreads)
    write_kernel(const int32_t *res, uint64_t items, uint32_t slots, const uint8_t *in, uint64_t n,
                 int64_t base_offset, const unsigned long long *block_counts, gpj_match *matches,
                 uint64_t match_cap, uint8_t *arena, uint64_t arena_cap) {
  const uint64_t first = uint64_t(blockIdx.x) * kItemsPerBlock + uint64_t(threadIdx.x) * kItemsPerThread;
  Item its[kItemsPerThread];
  uint64_t m = 0, b = 0;
#pragma unroll
  for (int k = 0; k < kItemsPerThread; ++k) {
    its[k] = {0, 0};
    if (first + k < items) {
      const int32_t s = res[2 * (first + k)], e = res[2 * (first + k) + 1];
      if (s >= 0 && e >= 0 && s <= e && uint64_t(e) <= n) its[k] = {1, uint64_t(e - s)};
    }
    m += its[k].match;
    b += its[k].bytes;
  }
  uint64_t tm, tb;
  block_scan2(m, b, tm, tb);
  m += block_counts[2 * blockIdx.x];
  b += block_counts[2 * blockIdx.x + 1];
#pragma unroll
  for (int k = 0; k < kItemsPerThread; ++k) {
    if (!its[k].match) continue;
    const uint64_t i = first + k;
    const int32_t s = res[2 * i];
    const uint64_t len = its[k].bytes;
    if (m < match_cap) {
      gpj_match g;
      g.line = i / slots;
      g.slot = uint32_t(i % slots);
      g.length = uint32_t(len);
      g.start = base_offset + int64_t(s);
      g.end = base_offset + int64_t(s) + int64_t(len);
      g.text_offset = b;
      matches[m] = g;
    }
    if (arena != nullptr && in != nullptr && b + len <= arena_cap) {
      for (uint64_t j = 0; j < len; ++j) arena[b + j] = in[uint64_t(s) + j];
    }
    ++m;
    b += len;
  }
}

}  // namespace

uint64_t compact_scratch_bytes(uint64_t lines, uint32_t slots) {
  const uint64_t items = lines * uint64_t(slots);
  const uint64_t blocks = (items + kItemsPerBlock - 1) / kItemsPerBlock;
  return blocks * 16u + 256u;
}

cudaError_t compact_launch(const int32_t *d_results, uint64_t lines, uint32_t slots,
                           const uint8_t *d_input, uint64_t n, int64_t base_offset,
                           gpj_match *d_matches, uint64_t match_cap, uint8_t *d_arena,
                           uint64_t arena_cap, unsigned long long *d_counts, void *scratch,
                           cudaStream_t stream) {
  cudaError_t e = cudaMemsetAsync(d_counts, 0, 3 * sizeof(unsigned long long), stream);
  if (e != cudaSuccess) return e;
  const uint64_t items = lines * uint64_t(slots);
  if (items == 0) return cudaSuccess;
  const uint64_t blocks = (items + kItemsPerBlock - 1) / kItemsPerBlock;
  if (blocks > 0x7FFFFFFFull) return cudaErrorInvalidValue;
  auto *bc = static_cast<unsigned long long *>(scratch);
  count_kernel<<<uint32_t(blocks), kThreads, 0, stream>>>(d_results, items, n, bc, d_counts);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  scan_kernel<<<1, kThreads, 0, stream>>>(bc, blocks, d_counts);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  write_kernel<<<uint32_t(blocks), kThreads, 0, stream>>>(d_results, items, slots, d_input, n,
                                                          base_offset, bc, d_matches, match_cap,
                                                          d_arena, arena_cap);
  return cudaGetLastError();
}

}  // namespace gpjb
