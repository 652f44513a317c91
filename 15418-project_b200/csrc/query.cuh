// Host-side interface of the JSONPath query kernels (internal).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "indexer.cuh"

namespace gpjb {

constexpr int kMaxQueryLevels = 16;   // orig.hpp:10 kMaxQueryLevels
constexpr int kMaxQueryIrBytes = 4096;  // orig.hpp:11 kMaxQueryIrBytes

// Status bit a query raises when a record had more results than its slots:
// a "[*]" array or open slice longer than the wildcard limit, or more
// "..name" matches.
// Only IR with extension opcodes can raise it.  Kept clear of the indexer's
// error bits (1, 2, 4), with which it shares the batch's error word.
constexpr unsigned int kQueryStatusOverflow = 0x100u;

// One query over every record of one partition.
struct QueryLaunch {
  const uint8_t *in = nullptr;   // partition bytes
  int64_t n = 0;
  const int64_t *NL = nullptr;   // newline index
  int64_t num_lines = 0;
  const uint64_t *S = nullptr;   // string mask [W]
  const uint64_t *LB = nullptr;  // leveled bitmaps [L*W]
  int64_t W = 0;
  int ir_len = 0;
  int num_results = 0;           // result slots per record
  int num_levels = 0;            // levels present in LB; deeper reads see 0
  int base_level = 0;            // bitmap level of query level 0 (1: elements
                                 // of a top-level array are the records)
  int32_t *out32 = nullptr;      // [num_lines][num_results][2], or
  int64_t *out64 = nullptr;      // the same with 64-bit offsets
  unsigned int *status = nullptr;  // kQueryStatusOverflow is OR-ed here (optional)
};

// The IR travels in the kernel parameters (4 KiB, copied into shared memory
// by every CTA), so concurrent launches never share an IR buffer.
struct IrBlob {
  uint8_t bytes[kMaxQueryIrBytes];
};

cudaError_t query_launch(const QueryLaunch &q, const IrBlob &ir, int grid,
                         int block, cudaStream_t stream);

// True when the IR holds extension opcodes (numeric filters, "..name", the
// element checks of "[*]" and the open slices): those launch the
// interpreter variant that has them.
bool query_ir_uses_extensions(const uint8_t *ir, int len);

// Batched query over every record of every file of a multi-file index build:
// record r belongs to the file whose record range holds it (file_info from
// index_finalize_files); the file's query group selects the IR (packed in the
// IrBlob), slot count and record level.  The record count is read on the
// device, so the launch needs no host round trip.
constexpr int kMaxBatchGroups = 8;
struct BatchQueryGroup {
  int ir_off = 0;
  int ir_len = 0;
  int num_results = 0;
  int base_level = 0;
};
struct BatchQueryLaunch {
  const uint8_t *in = nullptr;
  const uint64_t *S = nullptr;
  const uint64_t *LB = nullptr;
  const int64_t *NL = nullptr;
  const IndexFile *files = nullptr;
  uint32_t num_files = 0;
  const uint64_t *file_info = nullptr;  // kFileInfoWords per file
  const uint64_t *totals = nullptr;
  int32_t *out = nullptr;
  unsigned int *status = nullptr;  // kQueryStatusOverflow is OR-ed here (optional)
  unsigned int *file_status = nullptr;  // or into one word per file (optional, first)
  // records are handed to warps 32 at a time from this counter, which the
  // launch zeroes first (optional; without it each thread strides)
  unsigned long long *record_counter = nullptr;
  int num_groups = 0;
  BatchQueryGroup groups[kMaxBatchGroups];
};

cudaError_t batch_query_launch(const BatchQueryLaunch &q, const IrBlob &ir, int grid,
                               int block, cudaStream_t stream);

}  // namespace gpjb
