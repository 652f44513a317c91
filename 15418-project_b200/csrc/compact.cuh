// Device-side compaction of query results (internal; the public surface is
// gpj_results_compact in include/gpjson_b200.h).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "gpjson_b200.h"

namespace gpjb {

// Bytes of scratch compact_launch needs (per-block counts), 256-byte aligned.
uint64_t compact_scratch_bytes(uint64_t lines, uint32_t slots);

// Clears d_counts, then: d_counts[0] = matches, [1] = arena bytes, [2] =
// invalid ranges.  Matches and bytes beyond the capacities are counted but
// not written.  d_arena or d_input may be null (no bytes gathered).
cudaError_t compact_launch(const int32_t *d_results, uint64_t lines, uint32_t slots,
                           const uint8_t *d_input, uint64_t n, int64_t base_offset,
                           gpj_match *d_matches, uint64_t match_cap, uint8_t *d_arena,
                           uint64_t arena_cap, unsigned long long *d_counts, void *scratch,
                           cudaStream_t stream);

}  // namespace gpjb
