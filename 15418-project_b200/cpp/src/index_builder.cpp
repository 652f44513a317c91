// IndexBuilder over the fused B200 indexer (gpj_index_build_async into
// DeviceArrays owned by the returned BuiltIndices).
#include "gpjson/error/error.hpp"
#include "gpjson/index/index_builder.hpp"
#include "gpjson_b200.h"
#include "internal.hpp"

#include <cuda_runtime_api.h>

#include <cstdint>

namespace gpjson::index {

std::ostream &operator<<(std::ostream &os, IndexBuilderType t) {
  switch (t) {
    case IndexBuilderType::UNCOMBINED: return os << "UNCOMBINED";
    case IndexBuilderType::COMBINED: return os << "COMBINED";
    case IndexBuilderType::FUSED: return os << "FUSED";
    case IndexBuilderType::SHAREMEM: return os << "SHAREMEM";
    case IndexBuilderType::B200: return os << "B200";
  }
  return os << "UNKNOWN(" << int(t) << ")";
}

std::ostream &operator<<(std::ostream &os, const IndexBuilderOptions &o) {
  return os << "IndexBuilderOptions{index_builder_type=" << o.index_builder_type
            << ", file_partition_size=" << o.file_partition_size
            << ", grid_size=" << o.grid_size << ", block_size=" << o.block_size
            << ", reduction_grid_size=" << o.reduction_grid_size
            << ", reduction_block_size=" << o.reduction_block_size << "}";
}

BuiltIndices B200IndexBuilder::build(const file::FilePartition &partition, size_t max_depth,
                                     const IndexBuilderOptions &, const gpjson::RunContext &rc) const {
  const size_t n = partition.size_bytes();
  if (n > 0 && partition.device_bytes() == nullptr)
    throw error::common::ImplementationError(
        "Index building requires a GPU-resident partition buffer");
  if (max_depth > size_t(GPJ_MAX_LEVELS))
    throw error::common::ImplementationError("max_depth exceeds the 22 leveled-bitmap levels");
  gpj_ctx *ctx = detail::engine_context();
  const size_t W = (n + 63) / 64;
  auto t = rc.profiler.begin("b200_fused_index");
  cuda::DeviceArray S(W * sizeof(uint64_t)), LB(W * max_depth * sizeof(uint64_t));
  cuda::DeviceArray summary(4 * sizeof(uint64_t));
  uint64_t cap = n / 32 + 1024;
  for (int attempt = 0;; ++attempt) {
    cuda::DeviceArray NL(cap * sizeof(int64_t));
    gpj_index ix{};
    ix.d_string = S.as<uint64_t>();
    ix.d_leveled = LB.as<uint64_t>();
    ix.d_newline = NL.as<int64_t>();
    ix.newline_capacity = cap;
    error::throw_for_status(
        gpj_index_build_async(ctx, static_cast<const uint8_t *>(partition.device_bytes()), n,
                              int(max_depth), 0u, &ix, summary.as<uint64_t>(), nullptr),
        "index build");
    uint64_t s[4] = {0, 0, 0, 0};
    summary.copy_to_host(s, sizeof(s));  // lines, in-string, depth, error bits
    if (s[3] != 0) error::throw_for_status(GPJ_ERR_TIMEOUT, "index build");
    if (s[0] <= cap || attempt == 1) {
      rc.profiler.end(t);
      // the newline array is sized to the line count, like the reference's
      cuda::DeviceArray exact(s[0] * sizeof(int64_t));
      cuda::check(cudaMemcpy(exact.data(), NL.data(), s[0] * sizeof(int64_t),
                             cudaMemcpyDeviceToDevice),
                  "cudaMemcpy newline index");
      return {NewlineIndex(std::move(exact), int(s[0])), StringIndex(std::move(S)),
              LeveledBitmapIndex(std::move(LB), int(max_depth))};
    }
    cap = s[0];
  }
}

}  // namespace gpjson::index
