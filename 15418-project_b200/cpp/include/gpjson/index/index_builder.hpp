// Index builders (interface of the reference's
// include/gpjson/index/index_builder.hpp, plus IndexBuilderType::B200).
// Every type builds through the fused B200 indexer: UNCOMBINED, COMBINED,
// FUSED and SHAREMEM produce the same bitmaps in the reference, and here they
// all name the one single-pass build.
#pragma once

#include "gpjson/file/file.hpp"
#include "gpjson/file/file_reader.hpp"
#include "gpjson/index/index.hpp"
#include "gpjson/run_context.hpp"

#include <cstddef>
#include <ostream>

namespace gpjson::index {

enum class IndexBuilderType { UNCOMBINED = 0, COMBINED, FUSED, SHAREMEM, B200 };

std::ostream &operator<<(std::ostream &os, IndexBuilderType type);

struct IndexBuilderOptions {
  IndexBuilderType index_builder_type{IndexBuilderType::UNCOMBINED};
  size_t file_partition_size{0};
  int grid_size{0};             // accepted for compatibility; the B200 build sizes itself
  int block_size{0};
  int reduction_grid_size{0};
  int reduction_block_size{0};
};

std::ostream &operator<<(std::ostream &os, const IndexBuilderOptions &options);

class IndexBuilder {
 public:
  virtual ~IndexBuilder() = default;
  virtual BuiltIndices build(const file::FilePartition &partition, size_t max_depth,
                             const IndexBuilderOptions &options,
                             const gpjson::RunContext &run_context) const = 0;
};

class B200IndexBuilder final : public IndexBuilder {
 public:
  explicit B200IndexBuilder(const file::FileReader &file_reader) : file_reader_(file_reader) {}
  BuiltIndices build(const file::FilePartition &partition, size_t max_depth,
                     const IndexBuilderOptions &options,
                     const gpjson::RunContext &run_context) const override;

 private:
  const file::FileReader &file_reader_;
};

// The reference's four builder classes, all backed by the fused build.
using UncombinedIndexBuilder = B200IndexBuilder;
using CombinedIndexBuilder = B200IndexBuilder;
using FusedIndexBuilder = B200IndexBuilder;
using SharememIndexBuilder = B200IndexBuilder;

}  // namespace gpjson::index
