// Query executor (interface of the reference's
// include/gpjson/query/query_executor.hpp): every query of a batch over one
// partition, one kernel launch per query, results materialised on the host.
#pragma once

#include "gpjson/file/file.hpp"
#include "gpjson/index/index.hpp"
#include "gpjson/query/query.hpp"

#include <ostream>

namespace gpjson {
struct EngineOptions;
}

namespace gpjson::query {

struct QueryExecutorOptions {
  int grid_size{512};
  int block_size{1024};
};

std::ostream &operator<<(std::ostream &os, const QueryExecutorOptions &options);

class QueryExecutor {
 public:
  explicit QueryExecutor(const gpjson::EngineOptions &options);
  BatchQueryResult execute_batch(const BatchCompiledQuery &queries,
                                 const file::FilePartition &partition,
                                 const index::BuiltIndices &built) const;

 private:
  int grid_size_ = 512;
  int block_size_ = 1024;
};

}  // namespace gpjson::query
