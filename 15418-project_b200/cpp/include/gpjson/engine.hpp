// Engine entry point (interface of the reference's include/gpjson/engine.hpp).
#pragma once

#include "gpjson/file/file_reader.hpp"
#include "gpjson/index/index_builder.hpp"
#include "gpjson/query/query.hpp"
#include "gpjson/query/query_executor.hpp"

#include <ostream>
#include <string>
#include <vector>

namespace gpjson {

struct EngineOptions {
  file::FileReaderOptions file_reader_options;
  index::IndexBuilderOptions index_builder_options;
  query::QueryExecutorOptions query_executor_options;
};

std::ostream &operator<<(std::ostream &os, const EngineOptions &options);

class Engine {
 public:
  // Compiles the queries, splits the file into newline-aligned partitions,
  // and per partition: copies it to the device, builds the indexes with the
  // fused B200 indexer, runs every query and materialises the matches.
  query::MaterializedBatchResult query(const std::string &file_path,
                                       const std::vector<std::string> &queries_src,
                                       const EngineOptions &options) const;
};

}  // namespace gpjson

#include "gpjson/query/query_compiler.hpp"
