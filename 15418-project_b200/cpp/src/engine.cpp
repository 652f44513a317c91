// Engine::query (flow of the reference's src/gpjson/engine.cpp:97-175):
// compile, partition, then per partition load -> fused index build -> queries
// -> materialise, merging the partitions' lines in order.
#include "gpjson/engine.hpp"
#include "gpjson/error/error.hpp"
#include "gpjson/run_context.hpp"

#include <memory>

namespace gpjson {

std::ostream &operator<<(std::ostream &os, const EngineOptions &o) {
  return os << "EngineOptions{file_reader_options=" << o.file_reader_options
            << ", index_builder_options=" << o.index_builder_options
            << ", query_executor_options=" << o.query_executor_options << "}";
}

query::MaterializedBatchResult Engine::query(const std::string &file_path,
                                             const std::vector<std::string> &queries_src,
                                             const EngineOptions &options) const {
  if (queries_src.empty()) return {};
  profiler::Profiler prof("Engine::query profiler");
  RunContext rc{prof};
  const auto engine_t = prof.begin("Engine::query");

  query::QueryCompiler compiler(options);
  query::QueryExecutor executor(options);
  const auto comp_t = prof.begin("query_compilation");
  query::BatchCompiledQuery compiled;
  for (const auto &q : queries_src) compiled.add(compiler.compile(q, options));
  prof.end(comp_t);

  std::unique_ptr<file::FileReader> reader;
  switch (options.file_reader_options.file_reader_type) {
    case file::FileReaderType::COPIED:
      reader = std::make_unique<file::CopiedFileReader>(file_path);
      break;
    case file::FileReaderType::MMAP:
      reader = std::make_unique<file::MmapFileReader>(file_path);
      break;
    default:
      throw error::common::ImplementationError("Undefined file reader type.");
  }
  const auto part_t = prof.begin("file_reader.create_partitions");
  reader->create_partitions(options.index_builder_options.file_partition_size);
  prof.end(part_t);

  index::B200IndexBuilder builder(*reader);
  std::vector<query::MaterializedQueryResult> merged;
  for (const auto &q : compiled.queries()) merged.emplace_back(q.query_text());

  for (auto &partition : reader->get_partitions()) {
    const size_t id = partition.partition_id();
    const auto total_t = prof.begin_nestedf("partition %zu total", id);
    auto t = prof.begin_nestedf("partition %zu load_to_device", id);
    partition.load_to_device();
    prof.end(t);
    t = prof.begin_nestedf("partition %zu build_index", id);
    index::BuiltIndices built = builder.build(partition, compiled.get_max_depth(),
                                              options.index_builder_options, rc);
    prof.end(t);
    t = prof.begin_nestedf("partition %zu execute_query", id);
    const query::BatchQueryResult batch = executor.execute_batch(compiled, partition, built);
    prof.end(t);
    t = prof.begin_nestedf("partition %zu materialize_results", id);
    const query::MaterializedBatchResult part = batch.materialize();
    prof.end(t);
    if (part.queries().size() != merged.size())
      throw error::common::ImplementationError(
          "Partition query results do not match the compiled query batch.");
    for (size_t q = 0; q < merged.size(); ++q)
      for (const auto &line : part.queries()[q].lines()) merged[q].add_line_result(line);
    prof.end(total_t);
  }
  query::MaterializedBatchResult out;
  for (auto &q : merged) out.add_query_result(std::move(q));
  prof.end(engine_t);
  return out;
}

}  // namespace gpjson
