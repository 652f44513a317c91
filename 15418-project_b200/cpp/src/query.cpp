// Compiled-query and result containers, compiler and executor of the C++ API
// (behaviour of the reference's src/gpjson/query/query.cpp,
// query_compiler.cpp and kernels/orig/query_executor_host.cu:80-241).
#include "gpjson/engine.hpp"
#include "gpjson/error/error.hpp"
#include "gpjson/query/query.hpp"
#include "gpjson/query/query_compiler.hpp"
#include "gpjson/query/query_executor.hpp"
#include "gpjson_b200.h"
#include "internal.hpp"

#include <cuda_runtime_api.h>

#include <algorithm>
#include <cstdint>
#include <limits>
#include <vector>

namespace gpjson::query {

CompiledQuery::CompiledQuery(std::string text, std::vector<std::byte> ir, size_t max_depth,
                             size_t slots)
    : query_text_(std::move(text)), ir_bytes_(std::move(ir)), max_depth_(max_depth),
      num_result_slots_(slots) {}

void BatchCompiledQuery::add(CompiledQuery q) {
  max_depth_ = std::max(max_depth_, q.max_depth());
  queries_.push_back(std::move(q));
}

void BatchQueryResult::add_line_result(size_t qi, LineQueryResult line) {
  if (qi < queries_.size()) queries_[qi].add_line_result(std::move(line));
}

void BatchQueryResult::merge(const BatchQueryResult &other) {
  if (queries_.size() != other.queries_.size()) return;
  for (size_t q = 0; q < queries_.size(); ++q) {
    if (texts_[q].empty()) texts_[q] = other.texts_[q];
    for (const auto &l : other.queries_[q].lines()) queries_[q].add_line_result(l);
  }
}

void BatchQueryResult::set_query_text(size_t qi, std::string text) {
  if (qi < texts_.size()) texts_[qi] = std::move(text);
}

MaterializedBatchResult BatchQueryResult::materialize() const {
  MaterializedBatchResult out;
  for (size_t q = 0; q < queries_.size(); ++q) {
    MaterializedQueryResult qr(texts_[q]);
    for (const auto &line : queries_[q].lines()) {
      MaterializedLineResult ml;
      for (const auto &o : line.offsets())
        if (o.json_text.has_value()) ml.add_value(MaterializedValue(*o.json_text));
      if (!ml.values().empty()) qr.add_line_result(std::move(ml));  // lines without matches drop
    }
    out.add_query_result(std::move(qr));
  }
  return out;
}

QueryCompiler::QueryCompiler(const gpjson::EngineOptions &) {}

CompiledQuery QueryCompiler::compile(const std::string &src, const gpjson::EngineOptions &) const {
  std::vector<uint8_t> ir(4096);
  uint64_t len = 0, depth = 0, slots = 0;
  int rc = gpj_compile(src.c_str(), 0, ir.data(), ir.size(), &len, &depth, &slots);
  if (rc == GPJ_ERR_CAPACITY) {
    ir.resize(len);
    rc = gpj_compile(src.c_str(), 0, ir.data(), ir.size(), &len, &depth, &slots);
  }
  error::throw_for_status(rc, "");
  std::vector<std::byte> bytes(len);
  for (uint64_t i = 0; i < len; ++i) bytes[i] = std::byte(ir[i]);
  return CompiledQuery(src, std::move(bytes), depth, slots);
}

std::ostream &operator<<(std::ostream &os, const QueryExecutorOptions &o) {
  return os << "QueryExecutorOptions{grid_size=" << o.grid_size
            << ", block_size=" << o.block_size << "}";
}

QueryExecutor::QueryExecutor(const gpjson::EngineOptions &options)
    : grid_size_(options.query_executor_options.grid_size),
      block_size_(options.query_executor_options.block_size) {}

namespace {
error::query::QueryExecutionError exec_error(const std::string &m) {
  return error::query::QueryExecutionError(m);
}
}  // namespace

BatchQueryResult QueryExecutor::execute_batch(const BatchCompiledQuery &queries,
                                              const file::FilePartition &partition,
                                              const index::BuiltIndices &built) const {
  BatchQueryResult result(queries.size());
  for (size_t q = 0; q < queries.size(); ++q)
    result.set_query_text(q, queries.queries()[q].query_text());
  if (queries.size() == 0 || partition.size_bytes() == 0 || partition.host_bytes() == nullptr)
    return result;
  if (partition.device_bytes() == nullptr)
    throw exec_error("Query execution requires a GPU-resident partition buffer");
  if (!cuda::device_available()) throw exec_error("CUDA device unavailable for query execution");
  const int num_lines = built.get_newline_index().num_lines();
  if (num_lines <= 0) return result;
  if (built.get_newline_index().data() == nullptr || built.get_string_index().data() == nullptr ||
      built.get_leveled_bitmap_index().data() == nullptr)
    throw exec_error("Query execution requires GPU-resident newline, string, and bitmap indices");
  if (partition.size_bytes() > size_t(std::numeric_limits<int>::max()))
    throw exec_error("partition size exceeds CUDA int range");

  gpj_ctx *ctx = detail::engine_context();
  profiler::Profiler prof("Engine::query profiler");
  const auto batch_t = prof.begin_nested("execute_batch");
  gpj_index ix{};
  ix.d_input = static_cast<const uint8_t *>(partition.device_bytes());
  ix.size_bytes = partition.size_bytes();
  ix.d_newline = const_cast<int64_t *>(
      static_cast<const int64_t *>(built.get_newline_index().data()));
  ix.num_lines = uint64_t(num_lines);
  ix.newline_capacity = uint64_t(num_lines);
  ix.d_string = const_cast<uint64_t *>(
      static_cast<const uint64_t *>(built.get_string_index().data()));
  ix.d_leveled = const_cast<uint64_t *>(
      static_cast<const uint64_t *>(built.get_leveled_bitmap_index().data()));
  ix.num_words = (ix.size_bytes + 63) / 64;
  ix.num_levels = built.get_leveled_bitmap_index().num_levels();

  const size_t base = partition.global_start_offset();
  for (size_t q = 0; q < queries.size(); ++q) {
    const auto total_t = prof.begin_nestedf("query %zu total", q);
    const CompiledQuery &cq = queries.queries()[q];
    if (cq.max_depth() > size_t(ix.num_levels))
      throw exec_error("Query requires more bitmap levels than the index provides");
    if (cq.max_depth() >= size_t(GPJ_MAX_QUERY_DEPTH))
      throw exec_error("Query exceeds the maximum CUDA executor depth");
    if (cq.ir_bytes().size() > size_t(GPJ_MAX_QUERY_IR))
      throw exec_error("Compiled query IR exceeds constant memory buffer");
    const size_t slots = cq.num_result_slots();
    const size_t count = size_t(num_lines) * slots * 2;
    auto alloc_t = prof.begin("allocate_device_result");
    cuda::DeviceArray dev(count * sizeof(int32_t));
    prof.end(alloc_t);
    auto kt = prof.begin("query");
    error::throw_for_status(
        gpj_query_run(ctx, &ix, reinterpret_cast<const uint8_t *>(cq.ir_bytes().data()),
                      cq.ir_bytes().size(), uint32_t(slots), dev.as<int32_t>(), nullptr),
        "query");
    cuda::synchronize_and_check();
    prof.end(kt);
    // Compaction on the device (gpj_results_compact): only the matches and
    // their bytes cross PCIe, not the int32[lines][slots][2] array.  A first
    // pass counts them, the second writes them into exact buffers.
    auto ct = prof.begin("copy_result_to_host");
    cuda::DeviceArray counts(3 * sizeof(uint64_t));
    uint64_t cnt[3] = {0, 0, 0};
    error::throw_for_status(
        gpj_results_compact(ctx, dev.as<int32_t>(), uint64_t(num_lines), uint32_t(slots),
                            ix.d_input, ix.size_bytes, int64_t(base), nullptr, 0, nullptr, 0,
                            counts.as<uint64_t>(), nullptr),
        "compact");
    counts.copy_to_host(cnt, sizeof(cnt));
    if (cnt[2] != 0) throw exec_error("Query kernel produced an invalid result range");
    std::vector<gpj_match> matches(static_cast<size_t>(cnt[0]));
    std::vector<char> arena(static_cast<size_t>(cnt[1]));
    if (cnt[0] > 0) {
      cuda::DeviceArray d_matches(static_cast<size_t>(cnt[0]) * sizeof(gpj_match));
      cuda::DeviceArray d_arena(std::max<size_t>(1, static_cast<size_t>(cnt[1])));
      error::throw_for_status(
          gpj_results_compact(ctx, dev.as<int32_t>(), uint64_t(num_lines), uint32_t(slots),
                              ix.d_input, ix.size_bytes, int64_t(base),
                              d_matches.as<gpj_match>(), cnt[0], d_arena.as<uint8_t>(), cnt[1],
                              counts.as<uint64_t>(), nullptr),
          "compact");
      d_matches.copy_to_host(matches.data(), matches.size() * sizeof(gpj_match));
      if (!arena.empty()) d_arena.copy_to_host(arena.data(), arena.size());
    }
    prof.end(ct);
    auto at = prof.begin("append_query_line_results");
    // every line keeps one offset per slot, empty where nothing matched
    // (query_executor_host.cu:80-119)
    size_t m = 0;
    for (int line = 0; line < num_lines; ++line) {
      LineQueryResult lr;
      for (size_t slot = 0; slot < slots; ++slot) {
        if (m < matches.size() && matches[m].line == uint64_t(line) && matches[m].slot == slot) {
          const gpj_match &g = matches[m++];
          QueryOffset o;
          o.start = size_t(g.start);
          o.end = size_t(g.end);
          o.json_text = std::string(arena.data() + g.text_offset, g.length);
          lr.add_offset(std::move(o));
        } else {
          lr.add_offset(QueryOffset{});
        }
      }
      result.add_line_result(q, std::move(lr));
    }
    prof.end(at);
    prof.end(total_t);
  }
  prof.end(batch_t);
  return result;
}

}  // namespace gpjson::query
