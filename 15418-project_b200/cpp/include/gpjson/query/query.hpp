// Compiled queries and result types (interface of the reference's
// include/gpjson/query/query.hpp).
#pragma once

#include <cstddef>
#include <optional>
#include <string>
#include <vector>

namespace gpjson::query {

enum class QueryOpcode : unsigned char {
  END = 0,
  STORE_RESULT = 1,
  MOVE_UP = 2,
  MOVE_DOWN = 3,
  MOVE_TO_KEY = 4,
  MOVE_TO_INDEX = 5,
  MOVE_TO_INDEX_REVERSE = 6,
  MARK_POSITION = 7,
  RESET_POSITION = 8,
  EXPRESSION_STRING_EQUALS = 9,
};

class CompiledQuery {
 public:
  CompiledQuery() = default;
  CompiledQuery(std::string query_text, std::vector<std::byte> ir_bytes, size_t max_depth,
                size_t num_result_slots);
  const std::string &query_text() const { return query_text_; }
  const std::vector<std::byte> &ir_bytes() const { return ir_bytes_; }
  size_t max_depth() const { return max_depth_; }
  size_t num_result_slots() const { return num_result_slots_; }

 private:
  std::string query_text_;
  std::vector<std::byte> ir_bytes_;
  size_t max_depth_ = 1;
  size_t num_result_slots_ = 1;
};

class BatchCompiledQuery {
 public:
  void add(CompiledQuery query);
  size_t size() const { return queries_.size(); }
  size_t get_max_depth() const { return max_depth_; }
  const std::vector<CompiledQuery> &queries() const { return queries_; }

 private:
  std::vector<CompiledQuery> queries_;
  size_t max_depth_ = 1;
};

struct QueryOffset {
  std::optional<size_t> start;
  std::optional<size_t> end;
  std::optional<std::string> json_text;
};

class LineQueryResult {
 public:
  const std::vector<QueryOffset> &offsets() const { return offsets_; }
  void add_offset(QueryOffset offset) { offsets_.push_back(std::move(offset)); }

 private:
  std::vector<QueryOffset> offsets_;
};

class QueryResult {
 public:
  void add_line_result(LineQueryResult line) { lines_.push_back(std::move(line)); }
  const std::vector<LineQueryResult> &lines() const { return lines_; }

 private:
  std::vector<LineQueryResult> lines_;
};

class MaterializedBatchResult;

class BatchQueryResult {
 public:
  explicit BatchQueryResult(size_t num_queries) : queries_(num_queries), texts_(num_queries) {}
  void add_line_result(size_t query_index, LineQueryResult line);
  void merge(const BatchQueryResult &other);
  void set_query_text(size_t query_index, std::string text);
  MaterializedBatchResult materialize() const;
  size_t num_queries() const { return queries_.size(); }
  const std::vector<QueryResult> &queries() const { return queries_; }

 private:
  std::vector<QueryResult> queries_;
  std::vector<std::string> texts_;
};

class MaterializedValue {
 public:
  explicit MaterializedValue(std::string json_text) : json_text_(std::move(json_text)) {}
  const std::string &json_text() const { return json_text_; }

 private:
  std::string json_text_;
};

class MaterializedLineResult {
 public:
  const std::vector<MaterializedValue> &values() const { return values_; }
  void add_value(MaterializedValue v) { values_.push_back(std::move(v)); }

 private:
  std::vector<MaterializedValue> values_;
};

class MaterializedQueryResult {
 public:
  explicit MaterializedQueryResult(std::string text) : query_text_(std::move(text)) {}
  const std::string &query_text() const { return query_text_; }
  const std::vector<MaterializedLineResult> &lines() const { return lines_; }
  void add_line_result(MaterializedLineResult line) { lines_.push_back(std::move(line)); }

 private:
  std::string query_text_;
  std::vector<MaterializedLineResult> lines_;
};

class MaterializedBatchResult {
 public:
  const std::vector<MaterializedQueryResult> &queries() const { return queries_; }
  void add_query_result(MaterializedQueryResult r) { queries_.push_back(std::move(r)); }

 private:
  std::vector<MaterializedQueryResult> queries_;
};

class QueryOptions {};

}  // namespace gpjson::query
