// JSONPath compiler (interface of the reference's QueryCompiler; the parser
// runs in the engine library through gpj_compile).
#pragma once

#include "gpjson/error/error.hpp"
#include "gpjson/query/query.hpp"

#include <string>

namespace gpjson {
struct EngineOptions;
}

namespace gpjson::query {

class QueryCompiler {
 public:
  explicit QueryCompiler(const gpjson::EngineOptions &options);
  // Throws MalformedQueryError / UnsupportedQueryError (and
  // std::invalid_argument / std::out_of_range for unparsable integers).
  CompiledQuery compile(const std::string &query_src, const gpjson::EngineOptions &options) const;
};

}  // namespace gpjson::query
