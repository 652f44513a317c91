// JSONPath compiler (host).  See compiler.cpp.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "gpjson_b200.h"

namespace gpjb {

struct CompiledIr {
  std::vector<uint8_t> ir;
  uint64_t max_depth = 0;
  uint64_t num_result_slots = 0;
};

struct CompileError {
  int code;             // GPJ_ERR_*
  std::string message;  // same text as the reference's exception
};

// Throws CompileError.
CompiledIr compile_query(const std::string &text, uint64_t wildcard_limit);

}  // namespace gpjb
