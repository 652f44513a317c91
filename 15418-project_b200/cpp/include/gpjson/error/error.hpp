// Exception hierarchy of the engine's C++ API (same names as the reference
// project's include/gpjson/error, query/error.hpp, file/error.hpp,
// cuda/error.hpp), so callers' catch clauses keep working.
#pragma once

#include <stdexcept>
#include <string>
#include <utility>

namespace gpjson::error {

class GpJSONError : public std::exception {
 public:
  explicit GpJSONError(std::string message) : message_(std::move(message)) {}
  const char *what() const noexcept override { return message_.c_str(); }

 private:
  std::string message_;
};

namespace common {
class ImplementationError : public GpJSONError {
 public:
  using GpJSONError::GpJSONError;
};
class NotImplementedError : public GpJSONError {
 public:
  using GpJSONError::GpJSONError;
};
}  // namespace common

namespace cuda {
class CudaError : public GpJSONError {
 public:
  using GpJSONError::GpJSONError;
};
}  // namespace cuda

namespace file {
class FileError : public GpJSONError {
 public:
  using GpJSONError::GpJSONError;
};
class FileOpenError : public FileError {
 public:
  using FileError::FileError;
};
class FileReadError : public FileError {
 public:
  using FileError::FileError;
};
class PartitionError : public FileError {
 public:
  using FileError::FileError;
};
}  // namespace file

namespace query {
class MalformedQueryError : public GpJSONError {
 public:
  using GpJSONError::GpJSONError;
};
class UnsupportedQueryError : public GpJSONError {
 public:
  using GpJSONError::GpJSONError;
};
class QueryExecutionError : public GpJSONError {
 public:
  using GpJSONError::GpJSONError;
};
}  // namespace query

// Throws the exception that matches a gpj_* status (no-op for GPJ_OK).
void throw_for_status(int status, const char *context);

}  // namespace gpjson::error
