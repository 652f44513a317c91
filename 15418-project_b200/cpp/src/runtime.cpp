// Errors, DeviceArray, profiler and the shared engine context of the C++ API.
#include "gpjson/cuda/cuda.hpp"
#include "gpjson/error/error.hpp"
#include "gpjson/profiler/profiler.hpp"
#include "gpjson_b200.h"
#include "internal.hpp"

#include <cuda_runtime_api.h>

#include <cstdarg>
#include <cstdio>
#include <mutex>
#include <stdexcept>
#include <string>

namespace gpjson::error {

void throw_for_status(int status, const char *context) {
  if (status == GPJ_OK) return;
  std::string m = gpj_last_error();
  if (context && *context) m = std::string(context) + ": " + m;
  switch (status) {
    case GPJ_ERR_CUDA:
    case GPJ_ERR_OOM:
    case GPJ_ERR_TIMEOUT:
      throw cuda::CudaError(m);
    case GPJ_ERR_MALFORMED_QUERY:
      throw query::MalformedQueryError(gpj_last_error());
    case GPJ_ERR_UNSUPPORTED_QUERY:
      throw query::UnsupportedQueryError(gpj_last_error());
    case GPJ_ERR_EXECUTION:
      throw query::QueryExecutionError(gpj_last_error());
    case GPJ_ERR_INVALID_ARGUMENT:
      throw std::invalid_argument(gpj_last_error());
    case GPJ_ERR_OUT_OF_RANGE:
      throw std::out_of_range(gpj_last_error());
    default:
      throw common::ImplementationError(m);
  }
}

}  // namespace gpjson::error

namespace gpjson::cuda {

void check(int status, const char *context) {
  if (status != cudaSuccess) {
    throw error::cuda::CudaError(std::string(context) + ": " +
                                 cudaGetErrorString(static_cast<cudaError_t>(status)));
  }
}

bool device_available() {
  int count = 0;
  return cudaGetDeviceCount(&count) == cudaSuccess && count > 0;
}

void synchronize_and_check() {
  check(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
  check(cudaGetLastError(), "cudaGetLastError");
}

DeviceArray::DeviceArray(size_t bytes) : size_bytes_(bytes) {
  if (bytes > 0) check(cudaMalloc(&ptr_, bytes), "cudaMalloc");
}

DeviceArray::~DeviceArray() {
  if (ptr_ != nullptr) cudaFree(ptr_);
}

DeviceArray::DeviceArray(DeviceArray &&o) noexcept : ptr_(o.ptr_), size_bytes_(o.size_bytes_) {
  o.ptr_ = nullptr;
  o.size_bytes_ = 0;
}

DeviceArray &DeviceArray::operator=(DeviceArray &&o) noexcept {
  if (this != &o) {
    if (ptr_ != nullptr) cudaFree(ptr_);
    ptr_ = o.ptr_;
    size_bytes_ = o.size_bytes_;
    o.ptr_ = nullptr;
    o.size_bytes_ = 0;
  }
  return *this;
}

void DeviceArray::copy_from_host(const void *src, size_t bytes) {
  if (bytes > size_bytes_)
    throw error::cuda::CudaError("copy_from_host: requested byte count exceeds allocation");
  if (bytes == 0) return;
  if (src == nullptr) throw error::cuda::CudaError("copy_from_host: host pointer is null");
  check(cudaMemcpy(ptr_, src, bytes, cudaMemcpyHostToDevice), "cudaMemcpy host to device");
}

void DeviceArray::copy_to_host(void *dst, size_t bytes) const {
  if (bytes > size_bytes_)
    throw error::cuda::CudaError("copy_to_host: requested byte count exceeds allocation");
  if (bytes == 0) return;
  if (dst == nullptr) throw error::cuda::CudaError("copy_to_host: host pointer is null");
  check(cudaMemcpy(dst, ptr_, bytes, cudaMemcpyDeviceToHost), "cudaMemcpy device to host");
}

void DeviceArray::memset(int value) {
  if (size_bytes_ > 0) check(cudaMemset(ptr_, value, size_bytes_), "cudaMemset");
}

}  // namespace gpjson::cuda

namespace gpjson::profiler {

Profiler::Profiler(std::string name) : name_(std::move(name)) {}

Profiler::SegmentId Profiler::open(std::string segment, bool nested) {
  Record r;
  r.name = std::move(segment);
  r.start = std::chrono::steady_clock::now();
  r.indent = indent_;
  r.opens_scope = nested;
  if (nested) ++indent_;
  records_.push_back(std::move(r));
  return SegmentId(records_.size() - 1);
}

Profiler::SegmentId Profiler::begin(const std::string &s) { return open(s, false); }
Profiler::SegmentId Profiler::begin_nested(const std::string &s) { return open(s, true); }

static std::string vformat(const char *fmt, va_list ap) {
  char buf[512];
  std::vsnprintf(buf, sizeof(buf), fmt, ap);
  return buf;
}

Profiler::SegmentId Profiler::beginf(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  std::string s = vformat(fmt, ap);
  va_end(ap);
  return open(std::move(s), false);
}

Profiler::SegmentId Profiler::begin_nestedf(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  std::string s = vformat(fmt, ap);
  va_end(ap);
  return open(std::move(s), true);
}

void Profiler::end(SegmentId id) {
  if (!id.valid_ || id.index_ >= records_.size()) return;
  Record &r = records_[id.index_];
  if (r.done) return;
  if (r.opens_scope && indent_ > 0) --indent_;
  r.done = true;
  const double ms =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - r.start).count();
  std::fprintf(stdout, "%s: %*s%s: %.3f ms\n", name_.c_str(), int(r.indent * 2), "",
               r.name.c_str(), ms);
  std::fflush(stdout);
}

}  // namespace gpjson::profiler

namespace gpjson::detail {

gpj_ctx *engine_context() {
  static std::mutex mu;
  static gpj_ctx *ctx = nullptr;
  std::lock_guard<std::mutex> lock(mu);
  if (ctx == nullptr) {
    int dev = 0;
    cudaGetDevice(&dev);
    error::throw_for_status(gpj_ctx_create(dev, &ctx), "gpj_ctx_create");
  }
  return ctx;
}

}  // namespace gpjson::detail
