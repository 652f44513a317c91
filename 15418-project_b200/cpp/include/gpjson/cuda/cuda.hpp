// RAII device array and CUDA helpers (interface of the reference project's
// include/gpjson/cuda/cuda.hpp).
#pragma once

#include <cstddef>

namespace gpjson::cuda {

class DeviceArray {
 public:
  DeviceArray() = default;
  explicit DeviceArray(size_t bytes);
  ~DeviceArray();
  DeviceArray(DeviceArray &&other) noexcept;
  DeviceArray &operator=(DeviceArray &&other) noexcept;
  DeviceArray(const DeviceArray &) = delete;
  DeviceArray &operator=(const DeviceArray &) = delete;

  void *data() { return ptr_; }
  const void *data() const { return ptr_; }
  size_t size_bytes() const { return size_bytes_; }
  bool empty() const { return size_bytes_ == 0; }
  template <typename T> T *as() { return static_cast<T *>(ptr_); }
  template <typename T> const T *as() const { return static_cast<const T *>(ptr_); }

  void copy_from_host(const void *src, size_t bytes);
  void copy_to_host(void *dst, size_t bytes) const;
  void memset(int value);

 private:
  void *ptr_ = nullptr;
  size_t size_bytes_ = 0;
};

// Throws error::cuda::CudaError("<context>: <CUDA message>") on failure.
void check(int cuda_status, const char *context);
bool device_available();
void synchronize_and_check();

}  // namespace gpjson::cuda
