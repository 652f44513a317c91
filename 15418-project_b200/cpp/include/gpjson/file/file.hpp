// A newline-aligned slice of a file: borrows the reader's host bytes and owns
// its device copy (interface of the reference's include/gpjson/file/file.hpp).
#pragma once

#include "gpjson/cuda/cuda.hpp"

#include <cstddef>
#include <string>

namespace gpjson::file {

class FilePartition {
 public:
  FilePartition() = default;
  FilePartition(size_t partition_id, size_t global_start_offset, size_t global_end_offset,
                const void *data);
  FilePartition(const FilePartition &) = delete;
  FilePartition &operator=(const FilePartition &) = delete;
  FilePartition(FilePartition &&) noexcept = default;
  FilePartition &operator=(FilePartition &&) noexcept = default;

  size_t partition_id() const { return partition_id_; }
  size_t global_start_offset() const { return global_start_offset_; }
  size_t global_end_offset() const { return global_end_offset_; }
  size_t size_bytes() const { return global_end_offset_ - global_start_offset_; }
  const void *host_bytes() const { return host_data_; }
  const void *device_bytes() const { return device_data_.data(); }
  bool device_loaded() const { return size_bytes() == 0 || device_data_.data() != nullptr; }
  // Copies the bytes to the device once; later calls keep the first copy.
  void load_to_device();

 private:
  size_t partition_id_ = 0;
  size_t global_start_offset_ = 0;
  size_t global_end_offset_ = 0;
  const void *host_data_ = nullptr;
  cuda::DeviceArray device_data_;
};

struct FileMetadata {
  std::string file_path;
  size_t file_size_bytes = 0;
  size_t num_partitions = 0;
};

}  // namespace gpjson::file
