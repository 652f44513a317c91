// File readers and newline-aligned partitioning (behaviour of the reference's
// src/gpjson/file/file_reader.cpp:18-77 and file.cpp:30-36).
#include "gpjson/error/error.hpp"
#include "gpjson/file/file_reader.hpp"
#include "gpjson_b200.h"
#include "internal.hpp"

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cerrno>
#include <cstring>
#include <fstream>
#include <sstream>

namespace gpjson::file {

FilePartition::FilePartition(size_t partition_id, size_t start, size_t end, const void *data)
    : partition_id_(partition_id), global_start_offset_(start), global_end_offset_(end),
      host_data_(data) {}

void FilePartition::load_to_device() {
  if (device_loaded()) return;
  device_data_ = cuda::DeviceArray(size_bytes());
  // mmap'd and other pageable bytes go through the engine context's pinned
  // staging ring (gpj_copy_to_device), not a synchronous pageable cudaMemcpy
  error::throw_for_status(gpj_copy_to_device(detail::engine_context(), device_data_.data(),
                                             host_data_, size_bytes(), nullptr),
                          "load_to_device");
  cuda::synchronize_and_check();
}

std::ostream &operator<<(std::ostream &os, FileReaderType type) {
  switch (type) {
    case FileReaderType::COPIED: return os << "COPIED";
    case FileReaderType::MMAP: return os << "MMAP";
  }
  return os << "UNKNOWN(" << int(type) << ")";
}

std::ostream &operator<<(std::ostream &os, const FileReaderOptions &o) {
  return os << "FileReaderOptions{file_reader_type=" << o.file_reader_type << "}";
}

std::vector<FilePartition> partition_bytes(const std::string &path, const unsigned char *base,
                                           size_t size, size_t psize) {
  std::vector<FilePartition> parts;
  if (psize == 0 || size == 0 || size <= psize) {
    parts.emplace_back(0, 0, size, base);
    return parts;
  }
  size_t start = 0, id = 0;
  while (size - start > psize) {
    // the last '\n' at or before start + psize ends this partition
    const size_t target = start + psize;
    size_t next = 0;
    for (size_t off = target;; --off) {
      if (base[off] == '\n') {
        next = off + 1;
        break;
      }
      if (off == start) {
        std::ostringstream m;
        m << "Cannot partition file '" << path << "' using partition size " << psize
          << ": no newline found before offset " << target << ".";
        throw error::file::PartitionError(m.str());
      }
    }
    if (next >= size) break;
    parts.emplace_back(id, start, next - 1, base == nullptr ? nullptr : base + start);
    start = next;
    ++id;
  }
  parts.emplace_back(id, start, size, base == nullptr ? nullptr : base + start);
  return parts;
}

static size_t file_size_of(const std::string &path) {
  struct stat st {};
  if (::stat(path.c_str(), &st) != 0)
    throw error::file::FileOpenError("Failed to get size for file '" + path +
                                     "': " + std::strerror(errno));
  return size_t(st.st_size);
}

CopiedFileReader::CopiedFileReader(std::string file_path) : file_path_(std::move(file_path)) {
  metadata_.file_path = file_path_;
}

void CopiedFileReader::create_partitions(size_t psize) {
  metadata_.file_size_bytes = file_size_of(file_path_);
  bytes_.assign(metadata_.file_size_bytes, 0);
  std::ifstream in(file_path_, std::ios::binary);
  if (!in) throw error::file::FileOpenError("Failed to open file '" + file_path_ + "' for reading.");
  if (!bytes_.empty()) {
    in.read(reinterpret_cast<char *>(bytes_.data()), std::streamsize(bytes_.size()));
    if (!in || size_t(in.gcount()) != bytes_.size())
      throw error::file::FileReadError("Failed to read all bytes from file '" + file_path_ + "'.");
  }
  partitions_ = partition_bytes(file_path_, bytes_.empty() ? nullptr : bytes_.data(),
                                bytes_.size(), psize);
  metadata_.num_partitions = partitions_.size();
}

MmapFileReader::MmapFileReader(std::string file_path) : file_path_(std::move(file_path)) {
  metadata_.file_path = file_path_;
}

MmapFileReader::~MmapFileReader() {
  if (mapped_ != nullptr && mapped_size_ > 0)
    munmap(const_cast<unsigned char *>(mapped_), mapped_size_);
  if (fd_ != -1) close(fd_);
}

void MmapFileReader::create_partitions(size_t psize) {
  if (fd_ == -1) {
    metadata_.file_size_bytes = file_size_of(file_path_);
    fd_ = open(file_path_.c_str(), O_RDONLY);
    if (fd_ == -1)
      throw error::file::FileOpenError("Failed to open file '" + file_path_ +
                                       "' for reading: " + std::strerror(errno) + ".");
    if (metadata_.file_size_bytes > 0) {
      void *p = mmap(nullptr, metadata_.file_size_bytes, PROT_READ, MAP_PRIVATE, fd_, 0);
      if (p == MAP_FAILED)
        throw error::file::FileReadError("Failed to mmap file '" + file_path_ +
                                         "': " + std::strerror(errno) + ".");
      mapped_ = static_cast<const unsigned char *>(p);
      mapped_size_ = metadata_.file_size_bytes;
    }
  }
  partitions_ = partition_bytes(file_path_, mapped_, metadata_.file_size_bytes, psize);
  metadata_.num_partitions = partitions_.size();
}

}  // namespace gpjson::file
