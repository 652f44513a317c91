// File readers (whole-file copy or mmap) and newline-aligned partitioning
// (interface of the reference's include/gpjson/file/file_reader.hpp).
#pragma once

#include "gpjson/file/file.hpp"

#include <cstddef>
#include <ostream>
#include <string>
#include <vector>

namespace gpjson::file {

enum class FileReaderType { COPIED = 0, MMAP };

std::ostream &operator<<(std::ostream &os, FileReaderType type);

struct FileReaderOptions {
  FileReaderType file_reader_type{FileReaderType::COPIED};
};

std::ostream &operator<<(std::ostream &os, const FileReaderOptions &options);

class FileReader {
 public:
  virtual ~FileReader() = default;
  virtual void create_partitions(size_t partition_size_bytes) = 0;
  virtual std::vector<FilePartition> &get_partitions() = 0;
  virtual const std::vector<FilePartition> &get_partitions() const = 0;
  virtual const FileMetadata &metadata() const = 0;

 protected:
  FileReader() = default;
};

class CopiedFileReader final : public FileReader {
 public:
  explicit CopiedFileReader(std::string file_path);
  void create_partitions(size_t partition_size_bytes) override;
  std::vector<FilePartition> &get_partitions() override { return partitions_; }
  const std::vector<FilePartition> &get_partitions() const override { return partitions_; }
  const FileMetadata &metadata() const override { return metadata_; }

 private:
  std::string file_path_;
  FileMetadata metadata_;
  std::vector<unsigned char> bytes_;
  std::vector<FilePartition> partitions_;
};

class MmapFileReader final : public FileReader {
 public:
  explicit MmapFileReader(std::string file_path);
  ~MmapFileReader() override;
  MmapFileReader(const MmapFileReader &) = delete;
  MmapFileReader &operator=(const MmapFileReader &) = delete;
  void create_partitions(size_t partition_size_bytes) override;
  std::vector<FilePartition> &get_partitions() override { return partitions_; }
  const std::vector<FilePartition> &get_partitions() const override { return partitions_; }
  const FileMetadata &metadata() const override { return metadata_; }

 private:
  std::string file_path_;
  FileMetadata metadata_;
  const unsigned char *mapped_ = nullptr;
  size_t mapped_size_ = 0;
  int fd_ = -1;
  std::vector<FilePartition> partitions_;
};

// Splits [0, size) into partitions of at most partition_size bytes that end
// just before a '\n' (the newline itself belongs to no partition); throws
// error::file::PartitionError when a window holds no newline.  Exposed for
// tests.
std::vector<FilePartition> partition_bytes(const std::string &file_path,
                                           const unsigned char *base, size_t size,
                                           size_t partition_size);

}  // namespace gpjson::file
