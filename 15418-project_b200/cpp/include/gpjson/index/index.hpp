// Device-resident structural indexes, RAII and move-only (interface of the
// reference's include/gpjson/index/index.hpp).
#pragma once

#include "gpjson/cuda/cuda.hpp"

#include <utility>

namespace gpjson::index {

class Index {
 public:
  Index() = default;
  virtual ~Index() = default;
  Index(Index &) = delete;
  Index &operator=(Index &) = delete;
  Index(Index &&) noexcept = default;
  Index &operator=(Index &&) noexcept = default;
  void *data() { return data_.data(); }
  const void *data() const { return data_.data(); }
  size_t size_bytes() const { return data_.size_bytes(); }

 protected:
  explicit Index(cuda::DeviceArray data) : data_(std::move(data)) {}
  cuda::DeviceArray data_;
};

class NewlineIndex final : public Index {
 public:
  NewlineIndex() = default;
  NewlineIndex(cuda::DeviceArray data, int num_lines)
      : Index(std::move(data)), num_lines_(num_lines) {}
  NewlineIndex(NewlineIndex &&) noexcept = default;
  NewlineIndex &operator=(NewlineIndex &&) noexcept = default;
  int num_lines() const { return num_lines_; }

 private:
  int num_lines_ = 0;
};

class StringIndex final : public Index {
 public:
  StringIndex() = default;
  explicit StringIndex(cuda::DeviceArray data) : Index(std::move(data)) {}
  StringIndex(StringIndex &&) noexcept = default;
  StringIndex &operator=(StringIndex &&) noexcept = default;
};

class LeveledBitmapIndex final : public Index {
 public:
  LeveledBitmapIndex() = default;
  LeveledBitmapIndex(cuda::DeviceArray data, int num_levels)
      : Index(std::move(data)), num_levels_(num_levels) {}
  LeveledBitmapIndex(LeveledBitmapIndex &&) noexcept = default;
  LeveledBitmapIndex &operator=(LeveledBitmapIndex &&) noexcept = default;
  int num_levels() const { return num_levels_; }

 private:
  int num_levels_ = 0;
};

class BuiltIndices {
 public:
  BuiltIndices() = default;
  BuiltIndices(NewlineIndex nl, StringIndex s, LeveledBitmapIndex lb)
      : newline_(std::move(nl)), string_(std::move(s)), leveled_(std::move(lb)) {}
  BuiltIndices(BuiltIndices &&) noexcept = default;
  BuiltIndices &operator=(BuiltIndices &&) noexcept = default;
  BuiltIndices(const BuiltIndices &) = delete;
  BuiltIndices &operator=(const BuiltIndices &) = delete;
  const NewlineIndex &get_newline_index() const { return newline_; }
  const StringIndex &get_string_index() const { return string_; }
  const LeveledBitmapIndex &get_leveled_bitmap_index() const { return leveled_; }

 private:
  NewlineIndex newline_;
  StringIndex string_;
  LeveledBitmapIndex leveled_;
};

}  // namespace gpjson::index
