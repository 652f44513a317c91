// Wall-clock segment profiler.  Prints "<name>: <indent><segment>: X.XXX ms"
// when a segment ends -- the line format the reference's eval tooling parses.
#pragma once

#include <chrono>
#include <cstddef>
#include <string>
#include <vector>

namespace gpjson::profiler {

class Profiler {
 public:
  class SegmentId {
   public:
    SegmentId() = default;

   private:
    friend class Profiler;
    explicit SegmentId(size_t index) : index_(index), valid_(true) {}
    size_t index_ = 0;
    bool valid_ = false;
  };

  explicit Profiler(std::string name);
  SegmentId begin(const std::string &segment);
  SegmentId begin_nested(const std::string &segment);
  SegmentId beginf(const char *fmt, ...);
  SegmentId begin_nestedf(const char *fmt, ...);
  void end(SegmentId id);

 private:
  struct Record {
    std::string name;
    std::chrono::steady_clock::time_point start;
    size_t indent = 0;
    bool opens_scope = false;
    bool done = false;
  };
  SegmentId open(std::string segment, bool nested);

  std::string name_;
  std::vector<Record> records_;
  size_t indent_ = 0;
};

}  // namespace gpjson::profiler
