// C++ API tests of the engine (mirrors the reference's gtest suites: engine
// integration, query executor, index builders for every builder type,
// compiler shapes and rejections, DeviceArray, partitioning).  Fixtures come
// from files whose paths tests/test_cpp_api_gpu.py passes on the command line:
//   argv[1] ld_json fixture, argv[2] bookstore record, argv[3] scratch dir.
#include "gpjson/engine.hpp"
#include "gpjson/error/error.hpp"
#include "gpjson/file/file_reader.hpp"
#include "gpjson/index/index_builder.hpp"

#include <cstdint>
#include <cstdio>
#include <fstream>
#include <functional>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

using namespace gpjson;

static int failures = 0;
#define CHECK(cond)                                                                   \
  do {                                                                                \
    if (!(cond)) throw std::runtime_error(std::string("check failed: ") + #cond);     \
  } while (0)

static void run(const char *name, const std::function<void()> &fn) {
  try {
    fn();
    std::cout << "PASS " << name << "\n";
  } catch (const std::exception &e) {
    ++failures;
    std::cout << "FAIL " << name << ": " << e.what() << "\n";
  }
}

static std::string slurp(const std::string &p) {
  std::ifstream in(p, std::ios::binary);
  std::stringstream ss;
  ss << in.rdbuf();
  return ss.str();
}

// Expected values restated from the reference tests' helpers
// (tests/index/{newline,string,leveled_bitmap}_index_test.cpp).
static std::vector<long> expect_newlines(const std::string &d) {
  std::vector<long> v{0};
  for (size_t i = 0; i < d.size(); ++i)
    if (d[i] == '\n') v.push_back(long(i));
  return v;
}
static bool escaped_quote(const std::string &d, size_t q) {
  size_t k = 0;
  for (size_t i = q; i > 0 && d[i - 1] == '\\'; --i) ++k;
  return k % 2 == 1;
}
static std::vector<uint64_t> expect_string(const std::string &d) {
  std::vector<uint64_t> w((d.size() + 63) / 64, 0);
  bool in = false;
  for (size_t i = 0; i < d.size(); ++i) {
    if (d[i] == '"' && !escaped_quote(d, i)) {
      if (!in) w[i / 64] |= uint64_t(1) << (i % 64);
      in = !in;
    } else if (in) {
      w[i / 64] |= uint64_t(1) << (i % 64);
    }
  }
  return w;
}
static std::vector<uint64_t> expect_leveled(const std::string &d, int L) {
  const size_t W = (d.size() + 63) / 64;
  auto s = expect_string(d);
  std::vector<uint64_t> lv(W * L, 0);
  int level = -1;
  for (size_t i = 0; i < d.size(); ++i) {
    const uint64_t bit = uint64_t(1) << (i % 64);
    if (s[i / 64] & bit) continue;
    const char c = d[i];
    if (c == '{' || c == '[') {
      ++level;
      if (level >= 0 && level < L) lv[W * level + i / 64] |= bit;
    } else if (c == '}' || c == ']') {
      if (level >= 0 && level < L) lv[W * level + i / 64] |= bit;
      --level;
    } else if (c == ':' || c == ',') {
      if (level >= 0 && level < L) lv[W * level + i / 64] |= bit;
    }
  }
  return lv;
}

int cudaMemcpy_host(void *dst, const void *src, size_t n);  // devcopy.cpp

template <class T>
static std::vector<T> to_host(const index::Index &ix) {
  std::vector<T> v(ix.size_bytes() / sizeof(T));
  if (!v.empty()) cuda::check(cudaMemcpy_host(v.data(), ix.data(), ix.size_bytes()), "copy index");
  return v;
}

int main(int argc, char **argv) {
  if (argc < 4) {
    std::cerr << "usage: api_test LD_FIXTURE BOOKSTORE SCRATCH_DIR\n";
    return 2;
  }
  const std::string ld = slurp(argv[1]);
  const std::string book = slurp(argv[2]);
  const std::string dir = argv[3];
  EngineOptions defaults{};

  run("DeviceArrayRoundTripAndMove", [] {
    cuda::DeviceArray a(16);
    const char src[16] = "0123456789abcde";
    a.copy_from_host(src, 16);
    cuda::DeviceArray b(std::move(a));
    CHECK(a.data() == nullptr && a.size_bytes() == 0 && b.size_bytes() == 16);
    char dst[16] = {};
    b.copy_to_host(dst, 16);
    CHECK(std::string(dst, 15) == "0123456789abcde");
    b.memset(0);
    b.copy_to_host(dst, 16);
    CHECK(dst[3] == 0);
    bool threw = false;
    try {
      b.copy_to_host(dst, 17);
    } catch (const error::cuda::CudaError &) {
      threw = true;
    }
    CHECK(threw);
  });

  run("PartitionsEndBeforeNewlines", [] {
    const std::string s = "aa\nbbb\ncccc\nd";
    auto p = file::partition_bytes("mem", reinterpret_cast<const unsigned char *>(s.data()),
                                   s.size(), 5);
    CHECK(p.size() == 4);
    CHECK(p[0].global_start_offset() == 0 && p[0].global_end_offset() == 2);
    CHECK(p[1].global_start_offset() == 3 && p[1].global_end_offset() == 6);
    CHECK(p[3].global_start_offset() == 12 && p[3].global_end_offset() == 13);
    bool threw = false;
    try {
      const std::string t = "abcdefgh\nx";
      file::partition_bytes("mem", reinterpret_cast<const unsigned char *>(t.data()), t.size(), 3);
    } catch (const error::file::PartitionError &) {
      threw = true;
    }
    CHECK(threw);
  });

  run("CompilerShapesAndRejections", [&] {
    query::QueryCompiler c(defaults);
    auto q = c.compile("$.arr[0:2]", defaults);
    CHECK(q.max_depth() == 2 && q.num_result_slots() == 2 && q.ir_bytes().size() == 16);
    bool a = false, b = false;
    try {
      c.compile("$..name", defaults);
    } catch (const error::query::UnsupportedQueryError &) {
      a = true;
    }
    try {
      c.compile("$.arr[-0]", defaults);
    } catch (const error::query::MalformedQueryError &) {
      b = true;
    }
    CHECK(a && b);
  });

  for (auto type : {index::IndexBuilderType::UNCOMBINED, index::IndexBuilderType::COMBINED,
                    index::IndexBuilderType::FUSED, index::IndexBuilderType::SHAREMEM,
                    index::IndexBuilderType::B200}) {
    std::ostringstream name;
    name << "BuildsIndexes/" << type;
    run(name.str().c_str(), [&] {
      file::FilePartition part(0, 0, ld.size(), ld.data());
      part.load_to_device();
      file::CopiedFileReader reader("in-memory.ldjson");
      index::B200IndexBuilder builder(reader);
      profiler::Profiler prof("test profiler");
      RunContext rc{prof};
      index::IndexBuilderOptions opts{type, 0, 1, 512, 1, 64};
      auto built = builder.build(part, 8, opts, rc);
      CHECK(built.get_newline_index().num_lines() == int(expect_newlines(ld).size()));
      CHECK(to_host<long>(built.get_newline_index()) == expect_newlines(ld));
      CHECK(to_host<uint64_t>(built.get_string_index()) == expect_string(ld));
      CHECK(built.get_leveled_bitmap_index().num_levels() == 8);
      CHECK(to_host<uint64_t>(built.get_leveled_bitmap_index()) == expect_leveled(ld, 8));
    });
  }

  run("ExecutorReferenceKnownAnswers", [&] {
    file::FilePartition part(0, 0, book.size(), book.data());
    part.load_to_device();
    file::CopiedFileReader reader("in-memory.json");
    index::B200IndexBuilder builder(reader);
    profiler::Profiler prof("test profiler");
    RunContext rc{prof};
    EngineOptions opts{};
    opts.query_executor_options.grid_size = 7;
    opts.query_executor_options.block_size = 32;
    query::QueryCompiler c(opts);
    query::BatchCompiledQuery batch;
    batch.add(c.compile("$.expensive", opts));
    batch.add(c.compile("$.store.book[1].author", opts));
    batch.add(c.compile("$.store.magazine", opts));
    auto built = builder.build(part, batch.get_max_depth(), opts.index_builder_options, rc);
    query::QueryExecutor ex(opts);
    auto res = ex.execute_batch(batch, part, built);
    auto mat = res.materialize();
    CHECK(res.num_queries() == 3 && res.queries()[0].lines().size() == 1);
    CHECK(mat.queries()[0].query_text() == "$.expensive");
    CHECK(mat.queries()[0].lines().size() == 1);
    CHECK(mat.queries()[0].lines()[0].values()[0].json_text() == "\"10\"");
    CHECK(mat.queries()[1].lines()[0].values()[0].json_text() == "\"Herman Melville\"");
    CHECK(mat.queries()[2].lines().empty());
  });

  run("LoadToDeviceIsIdempotent", [] {
    const std::string j = R"({"id":1})";
    file::FilePartition p(0, 0, j.size(), j.data());
    CHECK(!p.device_loaded());
    p.load_to_device();
    const void *d = p.device_bytes();
    CHECK(d != nullptr && p.device_loaded());
    p.load_to_device();
    CHECK(p.device_bytes() == d);
  });

  auto engine_case = [&](file::FileReaderType rt, index::IndexBuilderType bt, const char *fname) {
    const std::string path = dir + "/" + fname;
    {
      std::ofstream o(path, std::ios::binary);
      o << "{\"name\":\"Ada\",\"scores\":[1,2],\"lang\":\"en\"}\n"
        << "{\"name\":\"Bob\",\"scores\":[3,4],\"lang\":\"fr\"}\n";
    }
    EngineOptions opts{file::FileReaderOptions{rt}, index::IndexBuilderOptions{bt, 43, 1, 64, 1, 64},
                       query::QueryExecutorOptions{512, 1024}};
    Engine e;
    auto r = e.query(path, {"$.name", "$.scores[1]"}, opts);
    CHECK(r.queries().size() == 2);
    CHECK(r.queries()[0].query_text() == "$.name" && r.queries()[0].lines().size() == 2);
    CHECK(r.queries()[0].lines()[0].values()[0].json_text() == "\"Ada\"");
    CHECK(r.queries()[0].lines()[1].values()[0].json_text() == "\"Bob\"");
    CHECK(r.queries()[1].lines().size() == 2);
    CHECK(r.queries()[1].lines()[0].values()[0].json_text() == "2");
    CHECK(r.queries()[1].lines()[1].values()[0].json_text() == "4");
    std::remove(path.c_str());
  };
  run("EnginePartitionedCopied", [&] {
    engine_case(file::FileReaderType::COPIED, index::IndexBuilderType::UNCOMBINED, "e1.ldjson");
  });
  run("EngineMmapCombined", [&] {
    engine_case(file::FileReaderType::MMAP, index::IndexBuilderType::COMBINED, "e2.ldjson");
  });

  std::cout << (failures ? "FAILED " : "ALL PASSED ") << failures << "\n";
  return failures ? 1 : 0;
}
