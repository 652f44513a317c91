// Test harness for parity checks (not part of the product): runs the
// reference library, compiled from its own sources into oracle/_ref by
// oracle/ref/build_ref.py, on one input file and writes its outputs as raw
// little-endian int64 arrays.
//
//   ref_dump <input> <builder 0..3> <levels> <out_prefix> [query ...]
//
// writes <out_prefix>.S (string index words), .LB (leveled bitmap words),
// .NL (newline index, num_lines entries), .E and .Q (escape and quote
// bitmap words from the SHAREMEM escape_carry_index -> escape_index ->
// quote_index kernels, which the builders keep internal) and, per query q,
// .R<q> (int64
// [lines][slots][2], partition-local [start, end), -1 where a slot matched
// nothing), built with IndexBuilderType <builder> (0 UNCOMBINED, 1 COMBINED,
// 2 FUSED, 3 SHAREMEM) and <levels> leveled-bitmap levels (at least the
// queries' depth).  With REF_TIME_REPS=n set it also times n index builds
// and n query batches with CUDA events and prints "ms_index <x> ms_query <y>".
//
// Launch options: block 512 and enough threads that each thread's chunk is
// one 64-byte word (the configuration under which the reference's escape
// carry is word-local, as in its benchmark configs for inputs up to 1 GiB).
#include "gpjson/engine.hpp"
#include "gpjson/file/file.hpp"
#include "gpjson/file/file_reader.hpp"
#include "gpjson/index/index_builder.hpp"
#include "gpjson/index/kernels/sharemem.cuh"
#include "gpjson/profiler/profiler.hpp"
#include "gpjson/query/query_compiler.hpp"
#include "gpjson/query/query_executor.hpp"
#include "gpjson/run_context.hpp"

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

using namespace gpjson;

static void write_raw(const std::string &path, const std::vector<int64_t> &v) {
  std::ofstream out(path, std::ios::binary);
  out.write(reinterpret_cast<const char *>(v.data()), std::streamsize(v.size() * 8));
}

static std::vector<int64_t> device_words(const index::Index &ix) {
  std::vector<int64_t> v(ix.size_bytes() / 8);
  if (!v.empty()) cudaMemcpy(v.data(), ix.data(), v.size() * 8, cudaMemcpyDeviceToHost);
  return v;
}

static std::unique_ptr<index::IndexBuilder> make_builder(int type, const file::FileReader &r) {
  switch (type) {
  case 0: return std::make_unique<index::UncombinedIndexBuilder>(r);
  case 1: return std::make_unique<index::CombinedIndexBuilder>(r);
  case 2: return std::make_unique<index::FusedIndexBuilder>(r);
  default: return std::make_unique<index::SharememIndexBuilder>(r);
  }
}

int main(int argc, char **argv) {
  if (argc < 5) {
    std::cerr << "usage: ref_dump <input> <builder 0..3> <levels> <out_prefix> [query ...]\n";
    return 2;
  }
  try {
    const std::string input = argv[1];
    const int builder_type = std::atoi(argv[2]);
    const size_t levels = size_t(std::atoi(argv[3]));
    const std::string prefix = argv[4];
    std::vector<std::string> queries(argv + 5, argv + argc);

    file::CopiedFileReader reader(input);
    reader.create_partitions(0);  // partition size 0: the whole file as one partition
    const size_t n = reader.metadata().file_size_bytes;
    file::FilePartition &part = reader.get_partitions().at(0);
    part.load_to_device();

    EngineOptions opts;
    const size_t words = (n + 63) / 64;
    opts.index_builder_options = index::IndexBuilderOptions{
        index::IndexBuilderType(builder_type), 0, int(words / 512 + 1), 512, 32, 32};
    profiler::Profiler prof("ref_dump");
    RunContext ctx{prof};
    auto builder = make_builder(builder_type, reader);
    index::BuiltIndices built = builder->build(part, levels, opts.index_builder_options, ctx);
    cudaDeviceSynchronize();

    // escape and quote bitmaps: the first three kernels of the SHAREMEM
    // string index (sharemem_index_builder.cu:360-380, 219-229), one thread
    // per 64-byte word, block 512
    {
      const int block = 512, grid = int(words / 512 + 1);
      const size_t threads = size_t(grid) * size_t(block);
      char *carry = nullptr, *qcarry = nullptr;
      long *E = nullptr, *Q = nullptr;
      cudaMalloc(&carry, threads);
      cudaMalloc(&qcarry, threads);
      cudaMalloc(&E, threads * sizeof(long));
      cudaMalloc(&Q, threads * sizeof(long));
      cudaMemset(E, 0, threads * sizeof(long));
      cudaMemset(Q, 0, threads * sizeof(long));
      const char *file = static_cast<const char *>(part.device_bytes());
      index::kernels::sharemem::escape_carry_index<<<grid, block>>>(file, n, carry);
      index::kernels::sharemem::escape_index<<<grid, block>>>(file, n, carry, E);
      index::kernels::sharemem::quote_index<<<grid, block>>>(file, n, E, Q, qcarry);
      const cudaError_t e = cudaDeviceSynchronize();
      if (e != cudaSuccess) throw std::runtime_error(cudaGetErrorString(e));
      std::vector<int64_t> hE(words), hQ(words);
      if (words) {
        cudaMemcpy(hE.data(), E, words * 8, cudaMemcpyDeviceToHost);
        cudaMemcpy(hQ.data(), Q, words * 8, cudaMemcpyDeviceToHost);
      }
      write_raw(prefix + ".E", hE);
      write_raw(prefix + ".Q", hQ);
      cudaFree(carry);
      cudaFree(qcarry);
      cudaFree(E);
      cudaFree(Q);
    }
    write_raw(prefix + ".S", device_words(built.get_string_index()));
    write_raw(prefix + ".LB", device_words(built.get_leveled_bitmap_index()));
    std::vector<int64_t> nl = device_words(built.get_newline_index());
    nl.resize(size_t(built.get_newline_index().num_lines()));
    write_raw(prefix + ".NL", nl);

    query::QueryCompiler compiler(opts);
    query::BatchCompiledQuery batch;
    for (const auto &q : queries) batch.add(compiler.compile(q, opts));
    query::QueryExecutor executor(opts);
    if (!queries.empty()) {
      const query::BatchQueryResult res = executor.execute_batch(batch, part, built);
      for (size_t q = 0; q < res.queries().size(); ++q) {
        std::vector<int64_t> out;
        for (const auto &line : res.queries()[q].lines())
          for (const auto &o : line.offsets()) {
            out.push_back(o.start ? int64_t(*o.start - part.global_start_offset()) : -1);
            out.push_back(o.end ? int64_t(*o.end - part.global_start_offset()) : -1);
          }
        write_raw(prefix + ".R" + std::to_string(q), out);
      }
    }

    if (const char *reps_env = std::getenv("REF_TIME_REPS")) {
      const int reps = std::atoi(reps_env);
      cudaEvent_t e0, e1, e2;
      cudaEventCreate(&e0);
      cudaEventCreate(&e1);
      cudaEventCreate(&e2);
      float t_index = 0, t_query = 0;
      for (int r = 0; r < reps; ++r) {
        cudaEventRecord(e0);
        index::BuiltIndices b = builder->build(part, levels, opts.index_builder_options, ctx);
        cudaEventRecord(e1);
        if (!queries.empty()) (void)executor.execute_batch(batch, part, b);
        cudaEventRecord(e2);
        cudaEventSynchronize(e2);
        float a = 0, c = 0;
        cudaEventElapsedTime(&a, e0, e1);
        cudaEventElapsedTime(&c, e1, e2);
        t_index += a;
        t_query += c;
      }
      std::printf("ms_index %.4f ms_query %.4f\n", t_index / reps, t_query / reps);
    }
  } catch (const std::exception &e) {
    std::cerr << "ref_dump: " << e.what() << "\n";
    return 1;
  }
  return 0;
}
