// gpj_index_build_noalloc: the fused index build for callers that cannot
// allocate device memory.
//
// Some hosts reserve all of a GPU's memory up front and hand out pieces of it
// themselves (a database or serving engine that owns the device memory
// pool); any later cudaMalloc from a plugin fails or fragments their pool.
// Latency-critical loops also avoid cudaMalloc/cudaFree because those calls
// can synchronize the whole device.  Such callers pass every input and output
// buffer themselves; the only other memory the build needs -- one 8-byte
// look-back descriptor per 32 KiB tile plus a few counters -- comes from the
// fixed array below instead of the context's cudaMalloc'd scratch.
//
// The array is a file-scope __device__ object of kNoallocScratchBytes
// (1 MiB + 256 B), enough for inputs of up to kNoallocMaxInputBytes (4 GiB).
// Every GPU that loads this library holds it until the process exits.
#include "indexer.cuh"

#include "gpjson_b200.h"

#include <cuda_runtime.h>

#include <mutex>

namespace gpjb {
int report_error(int code, const char *message);  // capi.cu
}

namespace {

constexpr uint64_t kNoallocMaxTiles = 131072;
constexpr uint64_t kNoallocMaxInputBytes = kNoallocMaxTiles * gpjb::kTileBytes;  // 4 GiB
constexpr uint64_t kNoallocScratchBytes = kNoallocMaxTiles * 8u + 256u;

// Shared by every call on a device: calls whose work overlaps on that GPU
// race on it.  Its contents persist between calls; the build clears the part
// that must start at zero before each launch.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
void *g_scratch_addr[kMaxDevices];  // device address of the array, per device

// The array's name in host code is only a host-side stand-in; the kernels need
// its device address, looked up once per device with that device current.
int scratch_address(void **out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    (void)cudaGetLastError();
    return gpjb::report_error(GPJ_ERR_CUDA, "gpj_index_build_noalloc: no current CUDA device");
  }
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (g_scratch_addr[dev] == nullptr) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      (void)cudaGetLastError();
      return gpjb::report_error(GPJ_ERR_CUDA,
                                "gpj_index_build_noalloc: cudaGetSymbolAddress failed");
    }
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return GPJ_OK;
}

// Summary of an empty partition: one line, NL = [0], outside a string, depth -1.
__global__ void empty_partition_summary(unsigned long long *summary, int64_t *nl,
                                        uint64_t nl_cap) {
  summary[0] = 1ull;
  summary[1] = 0ull;
  summary[2] = ~0ull;
  summary[3] = 0ull;
  if (nl_cap > 0) nl[0] = 0;
}

}  // namespace

extern "C" int gpj_index_build_noalloc(const uint8_t *d_input, uint64_t size_bytes,
                                       int num_levels, uint32_t flags, gpj_index *index,
                                       uint64_t *d_summary, void *stream_) {
  if (index == nullptr || d_summary == nullptr)
    return gpjb::report_error(GPJ_ERR_INVALID_ARGUMENT,
                              "gpj_index_build_noalloc: index and d_summary are required");
  if (num_levels < 0 || num_levels > GPJ_MAX_LEVELS)
    return gpjb::report_error(GPJ_ERR_INVALID_ARGUMENT,
                              "gpj_index_build_noalloc: num_levels must be in [0, 22]");
  if (size_bytes > kNoallocMaxInputBytes)
    return gpjb::report_error(GPJ_ERR_CAPACITY,
                              "gpj_index_build_noalloc: input larger than 4 GiB (4294967296 "
                              "bytes), the size of its fixed scratch; use gpj_index_build_async");
  const uint64_t W = (size_bytes + 63u) / 64u;
  if (size_bytes > 0 && d_input == nullptr)
    return gpjb::report_error(GPJ_ERR_INVALID_ARGUMENT, "gpj_index_build_noalloc: null input");
  if (W > 0 && (index->d_string == nullptr || (num_levels > 0 && index->d_leveled == nullptr)))
    return gpjb::report_error(GPJ_ERR_INVALID_ARGUMENT,
                              "gpj_index_build_noalloc: missing output buffers");
  const bool eq = (flags & GPJ_INDEX_EMIT_ESCAPE_QUOTE) != 0;
  if (eq && W > 0 && (index->d_escape == nullptr || index->d_quote == nullptr))
    return gpjb::report_error(GPJ_ERR_INVALID_ARGUMENT,
                              "gpj_index_build_noalloc: escape/quote buffers required");

  void *scratch = nullptr;
  int rc = scratch_address(&scratch);
  if (rc != GPJ_OK) return rc;
  auto stream = static_cast<cudaStream_t>(stream_);

  index->d_input = d_input;
  index->size_bytes = size_bytes;
  index->num_words = W;
  index->num_levels = num_levels;

  if (size_bytes == 0) {
    empty_partition_summary<<<1, 1, 0, stream>>>(
        reinterpret_cast<unsigned long long *>(d_summary), index->d_newline,
        index->newline_capacity);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? GPJ_OK
                            : gpjb::report_error(GPJ_ERR_CUDA, cudaGetErrorString(e));
  }

  gpjb::IndexLaunch L;
  L.single.n = size_bytes;
  L.single.levels = num_levels;
  L.num_levels = num_levels;
  L.full_rows = size_bytes / 128u;
  L.S = index->d_string;
  L.LB = index->d_leveled;
  L.E = eq ? index->d_escape : nullptr;
  L.Q = eq ? index->d_quote : nullptr;
  L.NL = index->d_newline;
  L.nl_cap = index->newline_capacity;
  L.num_tiles = uint32_t(gpjb::index_num_tiles(size_bytes));
  L.in = d_input;
  gpjb::index_bind_scratch(L, scratch);

  // Unaligned inputs take the plain-load staging path (TMA needs 16-byte
  // aligned rows and there is no room to copy the input).
  CUtensorMap map;
  bool tma = false;
  if ((flags & GPJ_INDEX_NO_TMA) == 0) tma = gpjb::index_make_tensor_map(&map, d_input, size_bytes);

  // index_launch clears the descriptors and counters before the kernel.
  cudaError_t e = gpjb::index_launch(L, tma ? &map : nullptr, tma, stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_summary, L.summary, 24, cudaMemcpyDeviceToDevice, stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_summary + 3, 0, 8, stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_summary + 3, L.error, 4, cudaMemcpyDeviceToDevice, stream);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    return gpjb::report_error(GPJ_ERR_CUDA, cudaGetErrorString(e));
  }
  return GPJ_OK;
}
