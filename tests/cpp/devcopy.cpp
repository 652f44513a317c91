// Device-to-host copy helper of the C++ API tests.
#include <cuda_runtime_api.h>
#include <cstddef>
int cudaMemcpy_host(void *dst, const void *src, size_t n) {
  return int(cudaMemcpy(dst, src, n, cudaMemcpyDeviceToHost));
}
