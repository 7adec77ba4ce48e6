// Cache read-bandwidth probe: the denominator of the path kernel's roofline on scenes whose
// hierarchy, primitives and sampling tables stay resident in L2 (every benchmark scene but the
// 2.1 M-triangle mesh). Every SM streams a buffer with 16-byte loads that bypass L1
// (ld.global.cg), so a buffer smaller than L2 measures L2 read bandwidth and a larger one HBM.
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/toaster_cuda.h"

namespace tcb {

__global__ void __launch_bounds__(256) cache_read_kernel(const uint4* __restrict__ buf, size_t n16, int passes,
                                                         unsigned int* __restrict__ sink) {
  uint32_t acc = 0;
  const size_t stride = size_t(gridDim.x) * blockDim.x;
  const size_t first = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  for (int p = 0; p < passes; ++p) {
    size_t i = first;
    // Four independent 16-byte loads in flight per thread per iteration.
    for (; i + 3 * stride < n16; i += 4 * stride) {
      const uint4 a = __ldcg(buf + i), b = __ldcg(buf + i + stride), c = __ldcg(buf + i + 2 * stride),
                  d = __ldcg(buf + i + 3 * stride);
      acc ^= (a.x ^ a.y ^ a.z ^ a.w) + (b.x ^ b.y ^ b.z ^ b.w) + (c.x ^ c.y ^ c.z ^ c.w) + (d.x ^ d.y ^ d.z ^ d.w);
    }
    for (; i < n16; i += stride) {
      const uint4 a = __ldcg(buf + i);
      acc ^= a.x ^ a.y ^ a.z ^ a.w;
    }
  }
  // The buffer is zero-filled, so acc is 0; the store keeps the loads from being removed.
  if (acc == 0x9E3779B9u) atomicAdd(sink, 1u);
}

}  // namespace tcb

namespace {
thread_local std::string g_probe_error;
}

extern "C" {

int tc_probe_cache_read(int device_ordinal, size_t bytes, int passes, double* gb_per_s) {
  if (!gb_per_s || passes <= 0 || bytes < (1u << 20)) {
    g_probe_error = "tc_probe_cache_read needs a result pointer, passes > 0 and at least 1 MiB";
    return TC_ERR_INVALID;
  }
  *gb_per_s = 0.0;
  cudaError_t e = cudaSetDevice(device_ordinal);
  int sm = 0;
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, device_ordinal);
  void* buf = nullptr;
  unsigned int* sink = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  const size_t n16 = bytes / 16;
  if (e == cudaSuccess) e = cudaMalloc(&buf, n16 * 16);
  if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&sink), sizeof(unsigned int));
  if (e == cudaSuccess) e = cudaMemset(buf, 0, n16 * 16);
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  float ms = 0.0f;
  if (e == cudaSuccess) {
    const int grid = sm * 8;
    // One untimed pass brings the buffer into L2 (when it fits), then the timed passes.
    tcb::cache_read_kernel<<<grid, 256>>>(static_cast<const uint4*>(buf), n16, 1, sink);
    cudaEventRecord(e0);
    tcb::cache_read_kernel<<<grid, 256>>>(static_cast<const uint4*>(buf), n16, passes, sink);
    cudaEventRecord(e1);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (buf) cudaFree(buf);
  if (sink) cudaFree(sink);
  if (e != cudaSuccess) {
    g_probe_error = std::string("cache read probe: ") + cudaGetErrorString(e);
    return TC_ERR_CUDA;
  }
  *gb_per_s = double(n16) * 16.0 * passes / (double(ms) * 1e-3) / 1e9;
  return TC_OK;
}

const char* tc_probe_last_error(void) { return g_probe_error.c_str(); }

}  // extern "C"
