// Self-test of the tcgen05 path: one 128-row tile D = A * B^T with operands staged in shared
// memory in the canonical layouts of umma.cuh (A and B each K-major or MN-major), FP32
// accumulation in TMEM and a tcgen05.ld epilogue. The guiding network's kernels are built from
// exactly these pieces; the GPU test compares this tile against an FP32 matmul.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <string>

#include "../../include/toaster_cuda.h"
#include "umma.cuh"

namespace tcb {

constexpr int kSelfTestMaxK = 80;
constexpr int kSelfTestMaxN = 128;
constexpr int kSelfTestSmem = 128 * 1024;

// Byte offset of (row, k) in a layout whose row-dimension 8-groups are `row_group` bytes apart
// and K 8-groups `k_group` bytes apart; K-major puts 8 K values in one 16-byte row, MN-major
// 8 rows.
__device__ __forceinline__ uint32_t canon_offset(uint32_t row, uint32_t k, bool mn_major, uint32_t row_group,
                                                 uint32_t k_group) {
  if (!mn_major) return (row >> 3) * row_group + (k >> 3) * k_group + (row & 7u) * 16u + (k & 7u) * 2u;
  return (row >> 3) * row_group + (k >> 3) * k_group + (k & 7u) * 16u + (row & 7u) * 2u;
}

__global__ void __launch_bounds__(128) umma_selftest_kernel(const __nv_bfloat16* __restrict__ a,
                                                            const __nv_bfloat16* __restrict__ b, float* __restrict__ d,
                                                            int n, int k, int a_mn, int b_mn, int* status) {
  // Operands sit in a generous dynamic allocation (kSelfTestSmem) so that every descriptor read
  // of the 128 x K and N x K tiles stays inside the CTA's shared memory whatever the strides.
  extern __shared__ __align__(1024) unsigned char smem[];
  __nv_bfloat16* sa = reinterpret_cast<__nv_bfloat16*>(smem);
  __nv_bfloat16* sb = reinterpret_cast<__nv_bfloat16*>(smem + kSelfTestSmem / 2);
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x, warp = tid >> 5;

  // Strides: K-major operands keep K groups adjacent (128 B) and row groups k/8 * 128 B apart;
  // MN-major operands keep row groups adjacent (128 B) and K groups rows/8 * 128 B apart.
  const uint32_t a_row_group = a_mn ? 128u : uint32_t(k / 8) * 128u;
  const uint32_t a_k_group = a_mn ? 128u * 16u : 128u;  // 128 rows / 8 = 16 row groups
  const uint32_t b_row_group = b_mn ? 128u : uint32_t(k / 8) * 128u;
  const uint32_t b_k_group = b_mn ? uint32_t(n / 8) * 128u : 128u;
  char* pa = reinterpret_cast<char*>(sa);
  char* pb = reinterpret_cast<char*>(sb);
  for (int i = tid; i < 128 * k; i += 128) {
    const int r = i / k, c = i % k;
    *reinterpret_cast<__nv_bfloat16*>(pa + canon_offset(r, c, a_mn, a_row_group, a_k_group)) = a[i];
  }
  for (int i = tid; i < n * k; i += 128) {
    const int r = i / k, c = i % k;
    *reinterpret_cast<__nv_bfloat16*>(pb + canon_offset(r, c, b_mn, b_row_group, b_k_group)) = b[i];
  }
  if (warp == 0) umma::tmem_alloc(&tmem_base, 128);
  if (tid == 0) umma::mbar_init(&mbar, 1);
  umma::fence_async_smem();
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = tmem_base;
  if (tid == 0) {
    const uint32_t idesc = umma::idesc_bf16_f32(128, n, a_mn != 0, b_mn != 0);
    // In both layouts one K = 16 step spans two K groups: the LBO is the K-group stride and the
    // SBO the row-group stride.
    for (int kk = 0; kk < k / 16; ++kk) {
      const uint64_t da = umma::smem_desc(umma::smem_addr(pa + 2 * kk * a_k_group), a_k_group, a_row_group);
      const uint64_t db = umma::smem_desc(umma::smem_addr(pb + 2 * kk * b_k_group), b_k_group, b_row_group);
      umma::mma_bf16(tmem, da, db, idesc, kk > 0 ? 1u : 0u);
    }
    umma::commit(&mbar);
  }
  const bool done = umma::mbar_wait(&mbar, 0);
  if (!done && tid == 0) atomicExch(status, 1);
  umma::fence_after_sync();
  if (done) {
    const uint32_t lane_base = tmem + (uint32_t(warp * 32) << 16);
    const int row = warp * 32 + (tid & 31);
    for (int c = 0; c < n; c += 16) {
      float v[16];
      umma::tmem_ld16(lane_base + uint32_t(c), v);
      umma::tmem_wait_ld();
      for (int j = 0; j < 16; ++j) d[row * n + c + j] = v[j];
    }
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem, 128);
}

}  // namespace tcb

extern "C" int tc_umma_selftest(const uint16_t* a, const uint16_t* b, float* d, int n, int k, int a_mn_major,
                                int b_mn_major) {
  if (!a || !b || !d || n < 16 || n > tcb::kSelfTestMaxN || n % 16 || k < 16 || k > tcb::kSelfTestMaxK || k % 16)
    return TC_ERR_INVALID;
  void *da = nullptr, *db = nullptr, *dd = nullptr, *ds = nullptr;
  int status = 0;
  cudaError_t e = cudaSuccess;
  do {
    if ((e = cudaMalloc(&da, size_t(128) * k * 2)) != cudaSuccess) break;
    if ((e = cudaMalloc(&db, size_t(n) * k * 2)) != cudaSuccess) break;
    if ((e = cudaMalloc(&dd, size_t(128) * n * 4)) != cudaSuccess) break;
    if ((e = cudaMalloc(&ds, sizeof(int))) != cudaSuccess) break;
    if ((e = cudaMemset(ds, 0, sizeof(int))) != cudaSuccess) break;
    if ((e = cudaMemcpy(da, a, size_t(128) * k * 2, cudaMemcpyHostToDevice)) != cudaSuccess) break;
    if ((e = cudaMemcpy(db, b, size_t(n) * k * 2, cudaMemcpyHostToDevice)) != cudaSuccess) break;
    if ((e = cudaFuncSetAttribute(tcb::umma_selftest_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  tcb::kSelfTestSmem)) != cudaSuccess)
      break;
    tcb::umma_selftest_kernel<<<1, 128, tcb::kSelfTestSmem>>>(static_cast<const __nv_bfloat16*>(da), static_cast<const __nv_bfloat16*>(db),
                                          static_cast<float*>(dd), n, k, a_mn_major, b_mn_major, static_cast<int*>(ds));
    if ((e = cudaGetLastError()) != cudaSuccess) break;
    if ((e = cudaMemcpy(d, dd, size_t(128) * n * 4, cudaMemcpyDeviceToHost)) != cudaSuccess) break;
    if ((e = cudaMemcpy(&status, ds, sizeof(int), cudaMemcpyDeviceToHost)) != cudaSuccess) break;
  } while (false);
  cudaFree(da);
  cudaFree(db);
  cudaFree(dd);
  cudaFree(ds);
  if (e != cudaSuccess) return TC_ERR_CUDA;
  return status ? TC_ERR_DEVICE_STATUS : TC_OK;
}
