// Path-guiding network kernels on the 5th-generation tensor cores (tcgen05, sm_100a).
//
//   guide_images_kernel  FP32 master weights -> BF16 canonical K-major images (+ transposes)
//   guide_infer_kernel   persistent: per 128-query tile, encode -> 4 x (tcgen05.mma into TMEM ->
//                        tcgen05.ld epilogue: bias, ReLU, BF16 back to shared memory) -> decode
//                        the 8-lobe vMF mixture
//   guide_train_kernel   fused forward + loss + backward per 128-sample tile: activation
//                        gradients by MMA against the transposed weight images, weight gradients
//                        dW = dZ^T H accumulated in TMEM across all tiles a CTA owns (MN-major
//                        views of the same shared buffers), FP32 atomics once per CTA at the end
//   guide_adam_kernel    Adam on the FP32 master weights
//
// One elected thread issues the MMAs and commits them to an mbarrier; every wait is bounded and
// a timeout is reported through the status word instead of spinning forever. The NumPy
// restatement in oracle/guide_net.py defines the same encoding, network, loss and gradients.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <math_constants.h>

#include "guide.h"
#include "umma.cuh"

namespace tcb {

using umma::kmajor_offset;

// ------------------------------------------------------------------------ weight images
__global__ void guide_images_kernel(const float* __restrict__ p, uint8_t* __restrict__ img, float* __restrict__ biases) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  auto put = [&](uint32_t base, uint32_t off, float v) {
    *reinterpret_cast<__nv_bfloat16*>(img + base + off) = __float2bfloat16_rn(v);
  };
  if (i < 64 * 80) {  // W1 [out][in]
    const int o = i / 80, k = i % 80;
    put(kImgW1, kmajor_offset(o, k, 80), p[kOffW1 + i]);
  }
  if (i < 64 * 64) {
    const int o = i / 64, k = i % 64;
    put(kImgW2, kmajor_offset(o, k, 64), p[kOffW2 + i]);
    put(kImgW3, kmajor_offset(o, k, 64), p[kOffW3 + i]);
    put(kImgW2T, kmajor_offset(k, o, 64), p[kOffW2 + i]);  // row = input, K = output
    put(kImgW3T, kmajor_offset(k, o, 64), p[kOffW3 + i]);
  }
  if (i < 32 * 64) {
    const int o = i / 64, k = i % 64;
    put(kImgW4, kmajor_offset(o, k, 64), p[kOffW4 + i]);
    put(kImgW4T, kmajor_offset(k, o, 32), p[kOffW4 + i]);
  }
  if (i < 64) {
    biases[i] = p[kOffB1 + i];
    biases[64 + i] = p[kOffB2 + i];
    biases[128 + i] = p[kOffB3 + i];
  }
  if (i < 32) biases[192 + i] = p[kOffB4 + i];
}

cudaError_t guide_refresh_images(const GuideDevice& g, cudaStream_t stream) {
  guide_images_kernel<<<(64 * 80 + 255) / 256, 256, 0, stream>>>(g.params, g.images, g.biases);
  return cudaGetLastError();
}

// ------------------------------------------------------------------------ shared pieces
__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&v);
}
// max(lo, 0) and max(hi, 0) rounded to BF16 and packed, in one conversion (the ReLU of the
// hidden layers). The first source operand goes to the upper half.
__device__ __forceinline__ uint32_t pack_relu_bf16x2(float lo, float hi) {
  uint32_t r;
  asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
  return r;
}
__device__ __forceinline__ float tanh_fast(float x) {
  float r;
  asm("tanh.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// Encoding of one query written as row `row` of a K = 80 K-major tile (row-group stride 1280 B).
__device__ void encode_row(uint8_t* tile, int row, bool valid, float px, float py, float pz, float nx, float ny,
                           float nz, const GuideBounds& b) {
  float e[kGuideIn];
  if (valid) {
    const float q[3] = {(px - b.cx) * b.scale, (py - b.cy) * b.scale, (pz - b.cz) * b.scale};
    // Half-octave ladder 2^(k/2), k = 0..11 (1 to about 45 cycles per half scene width): the
    // incident-light field varies at room scale, and finer features only add noise dimensions
    // that a few hundred online steps cannot learn to ignore. The even rungs are doublings of
    // frequency 1 and the odd rungs doublings of frequency sqrt(2), so each axis needs two
    // sin/cos evaluations; the other ten pairs follow from the double-angle identities
    // sin 2x = 2 sin x cos x, cos 2x = 1 - 2 sin^2 x (each doubling at most doubles the absolute
    // error: at most 1.3e-5 after five in FP32 over 2e5 random coordinates, against 2e-3 for the
    // BF16 rounding of the encoded values).
#pragma unroll
    for (int a = 0; a < 3; ++a) {
#pragma unroll
      for (int chain = 0; chain < 2; ++chain) {
        float sn, cs;
        sincospif(q[a] * (chain ? 1.41421356f : 1.0f), &sn, &cs);
#pragma unroll
        for (int k = chain; k < kGuideFreqs; k += 2) {
          e[24 * a + 2 * k] = sn;
          e[24 * a + 2 * k + 1] = cs;
          const float s2 = 2.0f * sn * cs;
          cs = 1.0f - 2.0f * sn * sn;
          sn = s2;
        }
      }
    }
    e[72] = nx; e[73] = ny; e[74] = nz;
#pragma unroll
    for (int k = 75; k < 80; ++k) e[k] = 0.0f;
  } else {
#pragma unroll
    for (int k = 0; k < 80; ++k) e[k] = 0.0f;
  }
#pragma unroll
  for (int g = 0; g < 10; ++g) {
    uint4 v;
    v.x = pack_bf16x2(e[8 * g + 0], e[8 * g + 1]);
    v.y = pack_bf16x2(e[8 * g + 2], e[8 * g + 3]);
    v.z = pack_bf16x2(e[8 * g + 4], e[8 * g + 5]);
    v.w = pack_bf16x2(e[8 * g + 6], e[8 * g + 7]);
    *reinterpret_cast<uint4*>(tile + kmajor_offset(row, 8 * g, 80)) = v;
  }
}

// Hidden-layer epilogue: 64 accumulator columns of this thread's row -> bias, ReLU, BF16 -> row
// `row` of a K = 64 K-major tile.
__device__ __forceinline__ void epilogue_hidden(uint32_t lane_tmem, const float* bias, uint8_t* dst, int row) {
#pragma unroll
  for (int c = 0; c < 64; c += 16) {
    float v[16];
    umma::tmem_ld16(lane_tmem + uint32_t(c), v);
    umma::tmem_wait_ld();
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      float r[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) r[j] = v[8 * h + j] + bias[c + 8 * h + j];
      uint4 o;
      o.x = pack_relu_bf16x2(r[0], r[1]);
      o.y = pack_relu_bf16x2(r[2], r[3]);
      o.z = pack_relu_bf16x2(r[4], r[5]);
      o.w = pack_relu_bf16x2(r[6], r[7]);
      *reinterpret_cast<uint4*>(dst + kmajor_offset(row, c + 8 * h, 64)) = o;
    }
  }
}

// One layer: D[tmem] = A (128 x k, K-major, row-group stride k/8*128) * W^T (n x k K-major image).
__device__ __forceinline__ void issue_layer(uint32_t tmem, const uint8_t* a, const uint8_t* w, int k, int n) {
  const uint32_t sbo = uint32_t(k / 8) * 128u;
  const uint32_t idesc = umma::idesc_bf16_f32(128, n, false, false);
  for (int kk = 0; kk < k / 16; ++kk) {
    const uint64_t da = umma::smem_desc(umma::smem_addr(a + kk * 256), 128u, sbo);
    const uint64_t db = umma::smem_desc(umma::smem_addr(w + kk * 256), 128u, sbo);
    umma::mma_bf16(tmem, da, db, idesc, kk > 0 ? 1u : 0u);
  }
}

// Weight-gradient MMA: D[tmem] (+)= dZ^T (out x 128 batch) * H (128 batch x in). Both operands are
// the K-major activation tiles read as MN-major (batch is the reduction dimension). `dz_k` and
// `h_k` are the K extents the tiles were written with; M = 128 over-reads rows beyond `out`,
// whose results are never read.
__device__ __forceinline__ void issue_weight_grad(uint32_t tmem, const uint8_t* dz, int dz_k, const uint8_t* h,
                                                  int h_k, int n_in, bool accumulate) {
  const uint32_t a_lbo = uint32_t(dz_k / 8) * 128u;  // batch-group stride of the dZ tile
  const uint32_t b_lbo = uint32_t(h_k / 8) * 128u;   // batch-group stride of the H tile
  const uint32_t idesc = umma::idesc_bf16_f32(128, n_in, true, true);
  for (int kk = 0; kk < 8; ++kk) {  // 128 batch rows / 16
    const uint64_t da = umma::smem_desc(umma::smem_addr(dz + kk * 2 * a_lbo), a_lbo, 128u);
    const uint64_t db = umma::smem_desc(umma::smem_addr(h + kk * 2 * b_lbo), b_lbo, 128u);
    umma::mma_bf16(tmem, da, db, idesc, (accumulate || kk > 0) ? 1u : 0u);
  }
}

__device__ __forceinline__ void sync_for_mma() {
  umma::fence_async_smem();
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
}

// Mixture decoding (see guide.h): weights softmax(a), kappa = exp(clamp(b)), cos(theta) = tanh(c),
// phi = pi tanh(d).
constexpr float kKappaLo = -2.0f, kKappaHi = 7.0f;

__device__ void decode_mixture(const float* y, float4* out) {
  float amax = y[0];
#pragma unroll
  for (int j = 1; j < 8; ++j) amax = fmaxf(amax, y[4 * j]);
  float w[8], wsum = 0.0f;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    w[j] = __expf(y[4 * j] - amax);
    wsum += w[j];
  }
  const float inv = 1.0f / wsum;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    // Hardware approximations (relative error about 2^-11 for tanh, 2^-21 absolute for sin/cos on
    // [-pi, pi]): the decoded mixture is what both the sampler and its pdf read, so any rounding
    // here changes the proposal distribution, never the estimator's expectation.
    const float kappa = __expf(fminf(fmaxf(y[4 * j + 1], kKappaLo), kKappaHi));
    const float ct = tanh_fast(y[4 * j + 2]);
    const float st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
    float sp, cp;
    __sincosf(3.14159265358979f * tanh_fast(y[4 * j + 3]), &sp, &cp);
    out[j] = make_float4(st * cp, st * sp, ct, kappa);
  }
  out[8] = make_float4(w[0] * inv, w[1] * inv, w[2] * inv, w[3] * inv);
  out[9] = make_float4(w[4] * inv, w[5] * inv, w[6] * inv, w[7] * inv);
}

// ------------------------------------------------------------------------ inference
constexpr int kInferSmem = int(kImgFwdBytes) + 128 * 80 * 2 + 224 * 4;

__global__ void __launch_bounds__(128, 1) guide_infer_kernel(const float4* __restrict__ queries, uint32_t n,
                                                             const uint8_t* __restrict__ img,
                                                             const float* __restrict__ biases, GuideBounds bounds,
                                                             float4* __restrict__ out, int* status,
                                                             const uint32_t* __restrict__ n_dev) {
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t* s_w = smem;
  uint8_t* s_a = smem + kImgFwdBytes;
  float* s_bias = reinterpret_cast<float*>(smem + kImgFwdBytes + 128 * 80 * 2);
  __shared__ __align__(8) uint64_t mbar, mbar_w;
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x, warp = tid >> 5;
  // The weight images and biases arrive by two bulk copies completing on mbar_w.
  if (tid == 0) {
    umma::mbar_init(&mbar, 1);
    umma::mbar_init(&mbar_w, 1);
    umma::fence_mbar_init();
    umma::mbar_arrive_expect_tx(&mbar_w, kImgFwdBytes + 224 * 4);
    umma::bulk_copy_g2s(s_w, img, kImgFwdBytes, &mbar_w);
    umma::bulk_copy_g2s(s_bias, biases, 224 * 4, &mbar_w);
  }
  if (warp == 0) umma::tmem_alloc(&tmem_base, 64);
  sync_for_mma();
  if (!__syncthreads_and(umma::mbar_wait(&mbar_w, 0))) {
    if (tid == 0) atomicExch(status, 1);
    umma::fence_before_sync();
    __syncthreads();
    if (warp == 0) umma::tmem_dealloc(tmem_base, 64);
    return;
  }
  const uint32_t tmem = tmem_base;
  const uint32_t lane_tmem = tmem + (uint32_t(warp * 32) << 16);
  uint32_t phase = 0;
  bool ok = true;
  if (n_dev) n = min(*n_dev, n);
  const uint32_t tiles = (n + 127) / 128;
  for (uint32_t t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
    const uint32_t q = t * 128 + tid;
    const bool valid = q < n;
    float4 p = make_float4(0, 0, 0, 0), nn = p;
    if (valid) {
      p = queries[2 * size_t(q)];
      nn = queries[2 * size_t(q) + 1];
    }
    encode_row(s_a, tid, valid, p.x, p.y, p.z, nn.x, nn.y, nn.z, bounds);
    const int layer_k[4] = {80, 64, 64, 64};
    const uint32_t layer_w[4] = {kImgW1, kImgW2, kImgW3, kImgW4};
    for (int l = 0; l < 4 && ok; ++l) {
      sync_for_mma();
      if (tid == 0) {
        issue_layer(tmem, s_a, s_w + layer_w[l], layer_k[l], l == 3 ? 32 : 64);
        umma::commit(&mbar);
      }
      const bool done = umma::mbar_wait(&mbar, phase);
      phase ^= 1u;
      ok = __syncthreads_and(done) != 0;
      if (!ok) break;
      umma::fence_after_sync();
      if (l < 3) {
        epilogue_hidden(lane_tmem, s_bias + 64 * l, s_a, tid);
      } else {
        float y[32];
        umma::tmem_ld16(lane_tmem, y);
        umma::tmem_ld16(lane_tmem + 16, y + 16);
        umma::tmem_wait_ld();
#pragma unroll
        for (int j = 0; j < 32; ++j) y[j] += s_bias[192 + j];
        if (valid) {
          float4 dec[kGuideDecodedF4];
          decode_mixture(y, dec);
#pragma unroll
          for (int j = 0; j < kGuideDecodedF4; ++j) out[size_t(q) * kGuideDecodedF4 + j] = dec[j];
        }
      }
    }
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
  }
  if (!ok && tid == 0) atomicExch(status, 1);
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem, 64);
}

cudaError_t guide_launch_infer(const GuideDevice& g, const float4* queries, uint32_t n, float4* out, int sm_count,
                               cudaStream_t stream, const uint32_t* n_dev) {
  if (n == 0) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(guide_infer_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kInferSmem);
  if (e != cudaSuccess) return e;
  const uint32_t tiles = (n + 127) / 128;
  const int grid = int(tiles < uint32_t(4 * sm_count) ? tiles : uint32_t(4 * sm_count));
  guide_infer_kernel<<<grid, 128, kInferSmem, stream>>>(queries, n, g.images, g.biases, g.bounds, out, g.status,
                                                         n_dev);
  return cudaGetLastError();
}

// ------------------------------------------------------------------------ loss gradient
// Per-thread loss of one sample and d loss / d y (see oracle/guide_net.py:loss_and_dy).
__device__ float loss_and_grad(const float* y, float ox, float oy, float oz, float scale, float* dy) {
  float amax = y[0];
#pragma unroll
  for (int j = 1; j < 8; ++j) amax = fmaxf(amax, y[4 * j]);
  float w[8], wsum = 0.0f;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    w[j] = expf(y[4 * j] - amax);
    wsum += w[j];
  }
  const float log_wsum = logf(wsum);
  float t[8], kap[8], cosang[8], ct[8], st[8], sp[8], cp[8], thd[8];
  float tmax = -CUDART_INF_F;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    w[j] /= wsum;
    kap[j] = expf(fminf(fmaxf(y[4 * j + 1], kKappaLo), kKappaHi));
    ct[j] = tanhf(y[4 * j + 2]);
    st[j] = sqrtf(fmaxf(0.0f, 1.0f - ct[j] * ct[j]));
    thd[j] = tanhf(y[4 * j + 3]);
    sincospif(thd[j], &sp[j], &cp[j]);
    cosang[j] = st[j] * cp[j] * ox + st[j] * sp[j] * oy + ct[j] * oz;
    const float lv = logf(kap[j]) - logf(2.0f * CUDART_PI_F) - log1pf(-expf(-2.0f * kap[j])) + kap[j] * (cosang[j] - 1.0f);
    t[j] = (y[4 * j] - amax - log_wsum) + lv;
    tmax = fmaxf(tmax, t[j]);
  }
  float se = 0.0f;
#pragma unroll
  for (int j = 0; j < 8; ++j) se += expf(t[j] - tmax);
  const float logq = tmax + logf(se);
  const float g = -scale;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const float r = expf(t[j] - logq);
    dy[4 * j] = g * (r - w[j]);
    const float b = y[4 * j + 1];
    const float dlv = 1.0f / kap[j] - 2.0f / expm1f(2.0f * kap[j]) + (cosang[j] - 1.0f);
    dy[4 * j + 1] = (b > kKappaLo && b < kKappaHi) ? g * r * dlv * kap[j] : 0.0f;
    const float m = g * r * kap[j];
    const float dmx = m * ox, dmy = m * oy, dmz = m * oz;
    dy[4 * j + 2] = dmx * (-ct[j] * st[j] * cp[j]) + dmy * (-ct[j] * st[j] * sp[j]) + dmz * (st[j] * st[j]);
    dy[4 * j + 3] = (dmx * (-st[j] * sp[j]) + dmy * (st[j] * cp[j])) * (CUDART_PI_F * (1.0f - thd[j] * thd[j]));
  }
  return -scale * logq;
}

// Shared-memory map of the training kernel.
constexpr int kTrainX = int(kImgBytes);                 // 128 x 80 BF16
constexpr int kTrainH1 = kTrainX + 128 * 80 * 2;        // 128 x 64
constexpr int kTrainH2 = kTrainH1 + 128 * 64 * 2;
constexpr int kTrainH3 = kTrainH2 + 128 * 64 * 2;
constexpr int kTrainDZ = kTrainH3 + 128 * 64 * 2;       // 128 x 64 (+ slack for M = 128 over-reads)
constexpr int kTrainBias = kTrainDZ + 128 * 64 * 2 + 4096;
constexpr int kTrainDB = kTrainBias + 224 * 4;
constexpr int kTrainSmem = kTrainDB + 224 * 4;
// TMEM columns.
constexpr uint32_t kColFwd = 0, kColDH = 64, kColDW4 = 128, kColDW3 = 192, kColDW2 = 256, kColDW1 = 320;

// Bias gradient of one tile: column sums of the 128-row K-major BF16 dZ tile (the values the
// weight-gradient MMA consumes), added to db. Thread c < k sums column c, so no atomics are needed.
__device__ __forceinline__ void tile_column_sums(const uint8_t* tile, int k, float* db, int tid) {
  if (tid >= k) return;
  float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll 8
  for (int r = 0; r < 128; ++r)
    acc[r & 3] += __bfloat162float(*reinterpret_cast<const __nv_bfloat16*>(tile + kmajor_offset(r, tid, k)));
  db[tid] += (acc[0] + acc[1]) + (acc[2] + acc[3]);
}

// Activation-gradient epilogue: dh (64 accumulator columns) -> dz = dh * [h > 0] -> BF16 row of the
// dZ tile (K = 64).
__device__ __forceinline__ void epilogue_backward(uint32_t lane_tmem, const uint8_t* h_tile, uint8_t* dz_tile,
                                                  int row) {
#pragma unroll
  for (int c = 0; c < 64; c += 16) {
    float v[16];
    umma::tmem_ld16(lane_tmem + uint32_t(c), v);
    umma::tmem_wait_ld();
#pragma unroll
    for (int hh = 0; hh < 2; ++hh) {
      const uint4 hv = *reinterpret_cast<const uint4*>(h_tile + kmajor_offset(row, c + 8 * hh, 64));
      const __nv_bfloat16* hb = reinterpret_cast<const __nv_bfloat16*>(&hv);
      float r[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        r[j] = __bfloat162float(hb[j]) > 0.0f ? v[8 * hh + j] : 0.0f;
      }
      uint4 o;
      o.x = pack_bf16x2(r[0], r[1]);
      o.y = pack_bf16x2(r[2], r[3]);
      o.z = pack_bf16x2(r[4], r[5]);
      o.w = pack_bf16x2(r[6], r[7]);
      *reinterpret_cast<uint4*>(dz_tile + kmajor_offset(row, c + 8 * hh, 64)) = o;
    }
  }
}

__global__ void __launch_bounds__(128, 1) guide_train_kernel(const float4* __restrict__ samples, uint32_t n,
                                                             const uint8_t* __restrict__ img,
                                                             const float* __restrict__ biases, GuideBounds bounds,
                                                             float inv_batch, float* __restrict__ grad, int* status,
                                                             float w_scale, float w_clamp, uint32_t gather_seed,
                                                             uint32_t n_total) {
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t* s_w = smem;
  uint8_t* s_x = smem + kTrainX;
  uint8_t* s_h[3] = {smem + kTrainH1, smem + kTrainH2, smem + kTrainH3};
  uint8_t* s_dz = smem + kTrainDZ;
  float* s_bias = reinterpret_cast<float*>(smem + kTrainBias);
  float* s_db = reinterpret_cast<float*>(smem + kTrainDB);
  __shared__ __align__(8) uint64_t mbar, mbar_w;
  __shared__ uint32_t tmem_base;
  __shared__ float s_loss;
  const int tid = threadIdx.x, warp = tid >> 5;
  // The weight images (forward and transposed) and biases arrive by two bulk copies completing on mbar_w.
  if (tid == 0) {
    umma::mbar_init(&mbar, 1);
    umma::mbar_init(&mbar_w, 1);
    umma::fence_mbar_init();
    umma::mbar_arrive_expect_tx(&mbar_w, kImgBytes + 224 * 4);
    umma::bulk_copy_g2s(s_w, img, kImgBytes, &mbar_w);
    umma::bulk_copy_g2s(s_bias, biases, 224 * 4, &mbar_w);
    s_loss = 0.0f;
  }
  for (int i = tid; i < 224; i += 128) s_db[i] = 0.0f;
  if (warp == 0) umma::tmem_alloc(&tmem_base, 512);
  sync_for_mma();
  if (!__syncthreads_and(umma::mbar_wait(&mbar_w, 0))) {
    if (tid == 0) atomicExch(status, 1);
    umma::fence_before_sync();
    __syncthreads();
    if (warp == 0) umma::tmem_dealloc(tmem_base, 512);
    return;
  }
  const uint32_t tmem = tmem_base;
  const uint32_t lane = uint32_t(warp * 32) << 16;
  uint32_t phase = 0;
  bool ok = true;
  float loss = 0.0f;
  bool accumulate = false;
  const uint32_t tiles = (n + 127) / 128;

  auto wait_mma = [&]() {
    const bool done = umma::mbar_wait(&mbar, phase);
    phase ^= 1u;
    ok = __syncthreads_and(done) != 0;
    umma::fence_after_sync();
    return ok;
  };

  for (uint32_t t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
    const uint32_t q = t * 128 + tid;
    const bool valid = q < n;
    float4 p = make_float4(0, 0, 0, 0), nn = p, om = p;
    if (valid) {
      uint32_t idx = q;
      if (gather_seed) {  // hashed draw (SplitMix-style finaliser) from the whole sample set
        uint32_t h = q * 0x9E3779B9u ^ gather_seed;
        h ^= h >> 16; h *= 0x7FEB352Du; h ^= h >> 15; h *= 0x846CA68Bu; h ^= h >> 16;
        idx = h % n_total;
      }
      p = samples[3 * size_t(idx)];
      nn = samples[3 * size_t(idx) + 1];
      om = samples[3 * size_t(idx) + 2];
      p.w = fminf(p.w * w_scale, w_clamp);
    }
    encode_row(s_x, tid, valid, p.x, p.y, p.z, nn.x, nn.y, nn.z, bounds);
    // Forward.
    const uint8_t* a_in = s_x;
    int k_in = 80;
    const uint32_t wimg[3] = {kImgW1, kImgW2, kImgW3};
    for (int l = 0; l < 3; ++l) {
      sync_for_mma();
      if (tid == 0) {
        issue_layer(tmem + kColFwd, a_in, s_w + wimg[l], k_in, 64);
        umma::commit(&mbar);
      }
      if (!wait_mma()) break;
      epilogue_hidden(tmem + lane + kColFwd, s_bias + 64 * l, s_h[l], tid);
      a_in = s_h[l];
      k_in = 64;
    }
    if (!ok) break;
    sync_for_mma();
    if (tid == 0) {
      issue_layer(tmem + kColFwd, s_h[2], s_w + kImgW4, 64, 32);
      umma::commit(&mbar);
    }
    if (!wait_mma()) break;
    {
      float y[32], dy[32];
      umma::tmem_ld16(tmem + lane + kColFwd, y);
      umma::tmem_ld16(tmem + lane + kColFwd + 16, y + 16);
      umma::tmem_wait_ld();
#pragma unroll
      for (int j = 0; j < 32; ++j) y[j] += s_bias[192 + j];
      if (valid) {
        loss += loss_and_grad(y, om.x, om.y, om.z, p.w * inv_batch, dy);
      } else {
#pragma unroll
        for (int j = 0; j < 32; ++j) dy[j] = 0.0f;
      }
      // dY as a K = 32 K-major tile (row-group stride 512 B) and its bias gradient.
#pragma unroll
      for (int g = 0; g < 4; ++g) {
        float r[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) r[j] = dy[8 * g + j];
        uint4 o;
        o.x = pack_bf16x2(r[0], r[1]);
        o.y = pack_bf16x2(r[2], r[3]);
        o.z = pack_bf16x2(r[4], r[5]);
        o.w = pack_bf16x2(r[6], r[7]);
        *reinterpret_cast<uint4*>(s_dz + kmajor_offset(tid, 8 * g, 32)) = o;
      }
    }
    __syncthreads();
    tile_column_sums(s_dz, 32, s_db + 192, tid);
    // Backward: dH3 = dY W4 and dW4 += dY^T H3.
    sync_for_mma();
    if (tid == 0) {
      issue_layer(tmem + kColDH, s_dz, s_w + kImgW4T, 32, 64);
      issue_weight_grad(tmem + kColDW4, s_dz, 32, s_h[2], 64, 64, accumulate);
      umma::commit(&mbar);
    }
    if (!wait_mma()) break;
    epilogue_backward(tmem + lane + kColDH, s_h[2], s_dz, tid);
    __syncthreads();
    tile_column_sums(s_dz, 64, s_db + 128, tid);
    // dH2 = dZ3 W3, dW3 += dZ3^T H2.
    sync_for_mma();
    if (tid == 0) {
      issue_layer(tmem + kColDH, s_dz, s_w + kImgW3T, 64, 64);
      issue_weight_grad(tmem + kColDW3, s_dz, 64, s_h[1], 64, 64, accumulate);
      umma::commit(&mbar);
    }
    if (!wait_mma()) break;
    epilogue_backward(tmem + lane + kColDH, s_h[1], s_dz, tid);
    __syncthreads();
    tile_column_sums(s_dz, 64, s_db + 64, tid);
    // dH1 = dZ2 W2, dW2 += dZ2^T H1.
    sync_for_mma();
    if (tid == 0) {
      issue_layer(tmem + kColDH, s_dz, s_w + kImgW2T, 64, 64);
      issue_weight_grad(tmem + kColDW2, s_dz, 64, s_h[0], 64, 64, accumulate);
      umma::commit(&mbar);
    }
    if (!wait_mma()) break;
    epilogue_backward(tmem + lane + kColDH, s_h[0], s_dz, tid);
    __syncthreads();
    tile_column_sums(s_dz, 64, s_db, tid);
    // dW1 += dZ1^T X.
    sync_for_mma();
    if (tid == 0) {
      issue_weight_grad(tmem + kColDW1, s_dz, 64, s_x, 80, 80, accumulate);
      umma::commit(&mbar);
    }
    if (!wait_mma()) break;
    accumulate = true;
  }

  // Flush this CTA's weight gradients (TMEM rows = output units) and bias gradients.
  if (ok && accumulate) {
    auto flush = [&](uint32_t col, int rows, int cols, int off) {
      if (warp * 32 >= rows) return;
      const int r = warp * 32 + (tid & 31);
      for (int c = 0; c < cols; c += 16) {
        float v[16];
        umma::tmem_ld16(tmem + lane + col + uint32_t(c), v);
        umma::tmem_wait_ld();
        if (r < rows)
          for (int j = 0; j < 16; ++j) atomicAdd(&grad[off + r * cols + c + j], v[j]);
      }
    };
    flush(kColDW4, 32, 64, kOffW4);
    flush(kColDW3, 64, 64, kOffW3);
    flush(kColDW2, 64, 64, kOffW2);
    flush(kColDW1, 64, 80, kOffW1);
  }
  __syncthreads();
  if (ok) {
    for (int i = tid; i < 224; i += 128) {
      const int off = i < 64 ? kOffB1 + i : (i < 128 ? kOffB2 + i - 64 : (i < 192 ? kOffB3 + i - 128 : kOffB4 + i - 192));
      atomicAdd(&grad[off], s_db[i]);
    }
    atomicAdd(&s_loss, loss);
  }
  __syncthreads();
  if (tid == 0) {
    if (ok) atomicAdd(&grad[kGuideParams], s_loss);
    else atomicExch(status, 1);
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem, 512);
}

cudaError_t guide_launch_loss_grad(const GuideDevice& g, const float4* samples, uint32_t n, float inv_batch,
                                   int sm_count, cudaStream_t stream, float w_scale, float w_clamp,
                                   uint32_t gather_seed, uint32_t n_total) {
  if (n == 0) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(guide_train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kTrainSmem);
  if (e != cudaSuccess) return e;
  const uint32_t tiles = (n + 127) / 128;
  const int grid = int(tiles < uint32_t(sm_count) ? tiles : uint32_t(sm_count));
  guide_train_kernel<<<grid, 128, kTrainSmem, stream>>>(samples, n, g.images, g.biases, g.bounds, inv_batch, g.grad,
                                                         g.status, w_scale, w_clamp, gather_seed,
                                                         n_total ? n_total : n);
  return cudaGetLastError();
}

// ------------------------------------------------------------------------ Adam
__global__ void guide_adam_kernel(float* __restrict__ p, float* __restrict__ m, float* __restrict__ v,
                                  float* __restrict__ grad, float lr, float bc1, float bc2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kGuideParams) return;
  const float g = grad[i];
  const float mi = 0.9f * m[i] + 0.1f * g;
  const float vi = 0.999f * v[i] + 0.001f * g * g;
  m[i] = mi;
  v[i] = vi;
  const bool pad = i >= kOffW1 && i < kOffB1 && (i - kOffW1) % kGuideIn >= 75;
  if (!pad) p[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + 1e-8f);
  grad[i] = 0.0f;
}

cudaError_t guide_launch_adam(GuideDevice& g, float lr, cudaStream_t stream) {
  g.adam_step += 1;
  const float bc1 = 1.0f - powf(0.9f, float(g.adam_step));
  const float bc2 = 1.0f - powf(0.999f, float(g.adam_step));
  guide_adam_kernel<<<(kGuideParams + 255) / 256, 256, 0, stream>>>(g.params, g.adam_m, g.adam_v, g.grad, lr, bc1, bc2);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return guide_refresh_images(g, stream);
}

}  // namespace tcb
