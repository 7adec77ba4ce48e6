// Path-guiding network: parameter packing, device state and kernel launchers (guide.cu).
//
// The network maps an 80-wide encoding of a surface point (Fourier features of the normalised
// position at 12 half-octave frequencies 2^(k/2) + the normal) through three 64-wide ReLU layers to 32 outputs that
// parameterise an 8-lobe von Mises-Fisher mixture over outgoing directions.
#ifndef TOASTER_B200_GUIDE_H
#define TOASTER_B200_GUIDE_H

#include <cuda_runtime.h>
#include <stdint.h>

namespace tcb {

constexpr int kGuideIn = 80, kGuideHid = 64, kGuideOut = 32, kGuideLobes = 8, kGuideFreqs = 12;
// FP32 master parameters packed as W1[64][80], b1, W2[64][64], b2, W3[64][64], b3, W4[32][64], b4.
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kGuideHid * kGuideIn;
constexpr int kOffW2 = kOffB1 + kGuideHid;
constexpr int kOffB2 = kOffW2 + kGuideHid * kGuideHid;
constexpr int kOffW3 = kOffB2 + kGuideHid;
constexpr int kOffB3 = kOffW3 + kGuideHid * kGuideHid;
constexpr int kOffW4 = kOffB3 + kGuideHid;
constexpr int kOffB4 = kOffW4 + kGuideOut * kGuideHid;
constexpr int kGuideParams = kOffB4 + kGuideOut;  // 15,584
// Decoded mixture per query: 8 x (mu.xyz, kappa) then 8 weights -> 10 float4.
constexpr int kGuideDecodedF4 = 10;

// BF16 weight images in the canonical K-major shared-memory layout, byte offsets.
constexpr uint32_t kImgW1 = 0;                        // 64 x 80
constexpr uint32_t kImgW2 = kImgW1 + 64 * 80 * 2;     // 64 x 64
constexpr uint32_t kImgW3 = kImgW2 + 64 * 64 * 2;     // 64 x 64
constexpr uint32_t kImgW4 = kImgW3 + 64 * 64 * 2;     // 32 x 64
constexpr uint32_t kImgFwdBytes = kImgW4 + 32 * 64 * 2;
constexpr uint32_t kImgW2T = kImgFwdBytes;            // 64 x 64 (rows = inputs, K = outputs)
constexpr uint32_t kImgW3T = kImgW2T + 64 * 64 * 2;   // 64 x 64
constexpr uint32_t kImgW4T = kImgW3T + 64 * 64 * 2;   // 64 x 32
constexpr uint32_t kImgBytes = kImgW4T + 64 * 32 * 2;

struct GuideBounds {
  float cx, cy, cz, scale;  // encoding uses (p - c) * scale
};

struct GuideDevice {
  float* params = nullptr;  // FP32 master weights (kGuideParams)
  float* adam_m = nullptr;
  float* adam_v = nullptr;
  float* grad = nullptr;    // FP32 gradient accumulator (kGuideParams) + 1 loss slot
  uint8_t* images = nullptr;  // kImgBytes of BF16 weight images
  float* biases = nullptr;    // b1 | b2 | b3 | b4 copied contiguously (224 floats)
  int* status = nullptr;
  GuideBounds bounds{};
  uint32_t adam_step = 0;
};

cudaError_t guide_refresh_images(const GuideDevice& g, cudaStream_t stream);
// queries: 2 float4 per query (position, normal); out: kGuideDecodedF4 float4 per query.
// When n_dev is non-null the query count is read from device memory (capped at n).
cudaError_t guide_launch_infer(const GuideDevice& g, const float4* queries, uint32_t n, float4* out, int sm_count,
                               cudaStream_t stream, const uint32_t* n_dev = nullptr);
// samples: 3 float4 per sample (position + weight, normal, direction); gradient of the mean
// weighted NLL accumulated into g.grad[0..kGuideParams), the loss into g.grad[kGuideParams].
// Sample weights are scaled by w_scale and clamped at w_clamp. With gather_seed != 0 the n
// samples of the batch are drawn (hashed indices) from the first n_total samples.
cudaError_t guide_launch_loss_grad(const GuideDevice& g, const float4* samples, uint32_t n, float inv_batch,
                                   int sm_count, cudaStream_t stream, float w_scale = 1.0f,
                                   float w_clamp = 3.0e38f, uint32_t gather_seed = 0, uint32_t n_total = 0);
cudaError_t guide_launch_adam(GuideDevice& g, float lr, cudaStream_t stream);

}  // namespace tcb

#endif
