// Display conversion on the device: linear-HDR averages -> exposure -> ACES fitted -> clamp ->
// sRGB transfer -> RGBA8, as crates/toaster-core/src/color.rs:24-74 and
// crates/toaster-gpu/src/image_output.rs:57-88 do on the host after readback. Converting before
// the copy moves 4 bytes per pixel across PCIe instead of 16.
#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>

#include "display.h"

namespace tcb {

// Every product and sum is rounded on its own (no contraction into FMA), as Rust's f32 arithmetic
// does, so the bytes match the reference's host conversion.
__device__ __forceinline__ float aces_fitted_channel(float c) {
  if (isnan(c)) return 0.0f;
  if (isinf(c)) return c > 0.0f ? 1.0f : 0.0f;
  c = fmaxf(c, 0.0f);
  const float num = __fmul_rn(c, __fadd_rn(__fmul_rn(2.51f, c), 0.03f));
  const float den = __fadd_rn(__fmul_rn(c, __fadd_rn(__fmul_rn(2.43f, c), 0.59f)), 0.14f);
  return __fdiv_rn(num, den);
}

// c^(1/2.4) is evaluated in double precision and rounded once to float: the correctly rounded
// f32 power, which the host powf also returns for these arguments.
__device__ __forceinline__ float linear_to_srgb(float c) {
  if (c <= 0.0031308f) return __fmul_rn(12.92f, c);
  const float p = float(pow(double(c), double(1.0f / 2.4f)));
  return __fsub_rn(__fmul_rn(1.055f, p), 0.055f);
}

__device__ __forceinline__ uint32_t channel_to_u8(float c) {
  return uint32_t(roundf(__fmul_rn(fminf(fmaxf(c, 0.0f), 1.0f), 255.0f)));
}

__device__ __forceinline__ uint32_t display_pixel(float r, float g, float b, float a, float scale) {
  const float rgb[3] = {__fmul_rn(r, scale), __fmul_rn(g, scale), __fmul_rn(b, scale)};
  uint32_t out = 0;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float t = fminf(fmaxf(aces_fitted_channel(rgb[c]), 0.0f), 1.0f);
    out |= channel_to_u8(linear_to_srgb(t)) << (8 * c);
  }
  return out | (channel_to_u8(a) << 24);
}

// From FP64 per-pixel sums (3 doubles per pixel) divided by the sample count.
__global__ void display_sums_kernel(const double* __restrict__ sums, uint32_t pixels, double inv_samples, float scale,
                                    uint32_t* __restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= pixels) return;
  const double* s = sums + size_t(3) * i;
  out[i] = display_pixel(float(s[0] * inv_samples), float(s[1] * inv_samples), float(s[2] * inv_samples), 1.0f, scale);
}

// From float4 linear-HDR pixels.
__global__ void display_rgba_kernel(const float4* __restrict__ px, uint32_t pixels, float scale,
                                    uint32_t* __restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= pixels) return;
  const float4 p = px[i];
  out[i] = display_pixel(p.x, p.y, p.z, p.w, scale);
}

// From FP64 per-pixel sums to interleaved RGB8 (the input of the JPEG encoder; JPEG drops alpha).
__global__ void display_rgb8_sums_kernel(const double* __restrict__ sums, uint32_t pixels, double inv_samples,
                                         float scale, uint8_t* __restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= pixels) return;
  const double* s = sums + size_t(3) * i;
  const uint32_t p =
      display_pixel(float(s[0] * inv_samples), float(s[1] * inv_samples), float(s[2] * inv_samples), 1.0f, scale);
  out[3 * size_t(i)] = uint8_t(p);
  out[3 * size_t(i) + 1] = uint8_t(p >> 8);
  out[3 * size_t(i) + 2] = uint8_t(p >> 16);
}

cudaError_t launch_display_rgb8_from_sums(const double* sums, uint32_t pixels, double inv_samples,
                                          float exposure_stops, uint8_t* out, cudaStream_t stream) {
  if (pixels == 0) return cudaSuccess;
  display_rgb8_sums_kernel<<<(pixels + 255) / 256, 256, 0, stream>>>(sums, pixels, inv_samples,
                                                                     std::exp2(exposure_stops), out);
  return cudaGetLastError();
}

cudaError_t launch_display_from_sums(const double* sums, uint32_t pixels, double inv_samples, float exposure_stops,
                                     uint32_t* out, cudaStream_t stream) {
  if (pixels == 0) return cudaSuccess;
  display_sums_kernel<<<(pixels + 255) / 256, 256, 0, stream>>>(sums, pixels, inv_samples, std::exp2(exposure_stops), out);
  return cudaGetLastError();
}

cudaError_t launch_display_from_rgba(const float4* px, uint32_t pixels, float exposure_stops, uint32_t* out,
                                     cudaStream_t stream) {
  if (pixels == 0) return cudaSuccess;
  display_rgba_kernel<<<(pixels + 255) / 256, 256, 0, stream>>>(px, pixels, std::exp2(exposure_stops), out);
  return cudaGetLastError();
}

}  // namespace tcb
