// Device display conversion (display.cu): linear HDR -> RGBA8 with the reference's exposure,
// ACES fitted tone mapping and sRGB transfer. Pixels are packed little-endian R, G, B, A.
#ifndef TOASTER_B200_DISPLAY_H
#define TOASTER_B200_DISPLAY_H

#include <cuda_runtime.h>
#include <stdint.h>

namespace tcb {

cudaError_t launch_display_from_sums(const double* sums, uint32_t pixels, double inv_samples, float exposure_stops,
                                     uint32_t* out, cudaStream_t stream);
cudaError_t launch_display_rgb8_from_sums(const double* sums, uint32_t pixels, double inv_samples,
                                          float exposure_stops, uint8_t* out, cudaStream_t stream);
cudaError_t launch_display_from_rgba(const float4* px, uint32_t pixels, float exposure_stops, uint32_t* out,
                                     cudaStream_t stream);

}  // namespace tcb

#endif
