// Device refit of the sibling-pair hierarchy (refit.cu).
#ifndef TOASTER_B200_REFIT_H
#define TOASTER_B200_REFIT_H

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "../../include/toaster_cuda.h"
#include "layout.h"

namespace tcb {

// Pair-node indices grouped by tree depth (level 0 = the root's pair node), on the device, with
// host-side offsets: level l holds nodes[level_offsets[l] .. level_offsets[l + 1]).
struct RefitPlan {
  const uint32_t* nodes = nullptr;
  std::vector<uint32_t> level_offsets;
};

// Rewrites the primitive records from the new geometry (sph / tri in scene order, device memory)
// and recomputes every child box bottom-up, then the root record (device memory).
cudaError_t launch_refit(const RefitPlan& plan, PairNode* pairs, ChildRec* root, PrimRecord* prims,
                         uint32_t prim_count, const tc_gpu_sphere* sph, const tc_gpu_triangle* tri,
                         cudaStream_t stream);

}  // namespace tcb

#endif
