// Median-split hierarchy build on the device (bvh_device.cu).
//
// The reference tree (crates/toaster-bvh/src/bvh.rs:92-154) splits every node of more than four
// primitives at count/2 after a stable sort along the longest centroid axis. Its shape therefore
// depends on the primitive count alone, unless a node's centroid extent is <= f32::EPSILON (a
// degenerate leaf of more than four primitives). The plan fixes that shape on the host once per
// count: every node's range, its depth-first index among interior nodes (the pair index of the
// device layout) and the slot it fills in its parent. The build then runs level by level on the
// device: bounds and centroid bounds of every node (order-independent min/max), the split axis
// of every interior node, and one segmented stable sort of the primitive order per level. All
// launch sizes are fixed by the plan, so a build can be captured in a CUDA graph. A node that
// the reference would turn into a degenerate leaf sets a status word instead; the caller then
// uses the host build.
#ifndef TOASTER_B200_BVH_DEVICE_H
#define TOASTER_B200_BVH_DEVICE_H

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "../../include/toaster_cuda.h"
#include "layout.h"

namespace tcb {

class DeviceBvhBuilder {
 public:
  DeviceBvhBuilder() = default;
  ~DeviceBvhBuilder();
  DeviceBvhBuilder(const DeviceBvhBuilder&) = delete;
  DeviceBvhBuilder& operator=(const DeviceBvhBuilder&) = delete;

  // Plans (or re-plans, when the counts changed) a build for these primitive counts and sizes
  // every device buffer. Host work proportional to the node count; no device work.
  cudaError_t plan(uint32_t n_spheres, uint32_t n_triangles);

  // Enqueues the build on `stream`: from scene-order geometry (device memory) to the device
  // layout (pairs: pair_count() entries, root: one record, prims: n records). Material indices
  // come from the geometry records; attr_flags (device, n_triangles words, may be null) holds the
  // triangle attribute flags. *status (device word) is set to 1 when a node is degenerate.
  cudaError_t build(const tc_gpu_sphere* spheres, const tc_gpu_triangle* triangles, const uint32_t* attr_flags,
                    PairNode* pairs, ChildRec* root, PrimRecord* prims, uint32_t* status, cudaStream_t stream);

  uint32_t pair_count() const { return pair_count_; }
  uint32_t depth() const { return depth_; }
  // Pair indices grouped by depth (root level first) for the refit, with host-side offsets.
  const uint32_t* refit_nodes() const { return refit_nodes_; }
  const std::vector<uint32_t>& refit_levels() const { return refit_levels_; }

 private:
  void release();

  uint32_t ns_ = 0, nt_ = 0, n_ = 0;
  uint32_t pair_count_ = 0, depth_ = 0, node_count_ = 0;
  std::vector<uint32_t> level_nodes_;      // nodes of level l: [level_nodes_[l], level_nodes_[l + 1])
  std::vector<uint32_t> level_segments_;   // interior nodes (sort segments) of level l, same layout
  std::vector<uint32_t> level_chunks_;     // reduction chunks of level l, same layout
  std::vector<uint32_t> refit_levels_;
  // Device tables (node id = breadth-first index).
  uint32_t* node_lo_ = nullptr;
  uint32_t* node_hi_ = nullptr;
  uint32_t* node_link_ = nullptr;     // interior: own pair index; leaf: kLeafBit | first position
  uint32_t* node_parent_ = nullptr;   // parent's pair index << 1 | slot; 0xFFFFFFFF for the root
  uint32_t* seg_node_ = nullptr;      // interior node of each sort segment
  uint32_t* seg_begin_ = nullptr;
  uint32_t* seg_end_ = nullptr;
  uint32_t* chunk_node_ = nullptr;    // reduction chunks: node and position range
  uint32_t* chunk_lo_ = nullptr;
  uint32_t* chunk_hi_ = nullptr;
  uint32_t* last_ = nullptr;          // per position: 1 at the last primitive of a leaf
  uint32_t* refit_nodes_ = nullptr;
  // Working buffers.
  float* item_box_ = nullptr;         // per primitive: min xyz, max xyz, centroid xyz (9 floats)
  uint32_t* node_keys_ = nullptr;     // per node: 12 ordered keys (min xyz, max xyz, cmin xyz, cmax xyz)
  uint32_t* node_axis_ = nullptr;
  uint32_t* keys_[2] = {nullptr, nullptr};
  uint32_t* perm_[2] = {nullptr, nullptr};
  void* sort_temp_ = nullptr;
  size_t sort_temp_bytes_ = 0;
};

}  // namespace tcb

#endif
