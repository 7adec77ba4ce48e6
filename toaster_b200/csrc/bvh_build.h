// Host-side hierarchy construction and conversion to the sibling-pair device layout.
#ifndef TOASTER_B200_BVH_BUILD_H
#define TOASTER_B200_BVH_BUILD_H

#include <stddef.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "layout.h"

namespace tcb {

// One node of the reference's flat depth-first hierarchy (GpuBvhNode without padding).
struct FlatNode {
  float min[3], max[3];
  uint32_t first_or_right;
  uint32_t count;  // > 0 marks a leaf
};

struct PrimRef {
  uint32_t kind;  // 0 sphere, 1 triangle (GpuPrimitiveRef.kind)
  uint32_t index;
};

struct FlatHierarchy {
  std::vector<FlatNode> nodes;
  std::vector<PrimRef> prims;
};

struct SphereIn {
  float center[3];
  float radius;
};
struct TriangleIn {
  float v[3][3];
};

// Median-split build with the rules of crates/toaster-bvh/src/bvh.rs:92-154: union bounds,
// centroid bounds, longest axis (ties to the lower axis), leaf when n <= max_leaf or when the
// centroid extent on that axis is <= f32::EPSILON, stable sort by f32::total_cmp, split at n/2;
// emitted depth first with the left child right after its parent (flatten.rs:72-97).
// Spheres come first, then triangles with bounds padded by 1e-5 (scene_upload.rs:296-346).
FlatHierarchy build_median_split(const SphereIn* spheres, size_t n_spheres, const TriangleIn* triangles,
                                 size_t n_triangles, size_t max_leaf = 4);

// Device images of a hierarchy: sibling-pair nodes, the root record and leaf-ordered primitives.
struct DeviceHierarchy {
  std::vector<PairNode> pairs;
  ChildRec root;
  std::vector<PrimRecord> prims;
  uint32_t depth = 0;  // deepest node level (root = 1)
};

// Converts a flat hierarchy (built here or supplied by the caller in the reference layout)
// and the scene geometry into the device layout. Returns false with a message on malformed
// input (out-of-range links, cycles, primitive indices beyond the scene arrays).
bool to_device_layout(const FlatHierarchy& flat, const SphereIn* spheres, const uint32_t* sphere_materials,
                      size_t n_spheres, const TriangleIn* triangles, const uint32_t* triangle_materials,
                      const uint32_t* triangle_attr_flags, size_t n_triangles, DeviceHierarchy& out,
                      std::string& error);

}  // namespace tcb

#endif
