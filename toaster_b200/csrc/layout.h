// Device-side data layout of the toaster B200 path tracer (shared by host and device code).
//
// Hierarchy: the median-split BVH of crates/toaster-bvh (bvh.rs:92-154, flatten.rs:72-97) is
// stored as *sibling pairs*: one 64-byte PairNode per interior node holds the 32-byte records of
// both children (exact FP32 bounds, link, count). Visiting an interior node is one contiguous
// 64-byte fetch (four LDG.128) that yields everything the reference reads at that step (the two
// child boxes it tests at intersect.rs:230-258). Bounds stay exact FP32 (not quantised) so that
// box tests, entry distances and therefore the front-to-back order, including its tie rule,
// are bit-identical to the reference traversal.
//
// Primitives: the leaf-ordered primitive references are resolved into 48-byte PrimRecords
// stored in leaf order, so a leaf's primitives are contiguous and need no indirection:
//   triangle: {v0.xyz, tag} {e1.xyz, material} {e2.xyz, attribute flags}
//   sphere:   {center.xyz, tag} {radius, radius*radius, 0, material} {0, 0, 0, 0}
// e1 = v1 - v0 and e2 = v2 - v0 are the FP32 differences intersect.rs:96-97 computes, so
// precomputing them on the host changes no bit. The tag packs the scene index (bits 0-29),
// a last-in-leaf flag (bit 30) and the GpuPrimitiveRef kind (bit 31: 1 = triangle).
#ifndef TOASTER_B200_LAYOUT_H
#define TOASTER_B200_LAYOUT_H

#include <stdint.h>

#ifdef __CUDACC__
#define TC_HD __host__ __device__
#else
#define TC_HD
#endif

namespace tcb {

constexpr uint32_t kLeafBit = 0x80000000u;   // ChildRec.link: leaf (first prim record) vs pair index
constexpr uint32_t kTagTriangle = 0x80000000u;
constexpr uint32_t kTagLast = 0x40000000u;
constexpr uint32_t kTagIndexMask = 0x3FFFFFFFu;
constexpr uint32_t kMaxPrimitives = kTagIndexMask;  // scene indices must fit the tag
constexpr int kMaxStack = 64;                       // traversal stack entries (checked vs depth)

struct alignas(16) ChildRec {
  float min_x, min_y, min_z;
  uint32_t link;   // interior: PairNode index; leaf: kLeafBit | first PrimRecord
  float max_x, max_y, max_z;
  uint32_t count;  // leaf primitive count (0 for interior)
};
static_assert(sizeof(ChildRec) == 32, "ChildRec is 32 bytes");

struct alignas(16) PairNode {
  ChildRec child[2];  // [0] = left (flat index parent+1), [1] = right
};
static_assert(sizeof(PairNode) == 64, "PairNode is 64 bytes");

struct alignas(16) PrimRecord {
  float a[4];
  float b[4];
  float c[4];
};
static_assert(sizeof(PrimRecord) == 48, "PrimRecord is 48 bytes");

// Material kinds match GpuMaterial.kind (gpu_types.rs:129).
enum MaterialKind : uint32_t { kDiffuse = 0, kMetal = 1, kDielectric = 2, kEmissive = 3 };

struct alignas(16) DevMaterial {
  float albedo[3];      // diffuse / metal albedo (dielectric: 1)
  uint32_t kind;
  float emission[3];    // colour * strength for emissive materials
  float roughness;      // clamped to [0,1] on upload (integrator.rs:305)
  float ior;
  uint32_t tex_offset, tex_width, tex_height;
};
static_assert(sizeof(DevMaterial) == 48, "DevMaterial is 48 bytes");

// Emitter for next-event estimation; selection by a Walker alias table over weights.
struct alignas(16) DevLight {
  float p0[3];      // triangle v0 or sphere centre
  uint32_t kind;    // 0 triangle, 1 sphere (GpuLight.kind)
  float e1[3];      // triangle v1 - v0
  float radius;     // sphere radius
  float e2[3];      // triangle v2 - v0
  float pdf_area;   // selection probability / area (light.rs:160-168)
  float normal[3];  // unit triangle normal (light.rs:77)
  float alias_prob; // alias table: keep probability of this slot
  float emission[3];
  uint32_t alias;   // alias table: fallback light index
};
static_assert(sizeof(DevLight) == 80, "DevLight is 80 bytes");

}  // namespace tcb

#endif
