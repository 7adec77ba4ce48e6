// Per-frame geometry update without a rebuild: new sphere / triangle positions are written into
// the leaf-ordered primitive records, then the hierarchy's bounds are recomputed bottom-up, one
// launch per tree level (deepest first), keeping the topology of the last build. The reference
// rebuilds its BVH on the host every frame (crates/toaster-gpu/src/path_tracer.rs:611-638);
// refitting keeps every intersection exact (primitives are exact, boxes stay conservative) while
// the tree adapts less well to large motion, so images agree statistically, not hit for hit.
#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

#include "../../include/toaster_cuda.h"
#include "layout.h"
#include "refit.h"

namespace tcb {

// Bounds of one primitive in the build's definition (scene_upload.rs:296-346): spheres
// centre +- radius, triangles the vertex box padded by 1e-5.
__device__ __forceinline__ void prim_bounds(uint32_t tag, const tc_gpu_sphere* sph, const tc_gpu_triangle* tri,
                                            float* lo, float* hi) {
  const uint32_t idx = tag & kTagIndexMask;
  if (tag & kTagTriangle) {
    const tc_gpu_triangle& t = tri[idx];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      lo[a] = __fsub_rn(fminf(fminf(t.v0[a], t.v1[a]), t.v2[a]), 1e-5f);
      hi[a] = __fadd_rn(fmaxf(fmaxf(t.v0[a], t.v1[a]), t.v2[a]), 1e-5f);
    }
  } else {
    const tc_gpu_sphere& s = sph[idx];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      lo[a] = __fsub_rn(s.center_radius[a], s.center_radius[3]);
      hi[a] = __fadd_rn(s.center_radius[a], s.center_radius[3]);
    }
  }
}

__global__ void update_prims_kernel(PrimRecord* __restrict__ prims, uint32_t n, const tc_gpu_sphere* __restrict__ sph,
                                    const tc_gpu_triangle* __restrict__ tri) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  PrimRecord r = prims[k];
  const uint32_t tag = __float_as_uint(r.a[3]);
  const uint32_t idx = tag & kTagIndexMask;
  if (tag & kTagTriangle) {
    const tc_gpu_triangle& t = tri[idx];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      r.a[a] = t.v0[a];
      r.b[a] = __fsub_rn(t.v1[a], t.v0[a]);  // the same f32 differences the host build stores
      r.c[a] = __fsub_rn(t.v2[a], t.v0[a]);
    }
  } else {
    const tc_gpu_sphere& s = sph[idx];
#pragma unroll
    for (int a = 0; a < 3; ++a) r.a[a] = s.center_radius[a];
    r.b[0] = s.center_radius[3];
    r.b[1] = __fmul_rn(s.center_radius[3], s.center_radius[3]);
  }
  prims[k] = r;
}

__device__ void child_bounds(const ChildRec& c, const PairNode* pairs, const PrimRecord* prims,
                             const tc_gpu_sphere* sph, const tc_gpu_triangle* tri, float* lo, float* hi) {
  lo[0] = lo[1] = lo[2] = CUDART_INF_F;
  hi[0] = hi[1] = hi[2] = -CUDART_INF_F;
  if (c.link & kLeafBit) {
    for (uint32_t k = c.link & ~kLeafBit;; ++k) {
      const uint32_t tag = __float_as_uint(prims[k].a[3]);
      float l[3], h[3];
      prim_bounds(tag, sph, tri, l, h);
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        lo[a] = fminf(lo[a], l[a]);
        hi[a] = fmaxf(hi[a], h[a]);
      }
      if (tag & kTagLast) break;
    }
  } else {
    const PairNode& p = pairs[c.link];
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      const ChildRec& g = p.child[s];
      lo[0] = fminf(lo[0], g.min_x); lo[1] = fminf(lo[1], g.min_y); lo[2] = fminf(lo[2], g.min_z);
      hi[0] = fmaxf(hi[0], g.max_x); hi[1] = fmaxf(hi[1], g.max_y); hi[2] = fmaxf(hi[2], g.max_z);
    }
  }
}

__device__ __forceinline__ void store_bounds(ChildRec& c, const float* lo, const float* hi) {
  c.min_x = lo[0]; c.min_y = lo[1]; c.min_z = lo[2];
  c.max_x = hi[0]; c.max_y = hi[1]; c.max_z = hi[2];
}

// One level: the pair nodes listed in nodes[0..count) get both child records recomputed.
__global__ void refit_level_kernel(PairNode* __restrict__ pairs, const uint32_t* __restrict__ nodes, uint32_t count,
                                   const PrimRecord* __restrict__ prims, const tc_gpu_sphere* __restrict__ sph,
                                   const tc_gpu_triangle* __restrict__ tri) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 2 * count) return;
  const uint32_t node = nodes[i >> 1];
  ChildRec& c = pairs[node].child[i & 1];
  float lo[3], hi[3];
  child_bounds(c, pairs, prims, sph, tri, lo, hi);
  store_bounds(c, lo, hi);
}

__global__ void refit_root_kernel(ChildRec* root, const PairNode* __restrict__ pairs, const PrimRecord* __restrict__ prims,
                                  const tc_gpu_sphere* __restrict__ sph, const tc_gpu_triangle* __restrict__ tri) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  float lo[3], hi[3];
  child_bounds(*root, pairs, prims, sph, tri, lo, hi);
  store_bounds(*root, lo, hi);
}

cudaError_t launch_refit(const RefitPlan& plan, PairNode* pairs, ChildRec* root, PrimRecord* prims,
                         uint32_t prim_count, const tc_gpu_sphere* sph, const tc_gpu_triangle* tri,
                         cudaStream_t stream) {
  if (prim_count == 0) return cudaSuccess;
  update_prims_kernel<<<(prim_count + 255) / 256, 256, 0, stream>>>(prims, prim_count, sph, tri);
  for (int level = int(plan.level_offsets.size()) - 2; level >= 0; --level) {
    const uint32_t first = plan.level_offsets[size_t(level)];
    const uint32_t count = plan.level_offsets[size_t(level) + 1] - first;
    if (count == 0) continue;
    refit_level_kernel<<<(2 * count + 255) / 256, 256, 0, stream>>>(pairs, plan.nodes + first, count, prims, sph, tri);
  }
  refit_root_kernel<<<1, 32, 0, stream>>>(root, pairs, prims, sph, tri);
  return cudaGetLastError();
}

}  // namespace tcb
