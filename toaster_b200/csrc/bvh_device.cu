// Median-split hierarchy build on the device; see bvh_device.h for the scheme.
//
// Exactness against the host build (bvh_build.cpp, itself bit-compatible with toaster-bvh):
// primitive boxes and centroids use the same single-rounded f32 operations; node and centroid
// bounds are min/max reductions, which are exact in any order (they may pick the other zero of a
// +0/-0 tie, which no box test can tell apart); the split axis and the degenerate test compare
// the same f32 extents; the per-node stable sort by f32::total_cmp keys is a segmented stable
// radix sort of the same keys. Topology and primitive order are therefore identical.
#include <cuda_runtime.h>
#include <float.h>
#include <math_constants.h>
#include <stdint.h>

#include <cub/device/device_segmented_sort.cuh>

#include <algorithm>

#include "bvh_device.h"

namespace tcb {
namespace {

constexpr uint32_t kMaxLeaf = 4;
constexpr uint32_t kChunk = 1024;     // positions reduced by one warp
constexpr uint32_t kNoParent = 0xFFFFFFFFu;

// f32::total_cmp order as an unsigned key, and back.
__host__ __device__ __forceinline__ uint32_t order_key(float f) {
  uint32_t b;
  memcpy(&b, &f, 4);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float from_key(uint32_t k) {
  const uint32_t b = (k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k;
  return __uint_as_float(b);
}

template <class T>
cudaError_t alloc(T*& p, size_t count) {
  if (p) cudaFree(p);
  p = nullptr;
  if (count == 0) return cudaSuccess;
  return cudaMalloc(reinterpret_cast<void**>(&p), sizeof(T) * count);
}

// Primitive boxes in the build's definition (scene_upload.rs:296-346): spheres centre +- r,
// triangles the vertex box padded by 1e-5; centroid = 0.5 * (min + max).
__global__ void item_boxes_kernel(const tc_gpu_sphere* __restrict__ sph, uint32_t ns,
                                  const tc_gpu_triangle* __restrict__ tri, uint32_t n, float* __restrict__ box,
                                  uint32_t* __restrict__ perm) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n) return;
  float mn[3], mx[3];
  if (g < ns) {
    const tc_gpu_sphere& s = sph[g];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      mn[a] = __fsub_rn(s.center_radius[a], s.center_radius[3]);
      mx[a] = __fadd_rn(s.center_radius[a], s.center_radius[3]);
    }
  } else {
    const tc_gpu_triangle& t = tri[g - ns];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      mn[a] = __fsub_rn(fminf(fminf(t.v0[a], t.v1[a]), t.v2[a]), 1e-5f);
      mx[a] = __fadd_rn(fmaxf(fmaxf(t.v0[a], t.v1[a]), t.v2[a]), 1e-5f);
    }
  }
  float* b = box + 9 * size_t(g);
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    b[a] = mn[a];
    b[3 + a] = mx[a];
    b[6 + a] = __fmul_rn(0.5f, __fadd_rn(mn[a], mx[a]));
  }
  perm[g] = g;
}

// One warp per chunk: min/max of the boxes and centroids of the primitives at positions
// [lo, hi) of one node, merged into the node's 12 ordered keys with atomics.
__global__ void node_bounds_kernel(const uint32_t* __restrict__ chunk_node, const uint32_t* __restrict__ chunk_lo,
                                   const uint32_t* __restrict__ chunk_hi, uint32_t chunks,
                                   const uint32_t* __restrict__ perm, const float* __restrict__ box,
                                   uint32_t* __restrict__ node_keys) {
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const unsigned lane = threadIdx.x & 31u;
  if (warp >= chunks) return;
  const uint32_t lo = chunk_lo[warp], hi = chunk_hi[warp];
  uint32_t kmin[6], kmax[6];  // box min (0..2), centroid (3..5) lower keys; box max, centroid upper keys
#pragma unroll
  for (int a = 0; a < 6; ++a) {
    kmin[a] = 0xFFFFFFFFu;
    kmax[a] = 0u;
  }
  for (uint32_t p = lo + lane; p < hi; p += 32) {
    const float* b = box + 9 * size_t(perm[p]);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      kmin[a] = min(kmin[a], order_key(b[a]));
      kmax[a] = max(kmax[a], order_key(b[3 + a]));
      const uint32_t c = order_key(b[6 + a]);
      kmin[3 + a] = min(kmin[3 + a], c);
      kmax[3 + a] = max(kmax[3 + a], c);
    }
  }
#pragma unroll
  for (int a = 0; a < 6; ++a) {
    kmin[a] = __reduce_min_sync(0xffffffffu, kmin[a]);
    kmax[a] = __reduce_max_sync(0xffffffffu, kmax[a]);
  }
  if (lane == 0) {
    uint32_t* k = node_keys + 12 * size_t(chunk_node[warp]);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      atomicMin(k + a, kmin[a]);           // box min
      atomicMax(k + 3 + a, kmax[a]);       // box max
      atomicMin(k + 6 + a, kmin[3 + a]);   // centroid min
      atomicMax(k + 9 + a, kmax[3 + a]);   // centroid max
    }
  }
}

__global__ void init_keys_kernel(uint32_t* __restrict__ node_keys, uint32_t first, uint32_t count) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 12 * count) return;
  const uint32_t slot = i % 12;
  node_keys[12 * size_t(first) + i] = (slot < 3 || (slot >= 6 && slot < 9)) ? 0xFFFFFFFFu : 0u;
}

// Split axis of every interior node of a level: the longest centroid extent, ties to the lower
// axis; an extent <= f32::EPSILON makes the reference stop with a leaf, which the fixed plan
// cannot express, so it raises the status word.
__global__ void split_axis_kernel(const uint32_t* __restrict__ seg_node, uint32_t segs,
                                  const uint32_t* __restrict__ node_keys, uint32_t* __restrict__ node_axis,
                                  uint32_t* __restrict__ status) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= segs) return;
  const uint32_t node = seg_node[s];
  const uint32_t* k = node_keys + 12 * size_t(node);
  const float ex = __fsub_rn(from_key(k[9]), from_key(k[6]));
  const float ey = __fsub_rn(from_key(k[10]), from_key(k[7]));
  const float ez = __fsub_rn(from_key(k[11]), from_key(k[8]));
  const uint32_t axis = (ex >= ey && ex >= ez) ? 0u : (ey >= ez ? 1u : 2u);
  const float extent = axis == 0 ? ex : (axis == 1 ? ey : ez);
  if (extent <= FLT_EPSILON) atomicExch(status, 1u);
  node_axis[node] = axis;
}

// Sort keys of every position inside an interior node of the level (one warp per chunk).
__global__ void sort_keys_kernel(const uint32_t* __restrict__ chunk_node, const uint32_t* __restrict__ chunk_lo,
                                 const uint32_t* __restrict__ chunk_hi, uint32_t chunks,
                                 const uint32_t* __restrict__ node_link, const uint32_t* __restrict__ node_axis,
                                 const uint32_t* __restrict__ perm, const float* __restrict__ box,
                                 uint32_t* __restrict__ keys) {
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const unsigned lane = threadIdx.x & 31u;
  if (warp >= chunks) return;
  const uint32_t node = chunk_node[warp];
  if (node_link[node] & kLeafBit) return;
  const uint32_t axis = node_axis[node];
  for (uint32_t p = chunk_lo[warp] + lane; p < chunk_hi[warp]; p += 32)
    keys[p] = order_key(box[9 * size_t(perm[p]) + 6 + axis]);
}

// Child records into the parents' pair slots (or the root record).
__global__ void write_nodes_kernel(uint32_t nodes, const uint32_t* __restrict__ node_lo,
                                   const uint32_t* __restrict__ node_hi, const uint32_t* __restrict__ node_link,
                                   const uint32_t* __restrict__ node_parent, const uint32_t* __restrict__ node_keys,
                                   PairNode* __restrict__ pairs, ChildRec* __restrict__ root) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nodes) return;
  const uint32_t* k = node_keys + 12 * size_t(i);
  ChildRec r;
  r.min_x = from_key(k[0]);
  r.min_y = from_key(k[1]);
  r.min_z = from_key(k[2]);
  r.max_x = from_key(k[3]);
  r.max_y = from_key(k[4]);
  r.max_z = from_key(k[5]);
  r.link = node_link[i];
  r.count = (r.link & kLeafBit) ? node_hi[i] - node_lo[i] : 0u;
  const uint32_t parent = node_parent[i];
  if (parent == kNoParent) *root = r;
  else pairs[parent >> 1].child[parent & 1u] = r;
}

// Leaf-ordered primitive records, as to_device_layout writes them.
__global__ void write_prims_kernel(uint32_t n, uint32_t ns, const uint32_t* __restrict__ perm,
                                   const uint32_t* __restrict__ last, const tc_gpu_sphere* __restrict__ sph,
                                   const tc_gpu_triangle* __restrict__ tri, const uint32_t* __restrict__ attr_flags,
                                   PrimRecord* __restrict__ prims) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const uint32_t g = perm[k];
  PrimRecord rec;
#pragma unroll
  for (int a = 0; a < 4; ++a) rec.a[a] = rec.b[a] = rec.c[a] = 0.0f;
  uint32_t tag = (last[k] ? kTagLast : 0u);
  if (g < ns) {
    const tc_gpu_sphere& s = sph[g];
    tag |= g;
    rec.a[0] = s.center_radius[0];
    rec.a[1] = s.center_radius[1];
    rec.a[2] = s.center_radius[2];
    rec.b[0] = s.center_radius[3];
    rec.b[1] = __fmul_rn(s.center_radius[3], s.center_radius[3]);
    rec.b[3] = __uint_as_float(s.material_index);
  } else {
    const uint32_t j = g - ns;
    const tc_gpu_triangle& t = tri[j];
    tag |= j | kTagTriangle;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      rec.a[a] = t.v0[a];
      rec.b[a] = __fsub_rn(t.v1[a], t.v0[a]);
      rec.c[a] = __fsub_rn(t.v2[a], t.v0[a]);
    }
    rec.b[3] = __uint_as_float(t.material_index);
    rec.c[3] = __uint_as_float(attr_flags ? (attr_flags[j] & 3u) : 0u);
  }
  rec.a[3] = __uint_as_float(tag);
  prims[k] = rec;
}

}  // namespace

DeviceBvhBuilder::~DeviceBvhBuilder() { release(); }

void DeviceBvhBuilder::release() {
  for (uint32_t** p : {&node_lo_, &node_hi_, &node_link_, &node_parent_, &seg_node_, &seg_begin_, &seg_end_,
                       &chunk_node_, &chunk_lo_, &chunk_hi_, &last_, &refit_nodes_, &node_keys_, &node_axis_,
                       &keys_[0], &keys_[1], &perm_[0], &perm_[1]}) {
    if (*p) cudaFree(*p);
    *p = nullptr;
  }
  if (item_box_) cudaFree(item_box_);
  item_box_ = nullptr;
  if (sort_temp_) cudaFree(sort_temp_);
  sort_temp_ = nullptr;
  sort_temp_bytes_ = 0;
  n_ = ns_ = nt_ = 0;
}

cudaError_t DeviceBvhBuilder::plan(uint32_t n_spheres, uint32_t n_triangles) {
  if (n_ && ns_ == n_spheres && nt_ == n_triangles) return cudaSuccess;
  release();
  const uint32_t n = n_spheres + n_triangles;
  ns_ = n_spheres;
  nt_ = n_triangles;
  n_ = n;
  // Breadth-first node list of the fixed shape.
  std::vector<uint32_t> lo, hi, first_child;
  level_nodes_.assign(1, 0u);
  if (n > 0) {
    lo.push_back(0);
    hi.push_back(n);
  }
  size_t begin = 0;
  while (begin < lo.size()) {
    const size_t end = lo.size();
    level_nodes_.push_back(uint32_t(end));
    for (size_t i = begin; i < end; ++i) {
      const uint32_t count = hi[i] - lo[i];
      if (count > kMaxLeaf) {
        first_child.push_back(uint32_t(lo.size()));
        const uint32_t split = lo[i] + count / 2;
        lo.push_back(lo[i]);
        hi.push_back(split);
        lo.push_back(split);
        hi.push_back(hi[i]);
      } else {
        first_child.push_back(0xFFFFFFFFu);
      }
    }
    begin = end;
  }
  node_count_ = uint32_t(lo.size());
  depth_ = uint32_t(level_nodes_.size() - 1);
  // Depth-first pair indices of interior nodes (pre-order), parents' slots, leaf links.
  std::vector<uint32_t> link(node_count_), parent(node_count_, kNoParent), last(n, 0u);
  uint32_t next_pair = 0;
  std::vector<uint32_t> stack;
  if (node_count_) stack.push_back(0);
  while (!stack.empty()) {
    const uint32_t i = stack.back();
    stack.pop_back();
    if (first_child[i] == 0xFFFFFFFFu) {
      link[i] = kLeafBit | lo[i];
      last[hi[i] - 1] = 1u;
      continue;
    }
    link[i] = next_pair++;
    const uint32_t l = first_child[i], r = l + 1;
    parent[l] = link[i] << 1;
    parent[r] = (link[i] << 1) | 1u;
    stack.push_back(r);  // visited after the whole left subtree
    stack.push_back(l);
  }
  pair_count_ = next_pair;
  // Sort segments (interior nodes), reduction chunks and refit levels, level by level.
  std::vector<uint32_t> seg_node, seg_begin, seg_end, chunk_node, chunk_lo, chunk_hi, refit;
  level_segments_.assign(1, 0u);
  level_chunks_.assign(1, 0u);
  refit_levels_.assign(1, 0u);
  for (size_t l = 0; l + 1 < level_nodes_.size(); ++l) {
    for (uint32_t i = level_nodes_[l]; i < level_nodes_[l + 1]; ++i) {
      if (!(link[i] & kLeafBit)) {
        seg_node.push_back(i);
        seg_begin.push_back(lo[i]);
        seg_end.push_back(hi[i]);
        refit.push_back(link[i]);
      }
      for (uint32_t p = lo[i]; p < hi[i]; p += kChunk) {
        chunk_node.push_back(i);
        chunk_lo.push_back(p);
        chunk_hi.push_back(std::min(hi[i], p + kChunk));
      }
    }
    level_segments_.push_back(uint32_t(seg_node.size()));
    level_chunks_.push_back(uint32_t(chunk_node.size()));
    if (level_segments_[l + 1] > level_segments_[l]) refit_levels_.push_back(uint32_t(refit.size()));
  }
  cudaError_t e = cudaSuccess;
  auto put = [&](uint32_t*& dst, const std::vector<uint32_t>& src) {
    if (e != cudaSuccess || src.empty()) return;
    e = alloc(dst, src.size());
    if (e == cudaSuccess) e = cudaMemcpy(dst, src.data(), sizeof(uint32_t) * src.size(), cudaMemcpyHostToDevice);
  };
  put(node_lo_, lo);
  put(node_hi_, hi);
  put(node_link_, link);
  put(node_parent_, parent);
  put(seg_node_, seg_node);
  put(seg_begin_, seg_begin);
  put(seg_end_, seg_end);
  put(chunk_node_, chunk_node);
  put(chunk_lo_, chunk_lo);
  put(chunk_hi_, chunk_hi);
  put(last_, last);
  put(refit_nodes_, refit);
  if (e == cudaSuccess && n) e = alloc(item_box_, size_t(9) * n);
  if (e == cudaSuccess && node_count_) e = alloc(node_keys_, size_t(12) * node_count_);
  if (e == cudaSuccess && node_count_) e = alloc(node_axis_, node_count_);
  for (int b = 0; b < 2 && e == cudaSuccess && n; ++b) {
    e = alloc(keys_[b], n);
    if (e == cudaSuccess) e = alloc(perm_[b], n);
  }
  // Temporary storage of the largest segmented sort of any level.
  size_t temp = 0;
  for (size_t l = 0; e == cudaSuccess && l + 1 < level_segments_.size(); ++l) {
    const uint32_t segs = level_segments_[l + 1] - level_segments_[l];
    if (!segs) continue;
    size_t bytes = 0;
    e = cub::DeviceSegmentedSort::StableSortPairs(nullptr, bytes, keys_[0], keys_[1], perm_[0], perm_[1], int(n),
                                                  int(segs), seg_begin_ + level_segments_[l],
                                                  seg_end_ + level_segments_[l]);
    temp = std::max(temp, bytes);
  }
  if (e == cudaSuccess && temp) {
    e = cudaMalloc(&sort_temp_, temp);
    if (e == cudaSuccess) sort_temp_bytes_ = temp;
  }
  if (e != cudaSuccess) release();
  return e;
}

cudaError_t DeviceBvhBuilder::build(const tc_gpu_sphere* spheres, const tc_gpu_triangle* triangles,
                                    const uint32_t* attr_flags, PairNode* pairs, ChildRec* root, PrimRecord* prims,
                                    uint32_t* status, cudaStream_t stream) {
  if (n_ == 0) return cudaErrorInvalidValue;
  cudaError_t e;
  int cur = 0;
  item_boxes_kernel<<<(n_ + 255) / 256, 256, 0, stream>>>(spheres, ns_, triangles, n_, item_box_, perm_[0]);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  for (size_t l = 0; l + 1 < level_nodes_.size(); ++l) {
    const uint32_t n0 = level_nodes_[l], nodes = level_nodes_[l + 1] - n0;
    const uint32_t c0 = level_chunks_[l], chunks = level_chunks_[l + 1] - c0;
    const uint32_t s0 = level_segments_[l], segs = level_segments_[l + 1] - s0;
    init_keys_kernel<<<(12 * nodes + 255) / 256, 256, 0, stream>>>(node_keys_, n0, nodes);
    node_bounds_kernel<<<(chunks + 7) / 8, 256, 0, stream>>>(chunk_node_ + c0, chunk_lo_ + c0, chunk_hi_ + c0, chunks,
                                                             perm_[cur], item_box_, node_keys_);
    if (!segs) continue;
    split_axis_kernel<<<(segs + 255) / 256, 256, 0, stream>>>(seg_node_ + s0, segs, node_keys_, node_axis_, status);
    sort_keys_kernel<<<(chunks + 7) / 8, 256, 0, stream>>>(chunk_node_ + c0, chunk_lo_ + c0, chunk_hi_ + c0, chunks,
                                                           node_link_, node_axis_, perm_[cur], item_box_, keys_[cur]);
    // Positions outside this level's segments keep their order: start from a copy.
    if ((e = cudaMemcpyAsync(perm_[cur ^ 1], perm_[cur], sizeof(uint32_t) * n_, cudaMemcpyDeviceToDevice, stream)) !=
        cudaSuccess)
      return e;
    size_t bytes = sort_temp_bytes_;
    e = cub::DeviceSegmentedSort::StableSortPairs(sort_temp_, bytes, keys_[cur], keys_[cur ^ 1], perm_[cur],
                                                  perm_[cur ^ 1], int(n_), int(segs), seg_begin_ + s0, seg_end_ + s0,
                                                  stream);
    if (e != cudaSuccess) return e;
    cur ^= 1;
  }
  write_nodes_kernel<<<(node_count_ + 255) / 256, 256, 0, stream>>>(node_count_, node_lo_, node_hi_, node_link_,
                                                                     node_parent_, node_keys_, pairs, root);
  write_prims_kernel<<<(n_ + 255) / 256, 256, 0, stream>>>(n_, ns_, perm_[cur], last_, spheres, triangles, attr_flags,
                                                           prims);
  return cudaGetLastError();
}

}  // namespace tcb
