// Host hierarchy build (median split, bit-compatible with crates/toaster-bvh) and conversion
// to the sibling-pair device layout. Compiled with -ffp-contract=off: every bound, centroid and
// padding value must round exactly as the reference's IEEE f32 arithmetic does.
#include "bvh_build.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>

namespace tcb {
namespace {

struct Box {
  float mn[3], mx[3];
};

inline Box empty_box() {
  const float inf = std::numeric_limits<float>::infinity();
  return Box{{inf, inf, inf}, {-inf, -inf, -inf}};
}

inline void grow(Box& b, const float* mn, const float* mx) {
  for (int a = 0; a < 3; ++a) {
    b.mn[a] = std::fmin(b.mn[a], mn[a]);
    b.mx[a] = std::fmax(b.mx[a], mx[a]);
  }
}

// f32::total_cmp order as an unsigned key (sign-magnitude to two's-complement, then biased).
inline uint32_t order_key(float f) {
  int32_t bits;
  std::memcpy(&bits, &f, 4);
  bits ^= static_cast<int32_t>(static_cast<uint32_t>(bits >> 31) >> 1);
  return static_cast<uint32_t>(bits) ^ 0x80000000u;
}

struct Item {
  float mn[3], mx[3], c[3];
  PrimRef ref;
};

// Stable sort of items[lo, hi) by key(axis). Small ranges use std::stable_sort; larger ones a
// stable LSD radix sort (4 x 8-bit digits). Both are stable on the same key, so the permutation
// equals the reference's `sort_by(total_cmp)`.
void stable_sort_axis(std::vector<Item>& items, std::vector<Item>& scratch, size_t lo, size_t hi, int axis) {
  size_t n = hi - lo;
  if (n < 2) return;
  if (n <= 512) {
    std::stable_sort(items.begin() + lo, items.begin() + hi, [axis](const Item& x, const Item& y) {
      return order_key(x.c[axis]) < order_key(y.c[axis]);
    });
    return;
  }
  Item* src = items.data() + lo;
  Item* dst = scratch.data() + lo;
  for (int shift = 0; shift < 32; shift += 8) {
    size_t count[257] = {0};
    for (size_t i = 0; i < n; ++i) count[((order_key(src[i].c[axis]) >> shift) & 255u) + 1]++;
    bool trivial = false;
    for (int d = 1; d <= 256; ++d) {
      if (count[d] == n) trivial = true;
      count[d] += count[d - 1];
    }
    if (trivial) continue;  // every key shares this digit: the pass would be the identity
    for (size_t i = 0; i < n; ++i) dst[count[(order_key(src[i].c[axis]) >> shift) & 255u]++] = src[i];
    std::swap(src, dst);
  }
  if (src != items.data() + lo) std::copy(src, src + n, items.data() + lo);
}

}  // namespace

FlatHierarchy build_median_split(const SphereIn* spheres, size_t n_spheres, const TriangleIn* triangles,
                                 size_t n_triangles, size_t max_leaf) {
  FlatHierarchy out;
  max_leaf = std::max<size_t>(max_leaf, 1);
  const size_t n = n_spheres + n_triangles;
  if (n == 0) return out;
  std::vector<Item> items(n);
  for (size_t i = 0; i < n_spheres; ++i) {
    Item& it = items[i];
    for (int a = 0; a < 3; ++a) {
      it.mn[a] = spheres[i].center[a] - spheres[i].radius;
      it.mx[a] = spheres[i].center[a] + spheres[i].radius;
    }
    it.ref = PrimRef{0u, static_cast<uint32_t>(i)};
  }
  const float pad = 1e-5f;
  for (size_t i = 0; i < n_triangles; ++i) {
    Item& it = items[n_spheres + i];
    const TriangleIn& t = triangles[i];
    for (int a = 0; a < 3; ++a) {
      float lo = std::fmin(std::fmin(t.v[0][a], t.v[1][a]), t.v[2][a]);
      float hi = std::fmax(std::fmax(t.v[0][a], t.v[1][a]), t.v[2][a]);
      it.mn[a] = lo - pad;
      it.mx[a] = hi + pad;
    }
    it.ref = PrimRef{1u, static_cast<uint32_t>(i)};
  }
  for (Item& it : items)
    for (int a = 0; a < 3; ++a) it.c[a] = 0.5f * (it.mn[a] + it.mx[a]);

  std::vector<Item> scratch(n);
  out.nodes.reserve(2 * n);
  out.prims.reserve(n);

  // Explicit depth-first work list. A task is a primitive range plus, for right children, the
  // parent node whose link must receive this node's index once it is emitted.
  struct Task {
    size_t lo, hi;
    int64_t parent_for_right;
  };
  std::vector<Task> work;
  work.push_back(Task{0, n, -1});
  while (!work.empty()) {
    Task task = work.back();
    work.pop_back();
    const uint32_t index = static_cast<uint32_t>(out.nodes.size());
    if (task.parent_for_right >= 0) out.nodes[size_t(task.parent_for_right)].first_or_right = index;

    Box bounds = empty_box();
    for (size_t i = task.lo; i < task.hi; ++i) grow(bounds, items[i].mn, items[i].mx);
    FlatNode node{};
    std::memcpy(node.min, bounds.mn, sizeof(node.min));
    std::memcpy(node.max, bounds.mx, sizeof(node.max));
    const size_t count = task.hi - task.lo;

    bool leaf = count <= max_leaf;
    int axis = 0;
    if (!leaf) {
      Box cb = empty_box();
      for (size_t i = task.lo; i < task.hi; ++i) grow(cb, items[i].c, items[i].c);
      float ex = cb.mx[0] - cb.mn[0], ey = cb.mx[1] - cb.mn[1], ez = cb.mx[2] - cb.mn[2];
      axis = (ex >= ey && ex >= ez) ? 0 : (ey >= ez ? 1 : 2);
      float extent = axis == 0 ? ex : (axis == 1 ? ey : ez);
      leaf = extent <= std::numeric_limits<float>::epsilon();
    }
    if (leaf) {
      node.first_or_right = static_cast<uint32_t>(out.prims.size());
      node.count = static_cast<uint32_t>(count);
      for (size_t i = task.lo; i < task.hi; ++i) out.prims.push_back(items[i].ref);
      out.nodes.push_back(node);
      continue;
    }
    stable_sort_axis(items, scratch, task.lo, task.hi, axis);
    const size_t split = task.lo + count / 2;
    node.first_or_right = 0;
    node.count = 0;
    out.nodes.push_back(node);
    work.push_back(Task{split, task.hi, int64_t(index)});  // right, emitted after the left subtree
    work.push_back(Task{task.lo, split, -1});              // left = index + 1
  }
  return out;
}

bool to_device_layout(const FlatHierarchy& flat, const SphereIn* spheres, const uint32_t* sphere_materials,
                      size_t n_spheres, const TriangleIn* triangles, const uint32_t* triangle_materials,
                      const uint32_t* triangle_attr_flags, size_t n_triangles, DeviceHierarchy& out,
                      std::string& error) {
  out.pairs.clear();
  out.prims.clear();
  out.depth = 0;
  std::memset(&out.root, 0, sizeof(out.root));
  const size_t nn = flat.nodes.size();
  if (nn == 0) {
    // Empty hierarchy: a root that no ray can enter.
    out.root.min_x = out.root.min_y = out.root.min_z = std::numeric_limits<float>::infinity();
    out.root.max_x = out.root.max_y = out.root.max_z = -std::numeric_limits<float>::infinity();
    out.root.link = kLeafBit;
    return true;
  }
  if (n_spheres + n_triangles > kMaxPrimitives) {
    error = "scene has more primitives than the device tag can index";
    return false;
  }
  // Rank interior nodes (pair index) and validate links; depth via a parent-before-child walk.
  std::vector<uint32_t> rank(nn, 0xFFFFFFFFu);
  std::vector<uint32_t> depth(nn, 0);
  uint32_t interior = 0;
  for (size_t i = 0; i < nn; ++i)
    if (flat.nodes[i].count == 0) rank[i] = interior++;
  depth[0] = 1;
  uint32_t max_depth = 1;
  std::vector<uint8_t> seen(nn, 0);
  seen[0] = 1;
  for (size_t i = 0; i < nn; ++i) {
    const FlatNode& node = flat.nodes[i];
    if (!seen[i]) {
      error = "hierarchy node " + std::to_string(i) + " is unreachable";
      return false;
    }
    if (node.count > 0) {
      if (size_t(node.first_or_right) + node.count > flat.prims.size()) {
        error = "leaf " + std::to_string(i) + " references primitives beyond the primitive list";
        return false;
      }
      continue;
    }
    size_t left = i + 1, right = node.first_or_right;
    if (left >= nn || right >= nn || right <= i + 1 || seen[left] || seen[right]) {
      error = "interior node " + std::to_string(i) + " has an invalid child link";
      return false;
    }
    seen[left] = seen[right] = 1;
    depth[left] = depth[right] = depth[i] + 1;
    max_depth = std::max(max_depth, depth[i] + 1);
  }
  if (max_depth > uint32_t(kMaxStack)) {
    error = "hierarchy depth " + std::to_string(max_depth) + " exceeds the traversal stack";
    return false;
  }
  out.depth = max_depth;

  auto child_rec = [&](size_t j) {
    const FlatNode& c = flat.nodes[j];
    ChildRec r{};
    r.min_x = c.min[0]; r.min_y = c.min[1]; r.min_z = c.min[2];
    r.max_x = c.max[0]; r.max_y = c.max[1]; r.max_z = c.max[2];
    r.count = c.count;
    r.link = c.count > 0 ? (kLeafBit | c.first_or_right) : rank[j];
    return r;
  };
  out.root = child_rec(0);
  out.pairs.resize(interior);
  for (size_t i = 0; i < nn; ++i) {
    if (flat.nodes[i].count != 0) continue;
    PairNode& p = out.pairs[rank[i]];
    p.child[0] = child_rec(i + 1);
    p.child[1] = child_rec(flat.nodes[i].first_or_right);
  }

  // Leaf ranges must tile the primitive list exactly once (the last-in-leaf flag ends a leaf).
  std::vector<uint8_t> last(flat.prims.size(), 0);
  std::vector<uint8_t> covered(flat.prims.size(), 0);
  for (size_t i = 0; i < nn; ++i) {
    const FlatNode& node = flat.nodes[i];
    if (node.count == 0) continue;
    for (size_t k = node.first_or_right; k < size_t(node.first_or_right) + node.count; ++k) {
      if (covered[k]) {
        error = "leaf ranges overlap at primitive slot " + std::to_string(k);
        return false;
      }
      covered[k] = 1;
    }
    last[node.first_or_right + node.count - 1] = 1;
  }
  for (size_t k = 0; k < covered.size(); ++k) {
    if (!covered[k]) {
      error = "primitive slot " + std::to_string(k) + " is in no leaf";
      return false;
    }
  }
  out.prims.resize(flat.prims.size());
  for (size_t k = 0; k < flat.prims.size(); ++k) {
    const PrimRef& r = flat.prims[k];
    PrimRecord rec{};
    uint32_t tag = r.index | (last[k] ? kTagLast : 0u);
    if (r.kind == 0) {
      if (r.index >= n_spheres) {
        error = "primitive reference to sphere " + std::to_string(r.index) + " is out of range";
        return false;
      }
      const SphereIn& s = spheres[r.index];
      rec.a[0] = s.center[0]; rec.a[1] = s.center[1]; rec.a[2] = s.center[2];
      std::memcpy(&rec.a[3], &tag, 4);
      rec.b[0] = s.radius;
      rec.b[1] = s.radius * s.radius;
      uint32_t m = sphere_materials ? sphere_materials[r.index] : 0u;
      std::memcpy(&rec.b[3], &m, 4);
    } else if (r.kind == 1) {
      if (r.index >= n_triangles) {
        error = "primitive reference to triangle " + std::to_string(r.index) + " is out of range";
        return false;
      }
      tag |= kTagTriangle;
      const TriangleIn& t = triangles[r.index];
      rec.a[0] = t.v[0][0]; rec.a[1] = t.v[0][1]; rec.a[2] = t.v[0][2];
      std::memcpy(&rec.a[3], &tag, 4);
      for (int a = 0; a < 3; ++a) {
        rec.b[a] = t.v[1][a] - t.v[0][a];
        rec.c[a] = t.v[2][a] - t.v[0][a];
      }
      uint32_t m = triangle_materials ? triangle_materials[r.index] : 0u;
      std::memcpy(&rec.b[3], &m, 4);
      uint32_t f = triangle_attr_flags ? triangle_attr_flags[r.index] : 0u;
      std::memcpy(&rec.c[3], &f, 4);
    } else {
      error = "primitive reference kind " + std::to_string(r.kind) + " is neither sphere (0) nor triangle (1)";
      return false;
    }
    out.prims[k] = rec;
  }
  return true;
}

}  // namespace tcb
