// Ray/primitive tests and ordered BVH traversal (device).
//
// Every operation that decides a hit or its distance uses explicitly rounded IEEE intrinsics
// (__fadd_rn, __fsub_rn, __fmul_rn, __frcp_rn, __fdiv_rn, __fsqrt_rn) so the compiler cannot
// fuse them into FMAs. This reproduces, bit for bit, the f32 arithmetic of
//   crates/toaster-bvh/src/aabb.rs:74-110            (slab test)
//   crates/toaster-cpu/src/intersect.rs:28-68        (sphere)
//   crates/toaster-cpu/src/intersect.rs:87-120       (Moller-Trumbore)
//   crates/toaster-cpu/src/intersect.rs:172-263,322  (ordered traversal, entry distance)
// assuming glam's scalar Vec3 (dot left to right, cross = a.y*b.z - b.y*a.z ...).
#ifndef TOASTER_B200_TRAVERSE_CUH
#define TOASTER_B200_TRAVERSE_CUH

#include <cuda_runtime.h>
#include <stdint.h>

#include "layout.h"

namespace tcb {

struct RayQ {
  float ox, oy, oz;
  float dx, dy, dz;
  float ix, iy, iz;   // 1/d, IEEE (f32::recip)
  bool sx, sy, sz;    // direction sign bits: choose the near plane without a swap
};

__device__ __forceinline__ RayQ make_ray(float ox, float oy, float oz, float dx, float dy, float dz) {
  RayQ r;
  r.ox = ox; r.oy = oy; r.oz = oz;
  r.dx = dx; r.dy = dy; r.dz = dz;
  r.ix = __frcp_rn(dx); r.iy = __frcp_rn(dy); r.iz = __frcp_rn(dz);
  r.sx = signbit(dx); r.sy = signbit(dy); r.sz = signbit(dz);
  return r;
}

// Slab test of one child box against [tmin, closest]. Returns the hit flag; `entry` is the
// reference's entry_distance (intersect.rs:322-338) and `tn` = max(tmin, entry), the value the
// reference's pop-time re-test compares against `closest`.
//
// Equivalence with aabb.rs: for a finite 1/d the near plane is fixed by the sign of d, and
// rounding is monotone, so the reference's `if near > far swap` picks the same pair. For an
// infinite 1/d (the reference's "parallel" branch) the products are +-inf when the origin is
// outside the slab (forcing a miss) and -inf/NaN when inside (dropped by fmaxf/fminf), which is
// exactly "reject if o < lo || o > hi, else skip the axis".
__device__ __forceinline__ bool box_test(float lox, float loy, float loz, float hix, float hiy, float hiz,
                                         const RayQ& r, float tmin, float closest, float& entry, float& tn) {
  const float ax = __fmul_rn(__fsub_rn(lox, r.ox), r.ix);
  const float bx = __fmul_rn(__fsub_rn(hix, r.ox), r.ix);
  const float ay = __fmul_rn(__fsub_rn(loy, r.oy), r.iy);
  const float by = __fmul_rn(__fsub_rn(hiy, r.oy), r.iy);
  const float az = __fmul_rn(__fsub_rn(loz, r.oz), r.iz);
  const float bz = __fmul_rn(__fsub_rn(hiz, r.oz), r.iz);
  const float nx = r.sx ? bx : ax, fx = r.sx ? ax : bx;
  const float ny = r.sy ? by : ay, fy = r.sy ? ay : by;
  const float nz = r.sz ? bz : az, fz = r.sz ? az : bz;
  entry = fmaxf(fmaxf(nx, ny), nz);
  tn = fmaxf(entry, tmin);
  const float tf = fminf(fminf(fx, fy), fminf(fz, closest));
  return tf >= tn;
}

// intersect.rs:87-120: double-sided Moller-Trumbore with eps 1e-8 and inclusive [tmin, tmax].
__device__ __forceinline__ bool hit_triangle(const RayQ& r, float4 A, float4 B, float4 C, float tmin, float tmax,
                                             float& t_out) {
  const float e1x = B.x, e1y = B.y, e1z = B.z;
  const float e2x = C.x, e2y = C.y, e2z = C.z;
  // p = d x e2
  const float px = __fsub_rn(__fmul_rn(r.dy, e2z), __fmul_rn(e2y, r.dz));
  const float py = __fsub_rn(__fmul_rn(r.dz, e2x), __fmul_rn(e2z, r.dx));
  const float pz = __fsub_rn(__fmul_rn(r.dx, e2y), __fmul_rn(e2x, r.dy));
  const float det = __fadd_rn(__fadd_rn(__fmul_rn(e1x, px), __fmul_rn(e1y, py)), __fmul_rn(e1z, pz));
  if (fabsf(det) < 1e-8f) return false;
  const float inv = __frcp_rn(det);
  const float sx = __fsub_rn(r.ox, A.x), sy = __fsub_rn(r.oy, A.y), sz = __fsub_rn(r.oz, A.z);
  const float u = __fmul_rn(__fadd_rn(__fadd_rn(__fmul_rn(sx, px), __fmul_rn(sy, py)), __fmul_rn(sz, pz)), inv);
  if (!(u >= 0.0f && u <= 1.0f)) return false;
  // q = s x e1
  const float qx = __fsub_rn(__fmul_rn(sy, e1z), __fmul_rn(e1y, sz));
  const float qy = __fsub_rn(__fmul_rn(sz, e1x), __fmul_rn(e1z, sx));
  const float qz = __fsub_rn(__fmul_rn(sx, e1y), __fmul_rn(e1x, sy));
  const float v = __fmul_rn(__fadd_rn(__fadd_rn(__fmul_rn(r.dx, qx), __fmul_rn(r.dy, qy)), __fmul_rn(r.dz, qz)), inv);
  if (v < 0.0f || __fadd_rn(u, v) > 1.0f) return false;
  const float t = __fmul_rn(__fadd_rn(__fadd_rn(__fmul_rn(e2x, qx), __fmul_rn(e2y, qy)), __fmul_rn(e2z, qz)), inv);
  if (t < tmin || t > tmax) return false;
  t_out = t;
  return true;
}

// intersect.rs:28-50: half-b quadratic, near root else far root, inclusive [tmin, tmax].
__device__ __forceinline__ bool hit_sphere(const RayQ& r, float4 A, float4 B, float tmin, float tmax,
                                           float& t_out) {
  const float ox = __fsub_rn(r.ox, A.x), oy = __fsub_rn(r.oy, A.y), oz = __fsub_rn(r.oz, A.z);
  const float a = __fadd_rn(__fadd_rn(__fmul_rn(r.dx, r.dx), __fmul_rn(r.dy, r.dy)), __fmul_rn(r.dz, r.dz));
  const float hb = __fadd_rn(__fadd_rn(__fmul_rn(ox, r.dx), __fmul_rn(oy, r.dy)), __fmul_rn(oz, r.dz));
  const float c = __fsub_rn(__fadd_rn(__fadd_rn(__fmul_rn(ox, ox), __fmul_rn(oy, oy)), __fmul_rn(oz, oz)), B.y);
  const float disc = __fsub_rn(__fmul_rn(hb, hb), __fmul_rn(a, c));
  if (disc < 0.0f) return false;
  const float sq = __fsqrt_rn(disc);
  float t = __fdiv_rn(__fsub_rn(-hb, sq), a);
  if (t < tmin || t > tmax) {
    t = __fdiv_rn(__fadd_rn(-hb, sq), a);
    if (t < tmin || t > tmax) return false;
  }
  t_out = t;
  return true;
}

// FP32 watertight ray/triangle test (Woop, Benthin and Wald, "Watertight Ray/Triangle
// Intersection", JCGT 2(1), 2013): a non-parity option. The ray is sheared so that it runs along
// +z from the origin; the triangle's vertices are projected into that frame and the three 2-D
// edge functions decide the hit, recomputed in double when one is exactly zero. Every product and
// sum is rounded on its own, so two triangles sharing an edge evaluate its edge function from the
// same projected vertices to exactly opposite values: a ray cannot pass between them.
struct RayW {
  int kx, ky, kz;   // the dominant direction axis is kz; kx, ky complete a right-handed frame
  float sx, sy, sz; // shear constants d[kx]/d[kz], d[ky]/d[kz], 1/d[kz]
};

__device__ __forceinline__ float axis_of(float x, float y, float z, int k) { return k == 0 ? x : (k == 1 ? y : z); }

__device__ __forceinline__ RayW make_ray_watertight(const RayQ& r) {
  const float ax = fabsf(r.dx), ay = fabsf(r.dy), az = fabsf(r.dz);
  RayW w;
  w.kz = ax > ay ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
  w.kx = w.kz == 2 ? 0 : w.kz + 1;
  w.ky = w.kx == 2 ? 0 : w.kx + 1;
  const float dz = axis_of(r.dx, r.dy, r.dz, w.kz);
  if (dz < 0.0f) {  // keeps the winding, so the edge-function signs mean the same for every ray
    const int t = w.kx;
    w.kx = w.ky;
    w.ky = t;
  }
  w.sx = __fdiv_rn(axis_of(r.dx, r.dy, r.dz, w.kx), dz);
  w.sy = __fdiv_rn(axis_of(r.dx, r.dy, r.dz, w.ky), dz);
  w.sz = __frcp_rn(dz);
  return w;
}

// Double-sided watertight test of triangle (v0, v1, v2) accepting t in [tmin, tmax].
__device__ __forceinline__ bool hit_triangle_watertight(const RayQ& r, const RayW& w, float4 v0, float4 v1, float4 v2,
                                                        float tmin, float tmax, float& t_out) {
  const float Ax0 = __fsub_rn(v0.x, r.ox), Ay0 = __fsub_rn(v0.y, r.oy), Az0 = __fsub_rn(v0.z, r.oz);
  const float Bx0 = __fsub_rn(v1.x, r.ox), By0 = __fsub_rn(v1.y, r.oy), Bz0 = __fsub_rn(v1.z, r.oz);
  const float Cx0 = __fsub_rn(v2.x, r.ox), Cy0 = __fsub_rn(v2.y, r.oy), Cz0 = __fsub_rn(v2.z, r.oz);
  const float Ak = axis_of(Ax0, Ay0, Az0, w.kz), Bk = axis_of(Bx0, By0, Bz0, w.kz), Ck = axis_of(Cx0, Cy0, Cz0, w.kz);
  const float Ax = __fsub_rn(axis_of(Ax0, Ay0, Az0, w.kx), __fmul_rn(w.sx, Ak));
  const float Ay = __fsub_rn(axis_of(Ax0, Ay0, Az0, w.ky), __fmul_rn(w.sy, Ak));
  const float Bx = __fsub_rn(axis_of(Bx0, By0, Bz0, w.kx), __fmul_rn(w.sx, Bk));
  const float By = __fsub_rn(axis_of(Bx0, By0, Bz0, w.ky), __fmul_rn(w.sy, Bk));
  const float Cx = __fsub_rn(axis_of(Cx0, Cy0, Cz0, w.kx), __fmul_rn(w.sx, Ck));
  const float Cy = __fsub_rn(axis_of(Cx0, Cy0, Cz0, w.ky), __fmul_rn(w.sy, Ck));
  float U = __fsub_rn(__fmul_rn(Cx, By), __fmul_rn(Cy, Bx));
  float V = __fsub_rn(__fmul_rn(Ax, Cy), __fmul_rn(Ay, Cx));
  float W = __fsub_rn(__fmul_rn(Bx, Ay), __fmul_rn(By, Ax));
  if (U == 0.0f || V == 0.0f || W == 0.0f) {
    // On an edge in single precision: decide with the exact products of the same inputs.
    U = float(__dsub_rn(__dmul_rn(double(Cx), double(By)), __dmul_rn(double(Cy), double(Bx))));
    V = float(__dsub_rn(__dmul_rn(double(Ax), double(Cy)), __dmul_rn(double(Ay), double(Cx))));
    W = float(__dsub_rn(__dmul_rn(double(Bx), double(Ay)), __dmul_rn(double(By), double(Ax))));
  }
  if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
  const float det = __fadd_rn(__fadd_rn(U, V), W);
  if (det == 0.0f) return false;
  const float T = __fadd_rn(__fadd_rn(__fmul_rn(U, __fmul_rn(w.sz, Ak)), __fmul_rn(V, __fmul_rn(w.sz, Bk))),
                            __fmul_rn(W, __fmul_rn(w.sz, Ck)));
  const float t = __fdiv_rn(T, det);
  if (!(t >= tmin && t <= tmax)) return false;
  t_out = t;
  return true;
}

struct TraceResult {
  float t;        // closest accepted distance (or tmax when nothing was accepted)
  uint32_t tag;   // PrimRecord tag of the accepted primitive
  uint32_t rec;   // PrimRecord index of the accepted primitive
};

constexpr uint32_t kNoNode = 0xFFFFFFFFu;  // never a valid link (leaf links stay below 0xC0000000)

// Ordered closest-hit traversal (any_hit = false) or first-hit occlusion query (any_hit = true)
// over the sibling-pair hierarchy, accepting primitives in [tmin, tmax].
//
// Closest-hit mode reproduces intersect.rs:172-263 exactly: children are tested against the
// current closest distance; when both are hit the one with the smaller entry distance is taken
// first (strictly smaller; ties take the right child first, as the reference's push order
// does); a stacked child is re-tested on pop, which for a box that passed at push time reduces
// to `tn <= closest`; leaf primitives are tested in leaf order and accepted on `t <= closest`.
// Stack depth never exceeds the hierarchy depth, which the host checks against kMaxStack.
//
// The loop is the "while-while" form: an inner loop descends through interior nodes until every
// lane holds a leaf (or has finished), then the lanes test their leaves together. Each ray still
// visits exactly the nodes, in exactly the order, of the sequential algorithm.
//
// The traversal is resumable, for persistent kernels that refill finished lanes while other lanes
// of the warp are still traversing ("dynamic ray fetching"): a lane can hand control back after
// any leaf, with its state in Traversal and its stack owned by the caller. Stack entries pack the
// node reference and its entry distance; the first `n_short` live in shared memory
// (`short_stack`, this thread's slots `stride` apart so a warp's accesses fall in distinct
// banks), deeper ones in local memory.
//
// Only what must survive between calls is kept here (five words); the ray itself stays with the
// caller, which passes it again on every call, so a persistent kernel holds no second copy of it
// while the lane shades.
struct Traversal {
  uint32_t cur;      // next node or leaf reference; kNoNode when the traversal is over
  int sp;
  float closest;
  uint32_t tag;      // PrimRecord tag of the accepted primitive
  uint32_t rec;      // PrimRecord index of the accepted primitive; kNoNode while none is accepted
  __device__ __forceinline__ bool found() const { return rec != kNoNode; }
};

__device__ __forceinline__ void trav_start(Traversal& T, const ChildRec& root, const RayQ& r, float tmin, float tmax) {
  T.closest = tmax;
  T.sp = 0;
  T.tag = 0u;
  T.rec = kNoNode;
  float entry, tn;
  T.cur = box_test(root.min_x, root.min_y, root.min_z, root.max_x, root.max_y, root.max_z, r, tmin, tmax, entry, tn)
              ? root.link
              : kNoNode;
}

// One step of a traversal that is not over: descend to the next leaf, test its primitives in
// leaf order, and pop the next stacked node that survives the re-test against the updated closest
// distance. The stack is the caller's: `st_local` (kMaxStack entries in local memory) below
// `short_stack` (n_short entries in shared memory, `stride` apart).
__device__ __forceinline__ void trav_step(Traversal& T, const RayQ& r, float tmin, bool any_hit,
                                          const PairNode* __restrict__ pairs, const PrimRecord* __restrict__ prims,
                                          uint2* st_local, uint2* short_stack, int n_short, int stride,
                                          uint32_t& node_visits) {
  uint32_t cur = T.cur;
  int sp = T.sp;
  float closest = T.closest;
  auto push = [&](uint32_t ref, float t) {
    const uint2 e = make_uint2(ref, __float_as_uint(t));
    if (sp < n_short) short_stack[sp * stride] = e;
    else st_local[sp - n_short] = e;
    ++sp;
  };
  auto top = [&]() -> uint2 { return sp < n_short ? short_stack[sp * stride] : st_local[sp - n_short]; };
  // Descend to a leaf.
  while ((cur & kLeafBit) == 0u) {
    ++node_visits;
    const float4* q = reinterpret_cast<const float4*>(pairs + cur);
    const float4 a0 = __ldg(q), a1 = __ldg(q + 1), b0 = __ldg(q + 2), b1 = __ldg(q + 3);
    float ea, ta, eb, tb;
    const bool ha = box_test(a0.x, a0.y, a0.z, a1.x, a1.y, a1.z, r, tmin, closest, ea, ta);
    const bool hb = box_test(b0.x, b0.y, b0.z, b1.x, b1.y, b1.z, r, tmin, closest, eb, tb);
    const uint32_t la = __float_as_uint(a0.w), lb = __float_as_uint(b0.w);
    if (ha && hb) {
      const bool a_first = ea < eb;
      push(a_first ? lb : la, a_first ? tb : ta);
      cur = a_first ? la : lb;
    } else if (ha) {
      cur = la;
    } else if (hb) {
      cur = lb;
    } else {
      cur = kNoNode;
      while (sp > 0) {
        --sp;
        const uint2 e = top();
        if (__uint_as_float(e.y) <= closest) {
          cur = e.x;
          break;
        }
      }
      if (cur == kNoNode) break;
    }
  }
  if (cur != kNoNode) {
    // Leaf: primitives in leaf order.
    uint32_t k = cur & ~kLeafBit;
    bool stop = false;
    for (;;) {
      const float4* p = reinterpret_cast<const float4*>(prims + k);
      const float4 A = __ldg(p);
      const float4 B = __ldg(p + 1);
      const uint32_t tag = __float_as_uint(A.w);
      float t;
      bool ok;
      if (tag & kTagTriangle) {
        const float4 C = __ldg(p + 2);
        ok = hit_triangle(r, A, B, C, tmin, closest, t);
      } else {
        ok = hit_sphere(r, A, B, tmin, closest, t);
      }
      if (ok) {
        closest = t;
        T.tag = tag;
        T.rec = k;
        if (any_hit) {
          stop = true;
          break;
        }
      }
      if (tag & kTagLast) break;
      ++k;
    }
    cur = kNoNode;
    while (!stop && sp > 0) {
      --sp;
      const uint2 e = top();
      if (__uint_as_float(e.y) <= closest) {
        cur = e.x;
        break;
      }
    }
  }
  T.cur = cur;
  T.sp = sp;
  T.closest = closest;
}

// Whole traversal of one ray in one call (the form every launch uses unless it pauses traversals
// for refills): the same node and primitive order as trav_step's, with the state in registers and
// the stack in local memory.
//
// kWatertight selects the watertight triangle test (hit_triangle_watertight) with the vertices of
// leaf-order primitive record k at verts[3k..3k+2]; the default is the reference's Moller-Trumbore.
template <bool kWatertight = false>
__device__ __forceinline__ bool trace_ray(const PairNode* __restrict__ pairs, const PrimRecord* __restrict__ prims,
                                          const ChildRec& root, const RayQ& r, float tmin, float tmax,
                                          bool any_hit, TraceResult& res, uint32_t& node_visits,
                                          const float4* __restrict__ verts = nullptr) {
  RayW rw;
  if constexpr (kWatertight) rw = make_ray_watertight(r);
  float closest = tmax;
  bool found = false;
  float entry, tn;
  if (!box_test(root.min_x, root.min_y, root.min_z, root.max_x, root.max_y, root.max_z, r, tmin, closest, entry, tn))
    return false;
  uint32_t st_ref[kMaxStack];
  float st_tn[kMaxStack];
  int sp = 0;
  uint32_t cur = root.link;
  while (cur != kNoNode) {
    // Descend: interior nodes until a leaf is reached or the stack is exhausted.
    while ((cur & kLeafBit) == 0u) {
      ++node_visits;
      const float4* q = reinterpret_cast<const float4*>(pairs + cur);
      const float4 a0 = __ldg(q), a1 = __ldg(q + 1), b0 = __ldg(q + 2), b1 = __ldg(q + 3);
      float ea, ta, eb, tb;
      const bool ha = box_test(a0.x, a0.y, a0.z, a1.x, a1.y, a1.z, r, tmin, closest, ea, ta);
      const bool hb = box_test(b0.x, b0.y, b0.z, b1.x, b1.y, b1.z, r, tmin, closest, eb, tb);
      const uint32_t la = __float_as_uint(a0.w), lb = __float_as_uint(b0.w);
      if (ha && hb) {
        const bool a_first = ea < eb;
        st_ref[sp] = a_first ? lb : la;
        st_tn[sp] = a_first ? tb : ta;
        ++sp;
        cur = a_first ? la : lb;
      } else if (ha) {
        cur = la;
      } else if (hb) {
        cur = lb;
      } else {
        cur = kNoNode;
        while (sp > 0) {
          --sp;
          if (st_tn[sp] <= closest) {
            cur = st_ref[sp];
            break;
          }
        }
        if (cur == kNoNode) break;
      }
    }
    if (cur == kNoNode) break;
    // Leaf: primitives in leaf order.
    uint32_t k = cur & ~kLeafBit;
    for (;;) {
      const float4* p = reinterpret_cast<const float4*>(prims + k);
      const float4 A = __ldg(p);
      const float4 B = __ldg(p + 1);
      const uint32_t tag = __float_as_uint(A.w);
      float t;
      bool ok;
      if (tag & kTagTriangle) {
        if constexpr (kWatertight) {
          const float4* v = verts + 3 * size_t(k);
          ok = hit_triangle_watertight(r, rw, __ldg(v), __ldg(v + 1), __ldg(v + 2), tmin, closest, t);
        } else {
          const float4 C = __ldg(p + 2);
          ok = hit_triangle(r, A, B, C, tmin, closest, t);
        }
      } else {
        ok = hit_sphere(r, A, B, tmin, closest, t);
      }
      if (ok) {
        closest = t;
        found = true;
        res.tag = tag;
        res.rec = k;
        if (any_hit) break;
      }
      if (tag & kTagLast) break;
      ++k;
    }
    if (any_hit && found) break;
    // Next stacked node that survives the re-test against the updated closest distance.
    cur = kNoNode;
    while (sp > 0) {
      --sp;
      if (st_tn[sp] <= closest) {
        cur = st_ref[sp];
        break;
      }
    }
  }
  res.t = closest;
  return found;
}

// Advances the unfinished traversals of the warp one leaf visit per round. It returns when all
// of them are done, or early when fewer than `min_active` lanes are still traversing and at
// least one lane can use the pause: a lane whose traversal is over while it still has work to
// take (`can_refill`). Lanes that cannot take work never stop the others, so every call makes
// progress and the warp never pauses for nothing. Every lane of the warp must call it together.
__device__ __forceinline__ void trav_advance(Traversal& T, const RayQ& r, float tmin, bool any_hit,
                                             const PairNode* __restrict__ pairs,
                                             const PrimRecord* __restrict__ prims, uint2* st_local, uint2* short_stack,
                                             int n_short, int stride, int min_active, bool can_refill,
                                             uint32_t& node_visits) {
  for (;;) {
    const unsigned act = __ballot_sync(0xffffffffu, T.cur != kNoNode);
    if (act == 0u) return;
    const unsigned ready = __ballot_sync(0xffffffffu, T.cur == kNoNode && can_refill);
    if (ready != 0u && __popc(act) < min_active) return;
    if (T.cur != kNoNode)
      trav_step(T, r, tmin, any_hit, pairs, prims, st_local, short_stack, n_short, stride, node_visits);
  }
}

}  // namespace tcb

#endif
