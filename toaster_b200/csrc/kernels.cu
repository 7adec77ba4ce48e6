// CUDA kernels of the toaster B200 path tracer (sm_100a).
//
//   trace_closest_kernel  closest-hit parity hook: one ray per thread, exact traversal
//   wf_logic_kernel       wavefront schedule, one slot per thread: shadow-ray results, the last
//                         hit (miss, emission or the slot's material queue), finished paths into
//                         the FP64 sums, new camera paths in free slots
//   wf_shade_kernel       wavefront schedule: the material queues in order (BSDF, light and
//                         environment NEE, the next ray), guided or recording when asked
//   wf_trace_kernel       wavefront schedule: extension rays then shadow rays, 32 per warp
//   wf_sort_* kernels     optional ray sorting before tracing (kind, octant, origin bucket)
//   render_kernel         persistent path-tracing megakernel (small frames, batched launches,
//                         captured animation frames)
//   env_* kernels         FP64 prefix sums and Walker alias tables of the environment's
//                         importance distribution
//   resolve_kernel        FP64 sums -> linear-HDR float4 averages
//
// The estimator is the one of crates/toaster-cpu/src/integrator.rs:99-244. The megakernel writes
// it as an iterative state machine so that every lane issues exactly one ray per loop iteration
// (extension, light shadow or environment shadow). All lanes therefore run the traversal loop
// together. Optionally (the kPause instantiation) a warp pauses it as soon as too few lanes are
// still traversing: the finished lanes consume their hit and produce their next ray while the
// others keep their traversal state (dynamic ray fetching). Idle lanes are refilled with new
// (pixel, sample-range) work items through one warp-aggregated atomic (ballot + popc + shuffle).
// The wavefront schedule splits the same estimator into the three launches above over per-path
// state in device memory; both draw a path's random numbers in the same order.
#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

#include <algorithm>

#include "device_scene.h"
#include "guide.h"
#include "traverse.cuh"

namespace tcb {

constexpr float kPiF = 3.14159265358979323846f;
constexpr float kRayEps = 0.001f;           // integrator.rs:11 RAY_EPSILON
constexpr float kOneMinusEps = 0.99999994f;  // 1 - f32::EPSILON (environment.rs:281-287)

// ------------------------------------------------------------------------ small vector math
struct V3 {
  float x, y, z;
};
__device__ __forceinline__ V3 mk(float x, float y, float z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 operator-(V3 a) { return V3{-a.x, -a.y, -a.z}; }
__device__ __forceinline__ V3 operator*(V3 a, V3 b) { return V3{a.x * b.x, a.y * b.y, a.z * b.z}; }
__device__ __forceinline__ V3 operator*(V3 a, float s) { return V3{a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ V3 operator*(float s, V3 a) { return V3{a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 cross(V3 a, V3 b) {
  return V3{a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
__device__ __forceinline__ V3 normalize(V3 a) { return a * rsqrtf(dot(a, a)); }
__device__ __forceinline__ V3 lerp3(V3 a, V3 b, float s) { return a + (b - a) * s; }

// ------------------------------------------------------------------------ random numbers
// PCG32 (O'Neill 2014, XSH-RR) seeded per (frame, pixel, sample) through SplitMix64, so any
// sample of any pixel can be regenerated independently of scheduling.
__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
__device__ __forceinline__ float luminance(V3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }
struct Pcg {
  uint64_t state, inc;
  __device__ __forceinline__ void seed(uint32_t frame, uint32_t pixel, uint32_t sample) {
    const uint64_t k = splitmix64(splitmix64((uint64_t(frame) << 32) ^ pixel ^ 0xA0761D6478BD642Full) ^ sample);
    state = k;
    inc = splitmix64(k) | 1ull;
  }
  __device__ __forceinline__ uint32_t next() {
    const uint64_t old = state;
    state = old * 6364136223846793005ull + inc;
    const uint32_t xs = uint32_t(((old >> 18u) ^ old) >> 27u);
    const uint32_t rot = uint32_t(old >> 59u);
    return (xs >> rot) | (xs << ((32u - rot) & 31u));
  }
  __device__ __forceinline__ float uniform() { return float(next() >> 8) * (1.0f / 16777216.0f); }
};

// ------------------------------------------------------------------------ environment
__device__ __forceinline__ float unit_interval(float v) { return fminf(fmaxf(v, 0.0f), kOneMinusEps); }

__device__ __forceinline__ float rem_euclid1(float a) {
  float r = fmodf(a, 1.0f);
  return r < 0.0f ? r + 1.0f : r;
}

// environment.rs:237-241: horizontal wrap, vertical clamp.
__device__ __forceinline__ V3 env_texel(const DevScene& s, int x, int y) {
  const int w = int(s.env_width), h = int(s.env_height);
  x %= w;
  if (x < 0) x += w;
  y = min(max(y, 0), h - 1);
  const float4 t = __ldg(s.env_rgb + size_t(y) * s.env_width + x);
  return mk(t.x, t.y, t.z);
}

// environment.rs:132-152: bilinear lat-long lookup times intensity.
__device__ V3 env_radiance(const DevScene& s, V3 d) {
  const float l2 = dot(d, d);
  if (!(l2 > 0.0f) || isinf(l2)) return mk(0.f, 0.f, 0.f);
  d = d * rsqrtf(l2);
  const float u = rem_euclid1(atan2f(d.z, d.x) / (2.0f * kPiF) + 0.5f + s.env_rotation_turns);
  const float v = acosf(fminf(fmaxf(d.y, -1.0f), 1.0f)) / kPiF;
  const float x = u * float(s.env_width) - 0.5f;
  const float y = v * float(s.env_height) - 0.5f;
  const float fx = floorf(x), fy = floorf(y);
  const int x0 = int(fx), y0 = int(fy);
  const float ax = x - fx, ay = y - fy;
  const V3 top = lerp3(env_texel(s, x0, y0), env_texel(s, x0 + 1, y0), ax);
  const V3 bottom = lerp3(env_texel(s, x0, y0 + 1), env_texel(s, x0 + 1, y0 + 1), ax);
  return lerp3(top, bottom, ay) * s.env_intensity;
}

// environment.rs:193-200 and :225-234: density per steradian of the importance distribution.
__device__ float env_pdf(const DevScene& s, V3 d) {
  if (!s.env_sampleable) return 0.0f;
  const float l2 = dot(d, d);
  if (!(l2 > 0.0f) || isinf(l2)) return 0.0f;
  d = d * rsqrtf(l2);
  const float u = rem_euclid1(atan2f(d.z, d.x) / (2.0f * kPiF) + 0.5f + s.env_rotation_turns);
  const float theta = acosf(fminf(fmaxf(d.y, -1.0f), 1.0f));
  const float v = theta / kPiF;
  const uint32_t x = uint32_t(floorf(u * float(s.env_width))) % s.env_width;
  const uint32_t y = min(uint32_t(floorf(v * float(s.env_height))), s.env_height - 1);
  const float p = __ldg(s.env_pdf + size_t(y) * s.env_width + x);
  const float st = sinf(theta);
  return (p > 0.0f && st > 0.0f) ? p / st : 0.0f;
}

// environment.rs:159-189: a texel drawn with the importance distribution's probability, then a
// uniform point inside it. The reference inverts one flat CDF by binary search; here the texel
// comes from two Walker alias tables (the marginal over rows, then the row's conditional over
// columns: two dependent loads instead of a search of about twenty), with the same texel
// probabilities. u1 draws the row, u2 the column, and the column draw's leftover fraction
// (uniform in [0, 1) given the column) places the point across the texel; u3 places it down.
__device__ bool env_sample(const DevScene& s, float u1, float u2, float u3, V3& dir, V3& rad, float& pdf) {
  if (!s.env_sampleable) return false;
  const float fy = unit_interval(u1) * float(s.env_height);
  uint32_t y = min(uint32_t(fy), s.env_height - 1);
  const uint2 ry = __ldg(s.env_alias_marg + y);
  if (!(fy - float(y) < __uint_as_float(ry.x))) y = ry.y;
  const float fx = unit_interval(u2) * float(s.env_width);
  uint32_t x = min(uint32_t(fx), s.env_width - 1);
  const float g = fx - float(x);
  const uint2 rx = __ldg(s.env_alias_cond + size_t(y) * s.env_width + x);
  const float keep = __uint_as_float(rx.x);
  float jx;
  if (g < keep) {
    jx = g / keep;
  } else {
    x = rx.y;
    jx = (g - keep) / (1.0f - keep);
  }
  const float u = (float(x) + unit_interval(jx)) / float(s.env_width);
  const float v = (float(y) + unit_interval(u3)) / float(s.env_height);
  const float theta = kPiF * v;
  const float phi = 2.0f * kPiF * (u - 0.5f - s.env_rotation_turns);
  float st, ct, sp, cp;
  sincosf(theta, &st, &ct);
  sincosf(phi, &sp, &cp);
  dir = mk(st * cp, ct, st * sp);
  const float p = __ldg(s.env_pdf + size_t(y) * s.env_width + x);
  pdf = (p > 0.0f && st > 0.0f) ? p / st : 0.0f;
  rad = env_radiance(s, dir);
  return true;
}

// ------------------------------------------------------------------------ materials
__device__ __forceinline__ float srgb_to_linear(float v) {
  return v <= 0.04045f ? v / 12.92f : powf((v + 0.055f) / 1.055f, 2.4f);
}
__device__ V3 texel_linear(const DevScene& s, const DevMaterial& m, int x, int y) {
  const int w = int(m.tex_width), h = int(m.tex_height);
  x %= w; if (x < 0) x += w;
  y %= h; if (y < 0) y += h;
  const uint32_t px = __ldg(s.texels + m.tex_offset + uint32_t(y) * m.tex_width + uint32_t(x));
  const float k = 1.0f / 255.0f;
  return mk(srgb_to_linear(float(px & 255u) * k), srgb_to_linear(float((px >> 8) & 255u) * k),
            srgb_to_linear(float((px >> 16) & 255u) * k));
}
// Textured diffuse albedo (integrator.rs:340-350; pathtrace_spheres.wgsl:247-273).
__device__ V3 base_color(const DevScene& s, const DevMaterial& m, float tu, float tv) {
  const V3 a = mk(m.albedo[0], m.albedo[1], m.albedo[2]);
  if (m.tex_width == 0 || m.tex_height == 0 || s.texels == nullptr) return a;
  const float u = tu - floorf(tu), v = tv - floorf(tv);
  const float px = u * float(m.tex_width) - 0.5f, py = v * float(m.tex_height) - 0.5f;
  const int bx = int(floorf(px)), by = int(floorf(py));
  const float ax = px - floorf(px), ay = py - floorf(py);
  const V3 top = lerp3(texel_linear(s, m, bx, by), texel_linear(s, m, bx + 1, by), ax);
  const V3 bottom = lerp3(texel_linear(s, m, bx, by + 1), texel_linear(s, m, bx + 1, by + 1), ax);
  return a * lerp3(top, bottom, ay);
}

__device__ __forceinline__ V3 uniform_sphere(float u1, float u2) {
  const float z = 1.0f - 2.0f * u1;
  const float r = sqrtf(fmaxf(0.0f, 1.0f - z * z));
  float sp, cp;
  sincosf(2.0f * kPiF * u2, &sp, &cp);
  return mk(r * cp, r * sp, z);
}
// Uniform point in the unit ball: the distribution of random_in_unit_sphere (integrator.rs:377).
__device__ __forceinline__ V3 uniform_ball(float u1, float u2, float u3) {
  return uniform_sphere(u1, u2) * cbrtf(u3);
}
__device__ __forceinline__ V3 reflect(V3 d, V3 n) { return d - 2.0f * dot(d, n) * n; }
__device__ __forceinline__ V3 refract(V3 d, V3 n, float ratio) {
  const float ct = fminf(dot(-d, n), 1.0f);
  const V3 perp = ratio * (d + ct * n);
  const V3 par = -sqrtf(fabsf(1.0f - dot(perp, perp))) * n;
  return perp + par;
}
__device__ __forceinline__ float schlick(float cosine, float ratio) {
  float r0 = (1.0f - ratio) / (1.0f + ratio);
  r0 = r0 * r0;
  const float m = 1.0f - cosine;
  return r0 + (1.0f - r0) * (m * m * m * m * m);
}
__device__ __forceinline__ float power_heuristic(float a, float b) {
  const float a2 = a * a, b2 = b * b, d = a2 + b2;
  return d > 0.0f ? a2 / d : 0.0f;
}

// ------------------------------------------------------------------------ parity kernel
__global__ void trace_closest_kernel(const DevScene s, const float* __restrict__ rays, uint64_t n, float tmin,
                                     uint32_t* __restrict__ prim, float* __restrict__ tout) {
  __shared__ ChildRec root;
  if (threadIdx.x == 0) root = *s.root;
  __syncthreads();
  const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float* r = rays + 6 * i;
  const RayQ q = make_ray(r[0], r[1], r[2], r[3], r[4], r[5]);
  TraceResult tr;
  uint32_t visits = 0;
  const bool hit = s.tri_verts
                       ? trace_ray<true>(s.pairs, s.prims, root, q, tmin, CUDART_INF_F, false, tr, visits, s.tri_verts)
                       : trace_ray(s.pairs, s.prims, root, q, tmin, CUDART_INF_F, false, tr, visits);
  prim[i] = hit ? (tr.tag & ~kTagLast) : 0xFFFFFFFFu;
  tout[i] = hit ? tr.t : CUDART_INF_F;
}

__global__ void triangle_vertices_kernel(const PrimRecord* __restrict__ prims, uint32_t n,
                                         const float4* __restrict__ tris, float4* __restrict__ verts) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const uint32_t tag = __float_as_uint(prims[k].a[3]);
  if (!(tag & kTagTriangle)) return;
  const float4* t = tris + 4 * size_t(tag & kTagIndexMask);  // tc_gpu_triangle: v0, v1, v2, material
  verts[3 * size_t(k)] = t[0];
  verts[3 * size_t(k) + 1] = t[1];
  verts[3 * size_t(k) + 2] = t[2];
}

cudaError_t launch_triangle_vertices(const PrimRecord* prims, uint32_t n, const void* triangles, float4* verts,
                                     cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  triangle_vertices_kernel<<<(n + 255) / 256, 256, 0, stream>>>(prims, n, static_cast<const float4*>(triangles), verts);
  return cudaGetLastError();
}

cudaError_t launch_trace_closest(const DevScene& s, const float* rays, uint64_t n, float tmin, uint32_t* prim,
                                 float* t, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  const int block = 128;
  const uint64_t grid = (n + block - 1) / block;
  trace_closest_kernel<<<unsigned(grid), block, 0, stream>>>(s, rays, n, tmin, prim, t);
  return cudaGetLastError();
}

// ------------------------------------------------------------------------ path kernel
enum Phase : int { kIdle = 0, kExtend = 1, kShadowLight = 2, kShadowEnv = 3, kScatter = 4 };

// Path-id word of a training record written for an unoccluded environment shadow ray.
constexpr uint32_t kNeeRecord = 0xFFFFFFFFu;

struct Lane {
  V3 ro, rd;         // next ray
  V3 thr;            // path throughput
  V3 rad;            // radiance of the current sample
  V3 hp, hn, alb;    // diffuse vertex: point, shading normal, albedo
  V3 pend;           // contribution of the pending shadow ray if unoccluded
  V3 acc;            // radiance sum of the current work item
  V3 acc2;           // squared-sample sum of the current work item
  float bsdf_pdf;    // solid-angle pdf of the last diffuse bounce, < 0 for none
  float tmax;        // distance limit of the pending ray
  int phase;
  int depth;         // remaining depth (ray_color_inner's remaining_depth)
  bool include_emission;
  uint32_t pixel, item_samples, item_done, sample;
  int mix_slot;      // guided mode: decoded mixture of the current diffuse vertex, or -1
  float nee_w;       // record mode: training weight of the pending environment shadow ray
  uint32_t job;      // batched launch: frame of the current work item
  Pcg rng;
};

// The frame a lane works on: the launch's own (single-frame) or its job's (batched).
template <bool kBatch>
__device__ __forceinline__ const FrameJob& frame_of(const RenderLaunch& L, const Lane& ln) {
  if constexpr (kBatch) return L.jobs[ln.job];
  else return L.f;
}

// ------------------------------------------------------------------------ guiding mixture
// Decoded 8-lobe von Mises-Fisher mixture: mix[j] = (mu.xyz, kappa), mix[8..9] = weights.
__device__ __forceinline__ float mix_pdf(const float4* __restrict__ mix, V3 w) {
  const float4 w0 = __ldg(mix + 8), w1 = __ldg(mix + 9);
  const float wt[8] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w};
  float p = 0.0f;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const float4 m = __ldg(mix + j);
    const float c = m.x * w.x + m.y * w.y + m.z * w.z;
    const float norm = m.w / (2.0f * kPiF * -expm1f(-2.0f * m.w));
    p += wt[j] * norm * __expf(m.w * (c - 1.0f));
  }
  return p;
}

// Lobe chosen by its weight with u1; direction from the vMF inverse CDF (cosine to the mean
// W = 1 + log(u2 + (1 - u2) e^{-2 kappa}) / kappa, azimuth 2 pi u3) in an orthonormal frame.
__device__ __forceinline__ V3 mix_sample(const float4* __restrict__ mix, float u1, float u2, float u3) {
  const float4 w0 = __ldg(mix + 8), w1 = __ldg(mix + 9);
  const float wt[8] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w};
  int j = 7;
  float acc = 0.0f;
#pragma unroll
  for (int k = 0; k < 7; ++k) {
    acc += wt[k];
    if (u1 < acc) { j = k; break; }
  }
  const float4 m = __ldg(mix + j);
  const float kappa = m.w;
  float W = 1.0f + __logf(u2 + (1.0f - u2) * __expf(-2.0f * kappa)) / kappa;
  W = fminf(fmaxf(W, -1.0f), 1.0f);
  const float r = sqrtf(fmaxf(0.0f, 1.0f - W * W));
  float sp, cp;
  sincospif(2.0f * u3, &sp, &cp);
  // Branchless orthonormal basis (Duff et al. 2017) around the lobe axis.
  const float sign = copysignf(1.0f, m.z);
  const float a = -1.0f / (sign + m.z);
  const float b = m.x * m.y * a;
  const V3 t = mk(1.0f + sign * m.x * m.x * a, sign * b, -sign * m.x);
  const V3 bb = mk(b, sign + m.y * m.y * a, -m.y);
  return mk(m.x, m.y, m.z) * W + (t * cp + bb * sp) * r;
}

// One slot of a counter shared by the lanes that reach this call together (one atomic per warp).
__device__ __forceinline__ uint32_t aggregated_increment(uint32_t* counter) {
  const unsigned active = __activemask();
  const int leader = __ffs(active) - 1;
  const unsigned lane = threadIdx.x & 31u;
  uint32_t base = 0;
  if (int(lane) == leader) base = atomicAdd(counter, uint32_t(__popc(active)));
  base = __shfl_sync(active, base, leader);
  return base + uint32_t(__popc(active & ((1u << lane) - 1u)));
}

__device__ __forceinline__ void start_sample(const FrameJob& J, Lane& ln) {
  const DevScene& s = J.scene;
  ln.rng.seed(J.frame_index_dev ? *J.frame_index_dev : J.frame_index, ln.pixel, ln.sample);
  const uint32_t x = ln.pixel % J.width, y = ln.pixel / J.width;
  const float u = (float(x) + ln.rng.uniform()) / float(J.width);
  const float v = 1.0f - (float(y) + ln.rng.uniform()) / float(J.height);
  V3 o, ll, h, vv;
  if (J.camera_dev) {
    const float4* c = reinterpret_cast<const float4*>(J.camera_dev);
    const float4 c0 = c[0], c1 = c[1], c2 = c[2], c3 = c[3];
    o = mk(c0.x, c0.y, c0.z);
    ll = mk(c1.x, c1.y, c1.z);
    h = mk(c2.x, c2.y, c2.z);
    vv = mk(c3.x, c3.y, c3.z);
  } else {
    o = mk(s.cam_origin[0], s.cam_origin[1], s.cam_origin[2]);
    ll = mk(s.cam_lower_left[0], s.cam_lower_left[1], s.cam_lower_left[2]);
    h = mk(s.cam_horizontal[0], s.cam_horizontal[1], s.cam_horizontal[2]);
    vv = mk(s.cam_vertical[0], s.cam_vertical[1], s.cam_vertical[2]);
  }
  ln.ro = o;
  ln.rd = normalize(ll + u * h + v * vv - o);
  ln.thr = mk(1.f, 1.f, 1.f);
  ln.rad = mk(0.f, 0.f, 0.f);
  ln.depth = int(J.max_bounces);
  ln.include_emission = true;
  ln.bsdf_pdf = -1.0f;
  ln.mix_slot = -1;
  ln.phase = kExtend;
}

template <int kMode, bool kMoments>
__device__ __forceinline__ void finish_sample(const RenderLaunch& L, const FrameJob& J, Lane& ln, uint32_t& n_paths) {
  if constexpr (kMode == kModeRecord) {
    const uint32_t path = (ln.sample - J.sample_base) * (J.width * J.height) + ln.pixel;
    L.g.path_radiance[path] = make_float4(ln.rad.x, ln.rad.y, ln.rad.z, 0.0f);
  }
  ln.acc = ln.acc + ln.rad;
  if (kMoments) ln.acc2 = ln.acc2 + ln.rad * ln.rad;
  ++n_paths;
  ++ln.item_done;
  ++ln.sample;
  if (ln.item_done >= ln.item_samples) {
    double* a = J.accum + size_t(3) * ln.pixel;
    atomicAdd(a, double(ln.acc.x));
    atomicAdd(a + 1, double(ln.acc.y));
    atomicAdd(a + 2, double(ln.acc.z));
    if (kMoments) {
      double* q = J.accum_sq + size_t(3) * ln.pixel;
      atomicAdd(q, double(ln.acc2.x));
      atomicAdd(q + 1, double(ln.acc2.y));
      atomicAdd(q + 2, double(ln.acc2.z));
    }
    ln.phase = kIdle;
  } else {
    start_sample(J, ln);
  }
}

// Light-sampling shadow ray (integrator.rs:168-205); false when the sample contributes nothing.
__device__ __forceinline__ bool prepare_light_shadow(const DevScene& s, Lane& ln) {
  if (s.light_count == 0) return false;
  const float u1 = ln.rng.uniform(), u2 = ln.rng.uniform(), u3 = ln.rng.uniform();
  const float scaled = u1 * float(s.light_count);
  uint32_t i = min(uint32_t(scaled), s.light_count - 1);
  const DevLight* Lt = s.lights + i;
  if (scaled - float(i) >= __ldg(&Lt->alias_prob)) Lt = s.lights + __ldg(&Lt->alias);
  const DevLight lt = *Lt;
  V3 pos, nrm;
  if (lt.kind == 0) {
    const float su = sqrtf(u2);
    const float w1 = su * (1.0f - u3), w2 = su * u3;
    pos = mk(lt.p0[0], lt.p0[1], lt.p0[2]) + mk(lt.e1[0], lt.e1[1], lt.e1[2]) * w1 + mk(lt.e2[0], lt.e2[1], lt.e2[2]) * w2;
    nrm = mk(lt.normal[0], lt.normal[1], lt.normal[2]);
  } else {
    nrm = uniform_sphere(u2, u3);
    pos = mk(lt.p0[0], lt.p0[1], lt.p0[2]) + nrm * lt.radius;
  }
  const V3 so = ln.hp + ln.hn * kRayEps;
  const V3 to = pos - so;
  const float d2 = dot(to, to);
  if (d2 <= kRayEps * kRayEps) return false;
  const float dist = sqrtf(d2);
  const V3 dir = to * (1.0f / dist);
  const float cs = fmaxf(dot(ln.hn, dir), 0.0f);
  const float cl = fmaxf(dot(nrm, -dir), 0.0f);
  if (cs <= 0.0f || cl <= 0.0f) return false;
  const float scale = cs * cl / (kPiF * d2 * lt.pdf_area);
  ln.pend = ln.thr * ln.alb * mk(lt.emission[0], lt.emission[1], lt.emission[2]) * scale;
  ln.ro = so;
  ln.rd = dir;
  // Occluded iff the closest hit lies strictly before dist - 2*eps (integrator.rs:196-199).
  ln.tmax = nextafterf(dist - 2.0f * kRayEps, -CUDART_INF_F);
  return true;
}

// Environment-sampling shadow ray with the power heuristic (integrator.rs:208-244). At a guided
// vertex the competing technique is the 50/50 BSDF / guide mixture, so its pdf enters the weight.
// kWeights (and record mode): also the ray's weight as a guide training sample (ln.nee_w).
template <int kMode, bool kWeights = false>
__device__ __forceinline__ bool prepare_env_shadow(const RenderLaunch& L, const FrameJob& J, Lane& ln) {
  const DevScene& s = J.scene;
  if (s.background != 2u || !s.env_sampleable) return false;
  const float u1 = ln.rng.uniform(), u2 = ln.rng.uniform(), u3 = ln.rng.uniform();
  V3 dir, rad;
  float pdf;
  if (!env_sample(s, u1, u2, u3, dir, rad, pdf)) return false;
  const float cs = fmaxf(dot(ln.hn, dir), 0.0f);
  if (cs <= 0.0f || pdf <= 0.0f) return false;
  float indirect_pdf = cs / kPiF;
  if constexpr (kMode == kModeGuided) {
    if (ln.mix_slot >= 0)
      indirect_pdf = (1.0f - L.g.guide_fraction) * indirect_pdf +
                     L.g.guide_fraction * mix_pdf(L.g.in_mix + 10 * size_t(ln.mix_slot), dir);
  }
  const float mis = power_heuristic(pdf, indirect_pdf);
  ln.pend = ln.thr * ln.alb * rad * (cs * mis / (kPiF * pdf));
  if constexpr (kMode == kModeRecord || kWeights) {
    // As a training sample this direction stands for the share of the incident radiance that
    // the BSDF side carries (1 - mis), the share a guided direction has to find: NEE samples the
    // visible sky far more often than cosine sampling does, and the sun's share stays near 0.
    ln.nee_w = luminance(rad) * (cs * (1.0f - mis) / (kPiF * pdf));
  }
  ln.ro = ln.hp + ln.hn * kRayEps;
  ln.rd = dir;
  ln.tmax = CUDART_INF_F;
  return true;
}

__device__ __forceinline__ V3 background(const DevScene& s, V3 d, float bsdf_pdf) {
  if (s.background == 0u) {
    const V3 dn = normalize(d);
    return lerp3(mk(1.f, 1.f, 1.f), mk(0.35f, 0.65f, 1.0f), 0.5f * (dn.y + 1.0f));
  }
  if (s.background != 2u || s.env_width == 0) return mk(0.f, 0.f, 0.f);
  const V3 r = env_radiance(s, d);
  const float w = bsdf_pdf >= 0.0f ? power_heuristic(bsdf_pdf, env_pdf(s, d)) : 1.0f;
  return r * w;
}

// Writes a path suspended at a diffuse vertex (guided mode) and the query for its mixture.
// Batched launches keep one region of the wave buffers per frame (FrameJob::wave_offset), so the
// frame's own network infers its queries; the frame index travels with the path.
template <bool kBatch>
__device__ __forceinline__ void suspend_path(const RenderLaunch& L, const Lane& ln) {
  uint32_t slot;
  if constexpr (kBatch) {
    // One atomic per group of lanes of the same frame.
    const unsigned group = __match_any_sync(__activemask(), ln.job);
    const int leader = __ffs(group) - 1;
    uint32_t base = 0;
    if (int(threadIdx.x & 31u) == leader) base = atomicAdd(L.g.job_out_count + ln.job, uint32_t(__popc(group)));
    base = __shfl_sync(group, base, leader);
    const uint32_t local = base + uint32_t(__popc(group & ((1u << (threadIdx.x & 31u)) - 1u)));
    const FrameJob& J = L.jobs[ln.job];
    if (local >= J.wave_capacity) return;  // cannot happen: the region covers every path of the frame's wave
    slot = J.wave_offset + local;
  } else {
    slot = aggregated_increment(L.g.out_count);
    if (slot >= L.g.capacity) return;  // cannot happen: capacity covers every path of the wave
  }
  float4* st = L.g.out_state + 6 * size_t(slot);
  st[0] = make_float4(ln.hp.x, ln.hp.y, ln.hp.z, ln.hn.x);
  st[1] = make_float4(ln.hn.y, ln.hn.z, ln.alb.x, ln.alb.y);
  st[2] = make_float4(ln.alb.z, ln.thr.x, ln.thr.y, ln.thr.z);
  st[3] = make_float4(ln.rad.x, ln.rad.y, ln.rad.z, __int_as_float(ln.depth));
  st[4] = make_float4(__uint_as_float(ln.pixel), __uint_as_float(uint32_t(ln.rng.state)),
                      __uint_as_float(uint32_t(ln.rng.state >> 32)), __uint_as_float(uint32_t(ln.rng.inc)));
  st[5] = make_float4(__uint_as_float(uint32_t(ln.rng.inc >> 32)), __uint_as_float(ln.job), 0.0f, 0.0f);
  float4* q = L.g.out_query + 2 * size_t(slot);
  q[0] = make_float4(ln.hp.x, ln.hp.y, ln.hp.z, 0.0f);
  q[1] = make_float4(ln.hn.x, ln.hn.y, ln.hn.z, 0.0f);
}

__device__ __forceinline__ void resume_path(const RenderLaunch& L, Lane& ln, uint32_t slot) {
  const float4* st = L.g.in_state + 6 * size_t(slot);
  const float4 a = st[0], b = st[1], c = st[2], d = st[3], e = st[4], f = st[5];
  ln.hp = mk(a.x, a.y, a.z);
  ln.hn = mk(a.w, b.x, b.y);
  ln.alb = mk(b.z, b.w, c.x);
  ln.thr = mk(c.y, c.z, c.w);
  ln.rad = mk(d.x, d.y, d.z);
  ln.depth = __float_as_int(d.w);
  ln.pixel = __float_as_uint(e.x);
  ln.rng.state = uint64_t(__float_as_uint(e.y)) | (uint64_t(__float_as_uint(e.z)) << 32);
  ln.rng.inc = uint64_t(__float_as_uint(e.w)) | (uint64_t(__float_as_uint(f.x)) << 32);
  ln.job = __float_as_uint(f.y);
  ln.include_emission = false;
  ln.bsdf_pdf = -1.0f;
  ln.mix_slot = int(slot);
  ln.item_samples = 1;
  ln.item_done = 0;
  ln.acc = mk(0.f, 0.f, 0.f);
  ln.acc2 = mk(0.f, 0.f, 0.f);
  ln.phase = kShadowLight;
}

// Surface seen by a ray at its closest hit: point, shading normal facing the ray, texture
// coordinates and material (intersect.rs:57-68, :122-148).
struct Surface {
  V3 hp, nrm;
  float tu, tv;
  bool front;
  uint32_t mat;
};

__device__ __forceinline__ Surface surface_at(const DevScene& s, V3 ro, V3 rd, const TraceResult& tr) {
  Surface f;
  const float4* p = reinterpret_cast<const float4*>(s.prims + tr.rec);
  const float4 A = __ldg(p), B = __ldg(p + 1);
  f.hp = ro + rd * tr.t;
  f.tu = 0.0f;
  f.tv = 0.0f;
  if (tr.tag & kTagTriangle) {
    const float4 C = __ldg(p + 2);
    const V3 e1 = mk(B.x, B.y, B.z), e2 = mk(C.x, C.y, C.z);
    const V3 gn = normalize(cross(e1, e2));
    f.front = dot(rd, gn) < 0.0f;
    V3 outward = gn;
    const uint32_t flags = __float_as_uint(C.w);
    if (flags != 0u && s.attributes != nullptr) {
      // Barycentrics for attribute interpolation (intersect.rs:124-135).
      const V3 sv = ro - mk(A.x, A.y, A.z);
      const V3 pv = cross(rd, e2);
      const float inv = 1.0f / dot(e1, pv);
      const float u = dot(sv, pv) * inv;
      const V3 qv = cross(sv, e1);
      const float v = dot(rd, qv) * inv;
      const float w0 = 1.0f - u - v;
      const float4* at = s.attributes + size_t(5) * (tr.tag & kTagIndexMask);
      if (flags & 1u) {
        const float4 n0 = __ldg(at), n1 = __ldg(at + 1), n2 = __ldg(at + 2);
        outward = normalize(mk(n0.x, n0.y, n0.z) * w0 + mk(n1.x, n1.y, n1.z) * u + mk(n2.x, n2.y, n2.z) * v);
        if (dot(outward, gn) < 0.0f) outward = -outward;
      }
      if (flags & 2u) {
        const float4 uv01 = __ldg(at + 3), uv2 = __ldg(at + 4);
        f.tu = w0 * uv01.x + u * uv01.z + v * uv2.x;
        f.tv = w0 * uv01.y + u * uv01.w + v * uv2.y;
      }
    }
    f.nrm = f.front ? outward : -outward;
  } else {
    const V3 outward = (f.hp - mk(A.x, A.y, A.z)) * (1.0f / B.x);
    f.front = dot(rd, outward) < 0.0f;
    f.nrm = f.front ? outward : -outward;
  }
  f.mat = __float_as_uint(B.w);
  return f;
}

// Fuzzy metal reflection (integrator.rs:303-313): false when the ray is absorbed (it points into
// the surface). On success the lane holds the reflected ray.
__device__ __forceinline__ bool bounce_metal(Lane& ln, const DevMaterial& m, const Surface& f) {
  const V3 refl = reflect(normalize(ln.rd), f.nrm);
  const V3 ball = uniform_ball(ln.rng.uniform(), ln.rng.uniform(), ln.rng.uniform());
  const V3 dir = refl + ball * m.roughness;
  if (dot(dir, f.nrm) <= 0.0f) return false;
  ln.ro = f.hp;
  ln.rd = normalize(dir);
  ln.thr = ln.thr * mk(m.albedo[0], m.albedo[1], m.albedo[2]);
  return true;
}

// Dielectric (integrator.rs:315-334): Schlick reflection or Snell refraction.
__device__ __forceinline__ void bounce_dielectric(Lane& ln, const DevMaterial& m, const Surface& f) {
  const float ratio = f.front ? 1.0f / m.ior : m.ior;
  const V3 unit = normalize(ln.rd);
  const float ct = fminf(dot(-unit, f.nrm), 1.0f);
  const float st = sqrtf(1.0f - ct * ct);
  const bool cannot = ratio * st > 1.0f;
  V3 dir;
  if (cannot || schlick(ct, ratio) > ln.rng.uniform()) dir = reflect(unit, f.nrm);
  else dir = refract(unit, f.nrm, ratio);
  ln.ro = f.hp;
  ln.rd = normalize(dir);
}

// Cosine-weighted diffuse direction about the lane's shading normal (integrator.rs:277-301).
__device__ __forceinline__ V3 cosine_direction(Lane& ln) {
  V3 dir = ln.hn + uniform_sphere(ln.rng.uniform(), ln.rng.uniform());
  if (dot(dir, dir) < 1e-8f) dir = ln.hn;
  return normalize(dir);
}

// The lane continues from its diffuse vertex along `dir` (drawn by cosine_direction).
__device__ __forceinline__ void take_diffuse_bounce(Lane& ln, V3 dir) {
  ln.ro = ln.hp;
  ln.rd = dir;
  ln.thr = ln.thr * ln.alb;
  ln.include_emission = false;
  ln.bsdf_pdf = fmaxf(dot(ln.hn, dir), 0.0f) / kPiF;
}

// Guided diffuse bounce: one-sample MIS of cosine and guide sampling (the balance heuristic =
// the mixture pdf, the guide taken with probability g.guide_fraction), so the estimator stays
// unbiased whatever the network predicts. `mix` is the vertex's decoded mixture. False when the
// sampled direction leaves below the surface (the path ends).
__device__ __forceinline__ bool take_guided_bounce(const GuideLaunch& g, const float4* __restrict__ mix, Lane& ln) {
  const float ut = ln.rng.uniform();
  V3 dir;
  if (ut < 1.0f - g.guide_fraction) {
    dir = cosine_direction(ln);
  } else {
    const float a = ln.rng.uniform(), b = ln.rng.uniform(), c = ln.rng.uniform();
    dir = mix_sample(mix, a, b, c);
  }
  const float cs = dot(ln.hn, dir);
  if (!(cs > 0.0f)) return false;
  const float p = (1.0f - g.guide_fraction) * cs / kPiF + g.guide_fraction * mix_pdf(mix, dir);
  ln.ro = ln.hp;
  ln.rd = dir;
  ln.thr = ln.thr * ln.alb * (cs / (kPiF * p));
  ln.include_emission = false;
  ln.bsdf_pdf = p;
  return true;
}

template <int kMode, bool kMoments, bool kBatch>
__device__ __forceinline__ void shade_hit(const RenderLaunch& L, const FrameJob& J, Lane& ln, const TraceResult& tr,
                                          uint32_t& n_paths) {
  const DevScene& s = J.scene;
  const Surface f = surface_at(s, ln.ro, ln.rd, tr);
  const DevMaterial m = s.materials[f.mat];
  if (m.kind == kEmissive) {
    if (ln.include_emission) ln.rad = ln.rad + ln.thr * mk(m.emission[0], m.emission[1], m.emission[2]);
    finish_sample<kMode, kMoments>(L, J, ln, n_paths);
    return;
  }
  if (m.kind == kDiffuse) {
    ln.hp = f.hp;
    ln.hn = f.nrm;
    ln.alb = base_color(s, m, f.tu, f.tv);
    ln.mix_slot = -1;
    ln.phase = kShadowLight;
    if constexpr (kMode == kModeGuided) {
      // A vertex that will scatter waits for the network's mixture; the last vertex only does NEE.
      if (ln.depth > 1) {
        suspend_path<kBatch>(L, ln);
        ln.phase = kIdle;
      }
    }
    return;
  }
  if (m.kind == kMetal) {
    if (!bounce_metal(ln, m, f)) {
      finish_sample<kMode, kMoments>(L, J, ln, n_paths);
      return;
    }
  } else {
    bounce_dielectric(ln, m, f);
  }
  ln.include_emission = true;
  ln.bsdf_pdf = -1.0f;
  ln.depth -= 1;
  ln.phase = kExtend;
}

// kPause selects the traversal: false = each ray traced to its end in one call (trace_ray);
// true = resumable traversals that a warp pauses to refill finished lanes (dynamic ray fetching,
// L.min_active) with an optional shared-memory short stack (L.short_stack).
template <int kMode, bool kMoments, bool kBatch, bool kPause>
__global__ void __launch_bounds__(256) render_kernel(const RenderLaunch L) {
  static_assert(!kBatch || kMode != kModeRecord, "batched launches do not record training samples");
  // The root record lives in device memory (a geometry refit rewrites it between launches);
  // single-frame launches stage it in shared memory once.
  __shared__ ChildRec root;
  __shared__ unsigned long long s_count[3];  // this block's share of the launch counters
  if (threadIdx.x < 3) s_count[threadIdx.x] = 0ull;
  if constexpr (!kBatch) {
    if (threadIdx.x == 0) root = *L.f.scene.root;
  }
  __syncthreads();
  extern __shared__ uint2 s_stack[];  // L.short_stack entries per thread, blockDim.x apart
  uint2* const my_stack = s_stack + threadIdx.x;
  const unsigned lane = threadIdx.x & 31u;
  const uint32_t npix = L.f.width * L.f.height;  // single-frame launches
  Lane ln;
  ln.phase = kIdle;
  ln.mix_slot = -1;
  ln.job = 0;
  // Pausing traversal only: the lane's ray in flight, kept across rounds of the loop.
  Traversal T;
  T.cur = kNoNode;
  T.rec = kNoNode;
  bool inflight = false;
  uint2 st_local[kPause ? kMaxStack : 1];  // its local-memory stack, also kept across rounds
  ln.acc = ln.acc2 = mk(0.f, 0.f, 0.f);
  bool finished = false;
  uint32_t n_paths = 0, n_ext = 0, n_shadow = 0, node_visits = 0;
  uint64_t total_items = L.total_items;
  if constexpr (kMode == kModeGuided) {
    if (L.g.resume) {
      if constexpr (kBatch) total_items = L.g.in_job_prefix[L.job_count];
      else total_items = *L.g.in_count < L.g.capacity ? *L.g.in_count : L.g.capacity;
    }
  }

  for (;;) {
    // Refill idle lanes: one atomic per warp for all of them.
    const bool want = !finished && ln.phase == kIdle;
    const unsigned want_mask = __ballot_sync(0xffffffffu, want);
    if (want_mask) {
      const int leader = __ffs(want_mask) - 1;
      unsigned long long base = 0;
      if (int(lane) == leader) base = atomicAdd(L.work_counter, (unsigned long long)__popc(want_mask));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (want) {
        const uint64_t item = base + __popc(want_mask & ((1u << lane) - 1u));
        if (item >= total_items) {
          finished = true;
        } else if (kMode == kModeGuided && L.g.resume) {
          if constexpr (kBatch) {
            // The frame whose share of this round's suspended paths holds the item.
            uint32_t lo = 0, hi = L.job_count - 1;
            while (lo < hi) {
              const uint32_t mid = (lo + hi + 1) >> 1;
              if (L.g.in_job_prefix[mid] <= item) lo = mid;
              else hi = mid - 1;
            }
            resume_path(L, ln, L.jobs[lo].wave_offset + uint32_t(item - L.g.in_job_prefix[lo]));
          } else {
            resume_path(L, ln, uint32_t(item));
          }
        } else if (kMode == kModeGuided && kBatch) {
          // One path per item; a frame's items are its wave's samples, pixel-major within each.
          const uint64_t ws = L.g.wave_spp;
          uint32_t lo = 0, hi = L.job_count - 1;
          while (lo < hi) {
            const uint32_t mid = (lo + hi + 1) >> 1;
            if (uint64_t(L.jobs[mid].pix_begin) * ws <= item) lo = mid;
            else hi = mid - 1;
          }
          ln.job = lo;
          const FrameJob& J = L.jobs[lo];
          const uint32_t fpix = J.width * J.height;
          const uint64_t local = item - uint64_t(J.pix_begin) * ws;
          const uint32_t k = uint32_t(local / fpix);
          ln.pixel = uint32_t(local - uint64_t(k) * fpix);
          ln.item_samples = 1;
          ln.item_done = 0;
          ln.sample = J.sample_base + L.g.wave_first_sample + k;
          ln.acc = mk(0.f, 0.f, 0.f);
          if (kMoments) ln.acc2 = mk(0.f, 0.f, 0.f);
          start_sample(J, ln);
        } else if (kMode == kModeGuided) {
          // One path per item: pixel-major within each sample of the wave.
          const uint32_t k = uint32_t(item / npix);
          ln.pixel = uint32_t(item - uint64_t(k) * npix);
          ln.item_samples = 1;
          ln.item_done = 0;
          ln.sample = L.g.wave_first_sample + k;
          ln.acc = mk(0.f, 0.f, 0.f);
          if (kMoments) ln.acc2 = mk(0.f, 0.f, 0.f);
          start_sample(L.f, ln);
        } else {
          uint64_t local = item;
          if constexpr (kBatch) {
            // The job whose item range holds this item (item_begin ascends with the job index).
            uint32_t lo = 0, hi = L.job_count - 1;
            while (lo < hi) {
              const uint32_t mid = (lo + hi + 1) >> 1;
              if (L.jobs[mid].item_begin <= item) lo = mid;
              else hi = mid - 1;
            }
            ln.job = lo;
            local = item - L.jobs[lo].item_begin;
          }
          const FrameJob& J = frame_of<kBatch>(L, ln);
          const uint32_t fpix = J.width * J.height;
          const uint32_t chunk = uint32_t(local / fpix);
          ln.pixel = uint32_t(local - uint64_t(chunk) * fpix);
          const uint32_t first = chunk * J.samples_per_item;
          ln.item_samples = min(J.samples_per_item, J.samples - first);
          ln.item_done = 0;
          ln.sample = J.sample_base + first;
          ln.acc = mk(0.f, 0.f, 0.f);
          if (kMoments) ln.acc2 = mk(0.f, 0.f, 0.f);
          start_sample(J, ln);
        }
      }
    }
    if (__all_sync(0xffffffffu, finished)) break;
    const FrameJob& J = frame_of<kBatch>(L, ln);
    const DevScene& s = J.scene;

    // Advance the lane's state machine to its next ray.
    bool have = false;
    while (!finished && !inflight && !have && ln.phase != kIdle) {
      switch (ln.phase) {
        case kExtend:
          if (ln.depth <= 0) {
            finish_sample<kMode, kMoments>(L, J, ln, n_paths);
          } else {
            have = true;
            ln.tmax = CUDART_INF_F;
          }
          break;
        case kShadowLight:
          if (prepare_light_shadow(s, ln)) have = true;
          else ln.phase = kShadowEnv;
          break;
        case kShadowEnv:
          if (prepare_env_shadow<kMode>(L, J, ln)) have = true;
          else ln.phase = kScatter;
          break;
        default: {  // kScatter: cosine-weighted diffuse bounce (integrator.rs:277-289)
          ln.depth -= 1;
          if (ln.depth <= 0) {
            finish_sample<kMode, kMoments>(L, J, ln, n_paths);
            break;
          }
          if constexpr (kMode == kModeGuided) {
            if (ln.mix_slot >= 0) {
              const float4* mix = L.g.in_mix + 10 * size_t(ln.mix_slot);
              ln.mix_slot = -1;
              if (!take_guided_bounce(L.g, mix, ln)) {
                finish_sample<kMode, kMoments>(L, J, ln, n_paths);
                break;
              }
              ln.phase = kExtend;
              break;
            }
          }
          const V3 dir = cosine_direction(ln);
          if constexpr (kMode == kModeRecord) {
            const uint32_t slot = aggregated_increment(L.g.record_count);
            if (slot < L.g.record_capacity) {
              const uint32_t path = (ln.sample - J.sample_base) * npix + ln.pixel;
              const V3 t = ln.thr * ln.alb;
              float4* r = L.g.records + 4 * size_t(slot);
              r[0] = make_float4(ln.hp.x, ln.hp.y, ln.hp.z, __uint_as_float(path));
              r[1] = make_float4(ln.hn.x, ln.hn.y, ln.hn.z, t.x);
              r[2] = make_float4(dir.x, dir.y, dir.z, t.y);
              r[3] = make_float4(ln.rad.x, ln.rad.y, ln.rad.z, t.z);
            }
          }
          take_diffuse_bounce(ln, dir);
          ln.phase = kExtend;
          break;
        }
      }
    }

    // The ray in flight is (ln.ro, ln.rd, ln.tmax): the state machine leaves them alone until it
    // has been consumed. Shadow rays (light and environment phases) stop at the first hit.
    const bool shadow = ln.phase == kShadowLight || ln.phase == kShadowEnv;
    bool hit = false, done = false;
    TraceResult tr;
    if constexpr (!kPause) {
      if (have) {
        const RayQ q = make_ray(ln.ro.x, ln.ro.y, ln.ro.z, ln.rd.x, ln.rd.y, ln.rd.z);
        if constexpr (kBatch) {
          const ChildRec rt = *s.root;
          hit = trace_ray(s.pairs, s.prims, rt, q, kRayEps, ln.tmax, shadow, tr, node_visits);
        } else {
          hit = trace_ray(s.pairs, s.prims, root, q, kRayEps, ln.tmax, shadow, tr, node_visits);
        }
        done = true;
      }
    } else {
    const RayQ q = make_ray(ln.ro.x, ln.ro.y, ln.ro.z, ln.rd.x, ln.rd.y, ln.rd.z);
    if (have) {
      if constexpr (kBatch) {
        const ChildRec rt = *s.root;
        trav_start(T, rt, q, kRayEps, ln.tmax);
      } else {
        trav_start(T, root, q, kRayEps, ln.tmax);
      }
      inflight = true;
    }
    // Traverse until too few of the warp's lanes are still busy; the finished ones consume
    // their result now and fetch their next ray in the next round while the others resume.
    trav_advance(T, q, kRayEps, shadow, s.pairs, s.prims, st_local, my_stack, L.short_stack, int(blockDim.x),
                 L.min_active, !finished, node_visits);
    if (inflight && T.cur == kNoNode) {
      inflight = false;
      done = true;
      hit = T.found();
      tr.t = T.closest;
      tr.tag = T.tag;
      tr.rec = T.rec;
    }
    }
    if (done) {
      if (ln.phase == kShadowLight) {
        ++n_shadow;
        if (!hit) ln.rad = ln.rad + ln.pend;
        ln.phase = kShadowEnv;
      } else if (ln.phase == kShadowEnv) {
        ++n_shadow;
        if (!hit) {
          ln.rad = ln.rad + ln.pend;
          if constexpr (kMode == kModeRecord) {
            if (ln.nee_w > 0.0f) {
              const uint32_t slot = aggregated_increment(L.g.record_count);
              if (slot < L.g.record_capacity) {
                float4* r = L.g.records + 4 * size_t(slot);
                r[0] = make_float4(ln.hp.x, ln.hp.y, ln.hp.z, __uint_as_float(kNeeRecord));
                r[1] = make_float4(ln.hn.x, ln.hn.y, ln.hn.z, 0.0f);
                r[2] = make_float4(ln.rd.x, ln.rd.y, ln.rd.z, 0.0f);
                r[3] = make_float4(ln.nee_w, 0.0f, 0.0f, 0.0f);
              }
            }
          }
        }
        ln.phase = kScatter;
      } else {
        ++n_ext;
        if (!hit) {
          ln.rad = ln.rad + ln.thr * background(s, ln.rd, ln.bsdf_pdf);
          finish_sample<kMode, kMoments>(L, J, ln, n_paths);
        } else {
          shade_hit<kMode, kMoments, kBatch>(L, J, ln, tr, n_paths);
        }
      }
    }
  }

  // Per-launch counters: summed per warp, then per block in shared memory, then one global atomic
  // per block and counter.
  const unsigned long long tp = __reduce_add_sync(0xffffffffu, n_paths);
  const unsigned long long te = __reduce_add_sync(0xffffffffu, n_ext);
  const unsigned long long ts = __reduce_add_sync(0xffffffffu, n_shadow);
  if (lane == 0) {
    atomicAdd(&s_count[0], tp);
    atomicAdd(&s_count[1], te);
    atomicAdd(&s_count[2], ts);
  }
  __syncthreads();
  if (threadIdx.x < 3 && s_count[threadIdx.x] != 0ull) atomicAdd(L.counters + threadIdx.x, s_count[threadIdx.x]);
}

static size_t stack_smem(int short_stack, int block_size) {
  return sizeof(uint2) * size_t(short_stack > 0 ? short_stack : 0) * size_t(block_size);
}

// Plain renders without moments pause traversals when asked to (refill lanes above 1 or a shared
// short stack); every other launch traces each ray to its end.
static bool pausing(const RenderLaunch& r) { return r.min_active > 1 || r.short_stack > 0; }

template <int kMode>
static cudaError_t launch_mode(const RenderLaunch& r, int block_size, int grid_size, bool moments, cudaStream_t stream) {
  if (kMode == kModePlain && !moments && pausing(r)) {
    render_kernel<kModePlain, false, false, true>
        <<<grid_size, block_size, stack_smem(r.short_stack, block_size), stream>>>(r);
  } else if (moments) {
    render_kernel<kMode, true, false, false><<<grid_size, block_size, 0, stream>>>(r);
  } else {
    render_kernel<kMode, false, false, false><<<grid_size, block_size, 0, stream>>>(r);
  }
  return cudaGetLastError();
}

cudaError_t launch_render_batch(const RenderLaunch& r, int block_size, int grid_size, cudaStream_t stream,
                                bool guided) {
  if (!r.jobs || r.job_count == 0) return cudaErrorInvalidValue;
  if (guided) render_kernel<kModeGuided, false, true, false><<<grid_size, block_size, 0, stream>>>(r);
  else render_kernel<kModePlain, false, true, false><<<grid_size, block_size, 0, stream>>>(r);
  return cudaGetLastError();
}

int render_batch_max_blocks_per_sm(int block_size, bool guided) {
  int blocks = 0;
  const cudaError_t e =
      guided ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, render_kernel<kModeGuided, false, true, false>,
                                                             block_size, 0)
             : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, render_kernel<kModePlain, false, true, false>,
                                                             block_size, 0);
  return e == cudaSuccess ? blocks : 0;
}

// Exclusive prefix of the per-frame suspended-path counts of one guided round; prefix[n] = total.
__global__ void job_prefix_kernel(const uint32_t* __restrict__ counts, const FrameJob* __restrict__ jobs, uint32_t n,
                                  uint32_t* __restrict__ prefix) {
  if (threadIdx.x != 0) return;
  uint32_t run = 0;
  for (uint32_t i = 0; i < n; ++i) {
    prefix[i] = run;
    run += min(counts[i], jobs[i].wave_capacity);
  }
  prefix[n] = run;
}

cudaError_t launch_job_prefix(const uint32_t* counts, const FrameJob* jobs, uint32_t n, uint32_t* prefix,
                              cudaStream_t stream) {
  job_prefix_kernel<<<1, 32, 0, stream>>>(counts, jobs, n, prefix);
  return cudaGetLastError();
}

cudaError_t launch_render(const RenderLaunch& r, int block_size, int grid_size, bool moments, cudaStream_t stream,
                          int mode) {
  if (mode == kModeRecord) return launch_mode<kModeRecord>(r, block_size, grid_size, moments, stream);
  if (mode == kModeGuided) return launch_mode<kModeGuided>(r, block_size, grid_size, moments, stream);
  return launch_mode<kModePlain>(r, block_size, grid_size, moments, stream);
}

template <int kMode>
static int blocks_for(int block_size, bool moments) {
  int blocks = 0;
  cudaError_t e = moments
      ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, render_kernel<kMode, true, false, false>, block_size, 0)
      : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, render_kernel<kMode, false, false, false>, block_size, 0);
  return e == cudaSuccess ? blocks : 0;
}

int render_max_blocks_per_sm(int block_size, bool moments, int mode, int short_stack, int min_active) {
  if (mode == kModePlain && !moments && (min_active > 1 || short_stack > 0)) {
    int blocks = 0;
    const cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &blocks, render_kernel<kModePlain, false, false, true>, block_size, stack_smem(short_stack, block_size));
    return e == cudaSuccess ? blocks : 0;
  }
  if (mode == kModeRecord) return blocks_for<kModeRecord>(block_size, moments);
  if (mode == kModeGuided) return blocks_for<kModeGuided>(block_size, moments);
  return blocks_for<kModePlain>(block_size, moments);
}

// ------------------------------------------------------------------------ wavefront schedule
// The estimator of render_kernel (plain mode), split into three launches per iteration over
// per-path state in device memory (WavefrontLaunch). Every path draws its random numbers in the
// order the megakernel does (camera jitter; then per diffuse vertex light NEE, environment NEE,
// scatter; per metal or dielectric vertex its BSDF draws) from the same per-(frame, pixel, sample)
// seed, and adds its contributions in the same order, so each path is the megakernel's path.

__device__ __forceinline__ unsigned lanes_below() { return (1u << (threadIdx.x & 31u)) - 1u; }

// Sort key of a queued ray: direction octant, and the bucket of the primitive record its origin
// lies on (records are in leaf order, so nearby records are nearby surfaces); camera rays, which
// start at the eye in pixel order, take the last bucket. Shadow rays use the second half of the bins.
__device__ __forceinline__ uint32_t wf_sort_key(const WavefrontLaunch& W, V3 d, uint32_t rec, bool shadow) {
  const uint32_t octant = (d.x < 0.0f ? 1u : 0u) | (d.y < 0.0f ? 2u : 0u) | (d.z < 0.0f ? 4u : 0u);
  const uint32_t bucket =
      rec == kNoNode ? uint32_t(kWfSortBuckets - 1)
                     : uint32_t((uint64_t(rec) * (kWfSortBuckets - 1)) / max(W.prim_count, 1u));
  return (shadow ? uint32_t(8 * kWfSortBuckets) : 0u) + octant * kWfSortBuckets + bucket;
}

// Reserves room on N queue counters for the whole block at once: thread t asks for n[i] entries of
// counter i and receives the first of them in pos[i]. One atomic per counter per block (all the
// block's warps append to the same few counters in every launch, so per-warp atomics would queue
// up at those addresses): warp-inclusive scans by shuffles, one pass over the warps' totals by N
// threads, two barriers. Every thread of the block (whole warps, at most kWfBlock threads) calls
// it together. `sh` holds N x kWfScanStride words; the next call may reuse it without a barrier in
// between, because before that call's first barrier a warp writes only its own totals, which no
// other warp reads.
constexpr int kWfBlock = 256;
constexpr int kWfScanStride = kWfBlock / 32 + 1;
template <int N>
__device__ __forceinline__ void block_reserve(uint32_t* const (&counter)[N], const uint32_t (&n)[N],
                                              uint32_t (&pos)[N], uint32_t* sh) {
  const unsigned lane = threadIdx.x & 31u;
  const int warp = int(threadIdx.x >> 5);
  uint32_t incl[N];
#pragma unroll
  for (int i = 0; i < N; ++i) {
    uint32_t v = n[i];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t u = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= unsigned(o)) v += u;
    }
    incl[i] = v;
    if (lane == 31u) sh[i * kWfScanStride + warp] = v;
  }
  __syncthreads();
  if (threadIdx.x < unsigned(N)) {
    const int i = int(threadIdx.x);
    uint32_t run = 0;
    for (int w = 0; w < int(blockDim.x >> 5); ++w) {
      const uint32_t c = sh[i * kWfScanStride + w];
      sh[i * kWfScanStride + w] = run;
      run += c;
    }
    sh[i * kWfScanStride + kWfScanStride - 1] = run ? atomicAdd(counter[i], run) : 0u;
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < N; ++i)
    pos[i] = sh[i * kWfScanStride + kWfScanStride - 1] + sh[i * kWfScanStride + warp] + (incl[i] - n[i]);
}

template <bool kMoments, bool kGuided>
__global__ void __launch_bounds__(kWfBlock) wf_logic_kernel(const WavefrontLaunch W) {
  __shared__ uint32_t sh[4 * kWfScanStride];
  __shared__ unsigned long long s_first;
  __shared__ uint32_t s_started;
  const FrameJob& J = W.r.f;
  const DevScene& s = J.scene;
  const uint32_t npix = J.width * J.height;
  uint32_t n_paths = 0, n_live = 0;

  // One slot per thread; whole warps are either in range or the last partial warp.
  {
    const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = slot < W.capacity;
    const uint32_t st = valid ? W.state[slot] : 0u;
    // Once all work is handed out, a block without a live slot starts and finishes nothing.
    if (W.work_done && !__syncthreads_or((st & kWfAlive) != 0u)) return;
    bool free_slot = valid && !(st & kWfAlive);
    int kind = -1;
    if (st & kWfAlive) {
      // Every load this slot may need is issued before any result is used: the state word alone
      // decides which of them matter.
      const float4 r4 = W.rad[slot];
      const float4 t4 = W.thr[slot];
      const bool nee_pending = (st & kWfNeePending) != 0u;
      const bool ext = (st & (kWfTerminate | kWfExtPending)) == kWfExtPending;
      const bool recording = W.r.g.records != nullptr;
      float4 na = make_float4(0.f, 0.f, 0.f, 0.f), nb = na;
      uint4 h = make_uint4(0u, kNoNode, 0u, 0u);
      uint2 rr = make_uint2(kNoNode, kNoNode);
      if (nee_pending) {
        na = W.nee[2 * size_t(slot)];
        nb = W.nee[2 * size_t(slot) + 1];
        if (recording) rr = W.rec_ref[slot];
      }
      if (ext) h = W.hit[slot];
      V3 rad = mk(r4.x, r4.y, r4.z);
      const V3 thr = mk(t4.x, t4.y, t4.z);
      if (nee_pending) {
        rad = rad + mk(na.x, na.y, na.z);
        rad = rad + mk(nb.x, nb.y, nb.z);
        // Recording: the scatter record takes the radiance gathered up to and including this
        // vertex's next-event estimates; the environment record stays only if its shadow ray
        // reached the sky (the trace launch clears the whole entry, marker included, otherwise).
        if (rr.x != kNoNode) {
          float* dst = reinterpret_cast<float*>(W.r.g.records + 4 * size_t(rr.x) + 3);
          dst[0] = rad.x;
          dst[1] = rad.y;
          dst[2] = rad.z;
        }
        if (rr.y != kNoNode && nb.w == 0.0f) reinterpret_cast<float*>(W.r.g.records + 4 * size_t(rr.y) + 3)[0] = 0.0f;
      }
      bool done = (st & kWfTerminate) != 0u;
      if (ext) {
        if (h.y == kNoNode) {
          const float4 d4 = W.ray_d[slot];
          rad = rad + thr * background(s, mk(d4.x, d4.y, d4.z), W.ray_o[slot].w);
          done = true;
        } else {
          const uint32_t mat = h.w & kWfMaterialMask;
          const uint32_t k = h.w >> kWfKindShift;
          if (k == kEmissive) {
            if (st & kWfEmission) {
              const DevMaterial& m = s.materials[mat];
              rad = rad + thr * mk(__ldg(&m.emission[0]), __ldg(&m.emission[1]), __ldg(&m.emission[2]));
            }
            done = true;
          } else {
            kind = int(k);
          }
        }
      }
      if (done) {
        const uint32_t pixel = __float_as_uint(t4.w);
        double* a = J.accum + size_t(3) * pixel;
        atomicAdd(a, double(rad.x));
        atomicAdd(a + 1, double(rad.y));
        atomicAdd(a + 2, double(rad.z));
        if (kMoments) {
          const V3 r2 = rad * rad;
          double* q2 = J.accum_sq + size_t(3) * pixel;
          atomicAdd(q2, double(r2.x));
          atomicAdd(q2 + 1, double(r2.y));
          atomicAdd(q2 + 2, double(r2.z));
        }
        if (recording) W.r.g.path_radiance[__float_as_uint(r4.w)] = make_float4(rad.x, rad.y, rad.z, 0.0f);
        ++n_paths;
        free_slot = true;
      } else {
        W.rad[slot] = make_float4(rad.x, rad.y, rad.z, r4.w);
      }
    }
    // One block-wide pass reserves room for every append of this launch: threads 0-2 on the
    // material queues (paths that go on; the shade launch rewrites their state), thread 3 on the
    // work counter for free slots and then on the extension queue for the camera paths that do
    // start (the block's first s_started free slots in block order: items past the frame's last
    // one start nothing). Consecutive work items are consecutive pixels of one sample, so a warp's
    // new rays are neighbours.
    const int warp = int(threadIdx.x >> 5);
    const unsigned m_mat[3] = {__ballot_sync(0xffffffffu, kind == 0), __ballot_sync(0xffffffffu, kind == 1),
                               __ballot_sync(0xffffffffu, kind == 2)};
    const unsigned m_free = __ballot_sync(0xffffffffu, free_slot);
    if ((threadIdx.x & 31u) == 0) {
#pragma unroll
      for (int k = 0; k < 3; ++k) sh[k * kWfScanStride + warp] = uint32_t(__popc(m_mat[k]));
      sh[3 * kWfScanStride + warp] = uint32_t(__popc(m_free));
    }
    __syncthreads();
    if (threadIdx.x < 4u) {
      const int k = int(threadIdx.x);
      uint32_t run = 0;
      for (int w = 0; w < int(blockDim.x >> 5); ++w) {
        const uint32_t c = sh[k * kWfScanStride + w];
        sh[k * kWfScanStride + w] = run;
        run += c;
      }
      uint32_t base = 0;
      if (k < 3) {
        base = run ? atomicAdd(W.q + kWfMatCount + k, run) : 0u;
      } else {
        const unsigned long long first = run ? atomicAdd(W.r.work_counter, (unsigned long long)run) : 0ull;
        const uint64_t left = first < W.r.total_items ? W.r.total_items - first : 0ull;
        const uint32_t n = left < run ? uint32_t(left) : run;
        s_first = first;
        s_started = n;
        base = n ? atomicAdd(W.q + kWfExtCount, n) : 0u;
      }
      sh[k * kWfScanStride + kWfScanStride - 1] = base;
    }
    __syncthreads();
    if (kind >= 0) {
      const int k = kind;
      const uint32_t pos = sh[k * kWfScanStride + kWfScanStride - 1] + sh[k * kWfScanStride + warp] +
                           uint32_t(__popc(m_mat[k] & lanes_below()));
      W.mat_q[size_t(k) * W.capacity + pos] = slot;
      if constexpr (kGuided) {
        if (k == kDiffuse) {
          // The query of the guide's inference launch, at the vertex's place in the diffuse
          // queue: the surface point and shading normal the shade launch will scatter from.
          // Vertices that only do next-event estimation (depth 1) get a query too, unused.
          const uint4 h = W.hit[slot];
          const float4 o4 = W.ray_o[slot], d4 = W.ray_d[slot];
          TraceResult tr;
          tr.t = __uint_as_float(h.x);
          tr.rec = h.y;
          tr.tag = h.z;
          const Surface f = surface_at(s, mk(o4.x, o4.y, o4.z), mk(d4.x, d4.y, d4.z), tr);
          W.query[2 * size_t(pos)] = make_float4(f.hp.x, f.hp.y, f.hp.z, 0.0f);
          W.query[2 * size_t(pos) + 1] = make_float4(f.nrm.x, f.nrm.y, f.nrm.z, 0.0f);
        }
      }
    }
    bool started = false;
    if (free_slot) {
      const uint32_t rank = sh[3 * kWfScanStride + warp] + uint32_t(__popc(m_free & lanes_below()));
      if (rank < s_started) {
        const uint64_t item = s_first + rank;
        const uint32_t chunk = uint32_t(item / npix);
        Lane ln;
        ln.pixel = uint32_t(item - uint64_t(chunk) * npix);
        ln.sample = J.sample_base + chunk;
        start_sample(J, ln);
        W.ray_o[slot] = make_float4(ln.ro.x, ln.ro.y, ln.ro.z, -1.0f);
        W.ray_d[slot] = make_float4(ln.rd.x, ln.rd.y, ln.rd.z, 0.0f);
        W.thr[slot] = make_float4(1.0f, 1.0f, 1.0f, __uint_as_float(ln.pixel));
        W.rad[slot] = make_float4(0.0f, 0.0f, 0.0f, __uint_as_float(uint32_t(item)));
        W.rng[slot] = make_uint4(uint32_t(ln.rng.state), uint32_t(ln.rng.state >> 32), uint32_t(ln.rng.inc),
                                 uint32_t(ln.rng.inc >> 32));
        W.state[slot] = kWfAlive | kWfExtPending | kWfEmission | (uint32_t(ln.depth) & kWfDepthMask);
        const uint32_t pos = sh[3 * kWfScanStride + kWfScanStride - 1] + rank;
        W.ext_q[pos] = slot;
        if (W.sorted) W.ext_key[pos] = wf_sort_key(W, mk(0.f, 0.f, 0.f), kNoNode, false);
        started = true;
      } else if (st & kWfAlive) {
        W.state[slot] = 0u;
      }
    }
    n_live += (kind >= 0 || started) ? 1u : 0u;
  }
  // Path and live-slot counts: one atomic per block each.
  __shared__ unsigned long long s_paths;
  __shared__ uint32_t s_live;
  if (threadIdx.x == 0) {
    s_paths = 0ull;
    s_live = 0u;
  }
  __syncthreads();
  const unsigned long long tp = __reduce_add_sync(0xffffffffu, n_paths);
  const uint32_t tl = __reduce_add_sync(0xffffffffu, n_live);
  if ((threadIdx.x & 31u) == 0) {
    if (tp) atomicAdd(&s_paths, tp);
    if (tl) atomicAdd(&s_live, tl);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (s_paths) atomicAdd(W.r.counters, s_paths);
    if (s_live) atomicAdd(W.q + kWfLive, s_live);
  }
}

// At most 80 registers (6 blocks of 128 per SM): the kernel waits on memory, so the warps it keeps
// resident count for more than the few spilled words this costs.
template <bool kGuided>
__global__ void __launch_bounds__(128, 6) wf_shade_kernel(const WavefrontLaunch W) {
  const FrameJob& J = W.r.f;
  const DevScene& s = J.scene;
  __shared__ uint32_t sh[3 * kWfScanStride];
  const uint32_t n0 = W.q[kWfMatCount], n1 = W.q[kWfMatCount + 1], n2 = W.q[kWfMatCount + 2];
  const uint32_t total = n0 + n1 + n2;
  const uint32_t stride = gridDim.x * blockDim.x;
  // Entries are numbered diffuse, then metal, then dielectric, and a warp takes 32 consecutive
  // ones, so all but the warps at the two boundaries shade a single material. The loop bound is
  // uniform across the block (its appends synchronise the block).
  for (uint32_t base = blockIdx.x * blockDim.x; base < total; base += stride) {
    const uint32_t i = base + threadIdx.x;
    const bool valid = i < total;
    uint32_t slot = 0, kind = 0;
    if (valid) {
      if (i < n0) {
        slot = W.mat_q[i];
      } else if (i < n0 + n1) {
        kind = kMetal;
        slot = W.mat_q[size_t(W.capacity) + (i - n0)];
      } else {
        kind = kDielectric;
        slot = W.mat_q[2 * size_t(W.capacity) + (i - n0 - n1)];
      }
    }
    bool shadow_l = false, shadow_e = false, extend = false;
    bool rec_s = false, rec_e = false;  // recording: this vertex's scatter and environment records
    V3 talb = mk(0.f, 0.f, 0.f);        // throughput x albedo before the scatter
    float env_w = 0.0f;
    uint32_t h_rec = kNoNode;  // primitive record of the vertex (sort key of the rays it spawns)
    Lane ln;
    float4 c0 = make_float4(0.f, 0.f, 0.f, 0.f), c1 = c0;
    float4 sl0, sl1, se0, se1;
    uint32_t nst = kWfAlive;
    if (valid) {
      const float4 o4 = W.ray_o[slot], d4 = W.ray_d[slot], t4 = W.thr[slot];
      const uint4 r4 = W.rng[slot], h = W.hit[slot];
      const uint32_t st = W.state[slot];
      ln.ro = mk(o4.x, o4.y, o4.z);
      ln.rd = mk(d4.x, d4.y, d4.z);
      ln.thr = mk(t4.x, t4.y, t4.z);
      ln.rng.state = uint64_t(r4.x) | (uint64_t(r4.y) << 32);
      ln.rng.inc = uint64_t(r4.z) | (uint64_t(r4.w) << 32);
      ln.depth = int(st & kWfDepthMask);
      TraceResult tr;
      tr.t = __uint_as_float(h.x);
      tr.rec = h.y;
      tr.tag = h.z;
      h_rec = h.y;
      const Surface f = surface_at(s, ln.ro, ln.rd, tr);
      const DevMaterial m = s.materials[f.mat];
      float bsdf_pdf = -1.0f;
      if (kind == kDiffuse) {
        ln.hp = f.hp;
        ln.hn = f.nrm;
        ln.alb = base_color(s, m, f.tu, f.tv);
        // Guided: a vertex that will scatter (depth > 1) uses the mixture inferred for its place i
        // in the diffuse queue, in the environment NEE weight and in the bounce, as render_kernel's
        // guided mode does.
        ln.mix_slot = (kGuided && ln.depth > 1) ? int(i) : -1;
        if (prepare_light_shadow(s, ln)) {
          shadow_l = true;
          sl0 = make_float4(ln.ro.x, ln.ro.y, ln.ro.z, ln.tmax);
          sl1 = make_float4(ln.rd.x, ln.rd.y, ln.rd.z, __uint_as_float(2u * slot));
          c0 = make_float4(ln.pend.x, ln.pend.y, ln.pend.z, 0.0f);
        }
        if (prepare_env_shadow<kGuided ? kModeGuided : kModePlain, true>(W.r, J, ln)) {
          shadow_e = true;
          se0 = make_float4(ln.ro.x, ln.ro.y, ln.ro.z, ln.tmax);
          se1 = make_float4(ln.rd.x, ln.rd.y, ln.rd.z, __uint_as_float(2u * slot + 1u));
          // w = 1 marks the entry as not (yet) occluded: an occluded shadow ray clears it.
          c1 = make_float4(ln.pend.x, ln.pend.y, ln.pend.z, 1.0f);
          env_w = ln.nee_w;
          rec_e = env_w > 0.0f;
        }
        W.nee[2 * size_t(slot)] = c0;
        W.nee[2 * size_t(slot) + 1] = c1;
        nst |= kWfNeePending;
        ln.depth -= 1;
        if (ln.depth > 0) {
          talb = ln.thr * ln.alb;
          if (kGuided && ln.mix_slot >= 0) {
            extend = take_guided_bounce(W.r.g, W.r.g.in_mix + 10 * size_t(ln.mix_slot), ln);
          } else {
            take_diffuse_bounce(ln, cosine_direction(ln));
            extend = true;
          }
          bsdf_pdf = ln.bsdf_pdf;
          rec_s = extend;
        }
      } else {
        const bool on = kind == kMetal ? bounce_metal(ln, m, f) : (bounce_dielectric(ln, m, f), true);
        ln.depth -= 1;
        extend = on && ln.depth > 0;
        nst |= kWfEmission;
      }
      if (extend) nst |= kWfExtPending | (uint32_t(ln.depth) & kWfDepthMask);
      else nst |= kWfTerminate;
      W.ray_o[slot] = make_float4(ln.ro.x, ln.ro.y, ln.ro.z, bsdf_pdf);
      W.ray_d[slot] = make_float4(ln.rd.x, ln.rd.y, ln.rd.z, 0.0f);
      W.thr[slot] = make_float4(ln.thr.x, ln.thr.y, ln.thr.z, t4.w);
      W.rng[slot] = make_uint4(uint32_t(ln.rng.state), uint32_t(ln.rng.state >> 32), uint32_t(ln.rng.inc),
                               uint32_t(ln.rng.inc >> 32));
      W.state[slot] = nst;
    }
    // Queue positions for this step's shadow rays, extension rays and (recording) training records:
    // one block-wide reservation on the three counters.
    const bool recording = W.r.g.records != nullptr;
    uint32_t* const counters[3] = {W.q + kWfShadowCount, W.q + kWfExtCount, W.r.g.record_count};
    const uint32_t want[3] = {uint32_t(shadow_l) + uint32_t(shadow_e), extend ? 1u : 0u,
                              recording ? uint32_t(rec_s) + uint32_t(rec_e) : 0u};
    uint32_t at[3];
    block_reserve<3>(counters, want, at, sh);
    if (recording && valid && kind == kDiffuse) {
      // Training records of the diffuse vertices (render_kernel's record mode): the scatter
      // (position + work item, normal + T.x, direction + T.y, radiance so far + T.z, with T the
      // throughput times albedo before the scatter; the next logic launch fills in the radiance)
      // and the environment shadow ray with its weight. T / (the scattered throughput) is
      // cos / (pi p) for a direction drawn with pdf p, so (radiance gathered after the vertex) / T
      // weighs a guided direction by cos L_i / p as the training loss wants.
      const uint32_t cap = W.r.g.record_capacity;
      const uint32_t ps = at[2], pn = at[2] + (rec_s ? 1u : 0u);
      uint2 ref = make_uint2(kNoNode, kNoNode);
      const float item = reinterpret_cast<const float*>(W.rad + slot)[3];
      if (rec_s && ps < cap) {
        float4* r = W.r.g.records + 4 * size_t(ps);
        r[0] = make_float4(ln.hp.x, ln.hp.y, ln.hp.z, item);
        r[1] = make_float4(ln.hn.x, ln.hn.y, ln.hn.z, talb.x);
        r[2] = make_float4(ln.rd.x, ln.rd.y, ln.rd.z, talb.y);
        r[3] = make_float4(0.0f, 0.0f, 0.0f, talb.z);
        ref.x = ps;
      }
      if (rec_e && pn < cap) {
        float4* r = W.r.g.records + 4 * size_t(pn);
        r[0] = make_float4(ln.hp.x, ln.hp.y, ln.hp.z, __uint_as_float(kNeeRecord));
        r[1] = make_float4(ln.hn.x, ln.hn.y, ln.hn.z, 0.0f);
        r[2] = make_float4(se1.x, se1.y, se1.z, 0.0f);
        r[3] = make_float4(env_w, 0.0f, 0.0f, 0.0f);
        ref.y = pn;
      }
      W.rec_ref[slot] = ref;
    }
    if (shadow_l) {
      const uint32_t pl = at[0];
      if (W.sorted) W.shadow_key[pl] = wf_sort_key(W, mk(sl1.x, sl1.y, sl1.z), h_rec, true);
      W.shadow_q[2 * size_t(pl)] = sl0;
      W.shadow_q[2 * size_t(pl) + 1] = sl1;
    }
    if (shadow_e) {
      const uint32_t pe = at[0] + (shadow_l ? 1u : 0u);
      if (W.sorted) W.shadow_key[pe] = wf_sort_key(W, mk(se1.x, se1.y, se1.z), h_rec, true);
      W.shadow_q[2 * size_t(pe)] = se0;
      W.shadow_q[2 * size_t(pe) + 1] = se1;
    }
    if (extend) {
      const uint32_t px = at[1];
      W.ext_q[px] = slot;
      if (W.sorted) W.ext_key[px] = wf_sort_key(W, ln.rd, h_rec, false);
    }
  }
}

// Loads queue entry i (extension rays first, then shadow rays) as a ray with its distance limit.
template <bool kSorted>
__device__ __forceinline__ RayQ wf_entry_ray(const WavefrontLaunch& W, uint32_t i, uint32_t n_ext, float& tmax,
                                             uint32_t& target) {
  if constexpr (kSorted) i = W.sorted[i];  // sorted position -> queue entry (extension entries sort first)
  if (i < n_ext) {
    target = W.ext_q[i];
    const float4 o = W.ray_o[target], d = W.ray_d[target];
    tmax = CUDART_INF_F;
    return make_ray(o.x, o.y, o.z, d.x, d.y, d.z);
  }
  const size_t j = i - n_ext;
  const float4 a = W.shadow_q[2 * j], b = W.shadow_q[2 * j + 1];
  tmax = a.w;
  target = __float_as_uint(b.w);
  return make_ray(a.x, a.y, a.z, b.x, b.y, b.z);
}

// Result of queue entry i: the closest hit of an extension ray, or the occlusion of a shadow ray
// (an occluded shadow ray drops its contribution, integrator.rs:196-199 and :233-238). An extension
// hit also records its material (index in bits 0-27, kind in bits 28-31), which the primitive
// record just tested holds, so the logic launch needs no dependent loads to classify the slot.
__device__ __forceinline__ void wf_entry_result(const WavefrontLaunch& W, uint32_t i, uint32_t n_ext, uint32_t target,
                                                bool hit, float t, uint32_t rec, uint32_t tag) {
  if (i < n_ext) {
    uint32_t mat = 0u;
    if (hit) {
      const uint32_t m = __float_as_uint(__ldg(&W.r.f.scene.prims[rec].b[3]));
      mat = m | (__ldg(&W.r.f.scene.materials[m].kind) << kWfKindShift);
    }
    W.hit[target] = make_uint4(__float_as_uint(t), hit ? rec : kNoNode, hit ? tag : 0u, mat);
  } else if (hit) {
    W.nee[target] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
}

// kRefill = false: a warp takes 32 consecutive queue entries and traces each to its end.
// kRefill = true: dynamic ray fetching; a lane whose ray is done takes the next queue entry as
// soon as fewer than W.refill_lanes lanes of its warp are still traversing (the others keep
// their traversal state and stack meanwhile).
// kWatertight: the watertight triangle test over the scene's vertex records.
// kSorted: queue entries are taken in the order of W.sorted (ray sorting).
template <bool kRefill, bool kWatertight, bool kSorted>
__global__ void __launch_bounds__(128) wf_trace_kernel(const WavefrontLaunch W) {
  static_assert(!(kRefill && kWatertight), "the resumable traversal tests triangles with Moller-Trumbore");
  __shared__ ChildRec root;
  __shared__ unsigned long long s_count[2];
  if (threadIdx.x == 0) root = *W.r.f.scene.root;
  if (threadIdx.x < 2) s_count[threadIdx.x] = 0ull;
  __syncthreads();
  const DevScene& s = W.r.f.scene;
  const uint32_t n_ext = W.q[kWfExtCount], total = n_ext + W.q[kWfShadowCount];
  const unsigned lane = threadIdx.x & 31u;
  uint32_t c_ext = 0, c_sh = 0, visits = 0;
  if constexpr (!kRefill) {
    // Extension rays come first, then shadow rays, so a warp traces one kind of ray (only the
    // warp at the boundary holds both).
    for (;;) {
      uint32_t base = 0;
      if (lane == 0) base = atomicAdd(W.q + kWfTraceCursor, 32u);
      base = __shfl_sync(0xffffffffu, base, 0);
      if (base >= total) break;
      const uint32_t i = base + lane;
      if (i < total) {
        float tmax;
        uint32_t target;
        const RayQ q = wf_entry_ray<kSorted>(W, i, n_ext, tmax, target);
        TraceResult tr;
        bool hit;
        if (i < n_ext) {
          hit = trace_ray<kWatertight>(s.pairs, s.prims, root, q, kRayEps, tmax, false, tr, visits, s.tri_verts);
          ++c_ext;
        } else {
          hit = trace_ray<kWatertight>(s.pairs, s.prims, root, q, kRayEps, tmax, true, tr, visits, s.tri_verts);
          ++c_sh;
        }
        wf_entry_result(W, i, n_ext, target, hit, tr.t, tr.rec, tr.tag);
      }
    }
  } else {
    Traversal T;
    T.cur = kNoNode;
    RayQ q = make_ray(0.f, 0.f, 0.f, 1.f, 1.f, 1.f);
    uint32_t idx = 0, target = 0;
    bool busy = false, exhausted = false;
    uint2 st_local[kMaxStack];
    for (;;) {
      // Lanes without a ray take the next entries, one atomic per warp.
      const bool need = !busy && !exhausted;
      const unsigned m = __ballot_sync(0xffffffffu, need);
      if (m) {
        const int leader = __ffs(m) - 1;
        uint32_t base = 0;
        if (int(lane) == leader) base = atomicAdd(W.q + kWfTraceCursor, uint32_t(__popc(m)));
        base = __shfl_sync(0xffffffffu, base, leader);
        if (need) {
          idx = base + uint32_t(__popc(m & lanes_below()));
          if (idx < total) {
            float tmax;
            q = wf_entry_ray<kSorted>(W, idx, n_ext, tmax, target);
            trav_start(T, root, q, kRayEps, tmax);
            busy = true;
            if (idx < n_ext) ++c_ext;
            else ++c_sh;
          } else {
            exhausted = true;
          }
        }
      }
      if (!__any_sync(0xffffffffu, busy)) break;
      trav_advance(T, q, kRayEps, idx >= n_ext, s.pairs, s.prims, st_local, nullptr, 0, 0, W.refill_lanes,
                   !exhausted, visits);
      if (busy && T.cur == kNoNode) {
        wf_entry_result(W, idx, n_ext, target, T.found(), T.closest, T.rec, T.tag);
        busy = false;
      }
    }
  }
  const unsigned long long te = __reduce_add_sync(0xffffffffu, c_ext);
  const unsigned long long ts = __reduce_add_sync(0xffffffffu, c_sh);
  if (lane == 0) {
    if (te) atomicAdd(&s_count[0], te);
    if (ts) atomicAdd(&s_count[1], ts);
  }
  __syncthreads();
  if (threadIdx.x < 2 && s_count[threadIdx.x] != 0ull) atomicAdd(W.r.counters + 1 + threadIdx.x, s_count[threadIdx.x]);
}

// Counting sort of one iteration's queued rays by key (extension entries 0..n_ext, then shadow
// entries): block b of kWfSortBlocks counts the keys of its contiguous share of the entries in
// shared memory and stores its counts bin-major; a one-block scan turns the counts into each
// (bin, block)'s first position; the scatter pass repeats the partition and places every entry.
__device__ __forceinline__ void wf_sort_share(const WavefrontLaunch& W, uint32_t& begin, uint32_t& end,
                                              uint32_t& n_ext) {
  n_ext = W.q[kWfExtCount];
  const uint32_t n = n_ext + W.q[kWfShadowCount];
  const uint32_t chunk = (n + gridDim.x - 1) / gridDim.x;
  begin = min(n, blockIdx.x * chunk);
  end = min(n, begin + chunk);
}

__global__ void __launch_bounds__(512) wf_sort_count_kernel(const WavefrontLaunch W) {
  __shared__ uint32_t hist[kWfSortBins];
  for (int b = threadIdx.x; b < kWfSortBins; b += blockDim.x) hist[b] = 0u;
  __syncthreads();
  uint32_t begin, end, n_ext;
  wf_sort_share(W, begin, end, n_ext);
  for (uint32_t i = begin + threadIdx.x; i < end; i += blockDim.x)
    atomicAdd(&hist[i < n_ext ? W.ext_key[i] : W.shadow_key[i - n_ext]], 1u);
  __syncthreads();
  for (int b = threadIdx.x; b < kWfSortBins; b += blockDim.x) W.sort_counts[b * kWfSortBlocks + blockIdx.x] = hist[b];
}

__global__ void __launch_bounds__(1024) wf_sort_scan_kernel(const WavefrontLaunch W) {
  constexpr uint32_t kN = uint32_t(kWfSortBins) * kWfSortBlocks;
  __shared__ uint32_t part[1024];
  const uint32_t per = (kN + 1023) / 1024;
  const uint32_t begin = min(kN, threadIdx.x * per), end = min(kN, begin + per);
  uint32_t sum = 0;
  for (uint32_t i = begin; i < end; ++i) sum += W.sort_counts[i];
  part[threadIdx.x] = sum;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t run = 0;
    for (int t = 0; t < 1024; ++t) {
      const uint32_t c = part[t];
      part[t] = run;
      run += c;
    }
  }
  __syncthreads();
  uint32_t run = part[threadIdx.x];
  for (uint32_t i = begin; i < end; ++i) {
    const uint32_t c = W.sort_counts[i];
    W.sort_counts[i] = run;
    run += c;
  }
}

__global__ void __launch_bounds__(512) wf_sort_scatter_kernel(const WavefrontLaunch W) {
  __shared__ uint32_t cursor[kWfSortBins];
  for (int b = threadIdx.x; b < kWfSortBins; b += blockDim.x) cursor[b] = W.sort_counts[b * kWfSortBlocks + blockIdx.x];
  __syncthreads();
  uint32_t begin, end, n_ext;
  wf_sort_share(W, begin, end, n_ext);
  for (uint32_t i = begin + threadIdx.x; i < end; i += blockDim.x) {
    const uint32_t key = i < n_ext ? W.ext_key[i] : W.shadow_key[i - n_ext];
    W.sorted[atomicAdd(&cursor[key], 1u)] = i;
  }
}

// Resident blocks per SM of a kernel at a block size.
template <class K>
static int resident_blocks(K kernel, int block) {
  int blocks = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kernel, block, 0) != cudaSuccess) return 1;
  return blocks > 0 ? blocks : 1;
}

cudaError_t launch_wavefront_iteration(const WavefrontLaunch& w, bool moments, int sm_count, cudaStream_t stream,
                                       const GuideDevice* guide, const cudaEvent_t* marks) {
  static const int shade_per_sm = resident_blocks(wf_shade_kernel<false>, 128);
  static const int guided_shade_per_sm = resident_blocks(wf_shade_kernel<true>, 128);
  static const int trace_per_sm = resident_blocks(wf_trace_kernel<false, false, false>, 128);
  static const int sorted_per_sm = resident_blocks(wf_trace_kernel<false, false, true>, 128);
  static const int refill_per_sm = resident_blocks(wf_trace_kernel<true, false, false>, 128);
  static const int watertight_per_sm = resident_blocks(wf_trace_kernel<false, true, false>, 128);
  const unsigned logic_grid = unsigned((uint64_t(w.capacity) + kWfBlock - 1) / kWfBlock);
  auto mark = [&](int i) {
    if (marks) cudaEventRecord(marks[i], stream);
  };
  mark(0);
  if (guide) {
    // Guided: the diffuse queue's queries are inferred between the logic and shade launches.
    if (moments) wf_logic_kernel<true, true><<<logic_grid, kWfBlock, 0, stream>>>(w);
    else wf_logic_kernel<false, true><<<logic_grid, kWfBlock, 0, stream>>>(w);
    mark(1);
    cudaError_t e = guide_launch_infer(*guide, w.query, w.capacity, const_cast<float4*>(w.r.g.in_mix), sm_count,
                                       stream, w.q + kWfMatCount);
    if (e != cudaSuccess) return e;
    mark(2);
    wf_shade_kernel<true><<<guided_shade_per_sm * sm_count, 128, 0, stream>>>(w);
  } else {
    if (moments) wf_logic_kernel<true, false><<<logic_grid, kWfBlock, 0, stream>>>(w);
    else wf_logic_kernel<false, false><<<logic_grid, kWfBlock, 0, stream>>>(w);
    mark(1);  // no inference: marks[2] stays unrecorded
    wf_shade_kernel<false><<<shade_per_sm * sm_count, 128, 0, stream>>>(w);
  }
  mark(3);
  // Ray sorting applies to the plain trace launch (the watertight and refilling ones take the
  // queues in append order).
  const bool sorted = w.sorted && !w.r.f.scene.tri_verts && w.refill_lanes <= 1;
  if (sorted) {
    wf_sort_count_kernel<<<kWfSortBlocks, 512, 0, stream>>>(w);
    wf_sort_scan_kernel<<<1, 1024, 0, stream>>>(w);
    wf_sort_scatter_kernel<<<kWfSortBlocks, 512, 0, stream>>>(w);
    wf_trace_kernel<false, false, true><<<sorted_per_sm * sm_count, 128, 0, stream>>>(w);
  } else if (w.r.f.scene.tri_verts) {
    wf_trace_kernel<false, true, false><<<watertight_per_sm * sm_count, 128, 0, stream>>>(w);
  } else if (w.refill_lanes > 1) {
    wf_trace_kernel<true, false, false><<<refill_per_sm * sm_count, 128, 0, stream>>>(w);
  } else {
    wf_trace_kernel<false, false, false><<<trace_per_sm * sm_count, 128, 0, stream>>>(w);
  }
  mark(4);
  return cudaGetLastError();
}

// ------------------------------------------------------------------------ training samples
// Training samples from the recorded scatters, appended to the sample pool (`out`, `out_capacity`
// samples; `out_count` and `weight_sum` keep running across batches). Only scatters whose
// direction carried radiance are kept (compacted through one atomic per warp): a zero weight adds
// nothing to the weighted likelihood, and in dim interiors most recorded directions carry none,
// so uniform draws over all records would leave almost every batch slot empty. Samples past the
// pool's capacity are dropped, and their weights left out of the sum.
__global__ void guide_samples_kernel(const float4* __restrict__ rec, const uint32_t* __restrict__ count,
                                     uint32_t capacity, const float4* __restrict__ path_rad,
                                     float4* __restrict__ out, uint32_t out_capacity, uint32_t* __restrict__ out_count,
                                     float* __restrict__ weight_sum) {
  const uint32_t n = min(*count, capacity);
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  float w = 0.0f;
  float4 a = make_float4(0, 0, 0, 0), b = a, c = a;
  if (i < n) {
    a = rec[4 * size_t(i)];
    b = rec[4 * size_t(i) + 1];
    c = rec[4 * size_t(i) + 2];
    const float4 d = rec[4 * size_t(i) + 3];
    if (__float_as_uint(a.w) == kNeeRecord) {
      w = d.x;  // environment shadow ray that reached the sky: its weight was computed at record time
    } else {
      const float4 end = path_rad[__float_as_uint(a.w)];
      // Radiance that arrived along the scattered direction: what the path gathered after this
      // vertex, divided by the throughput it had just after scattering.
      const float lx = b.w > 0.0f ? fmaxf(end.x - d.x, 0.0f) / b.w : 0.0f;
      const float ly = c.w > 0.0f ? fmaxf(end.y - d.y, 0.0f) / c.w : 0.0f;
      const float lz = d.w > 0.0f ? fmaxf(end.z - d.z, 0.0f) / d.w : 0.0f;
      w = 0.2126f * lx + 0.7152f * ly + 0.0722f * lz;
    }
    if (!(w > 0.0f) || !isfinite(w)) w = 0.0f;
  }
  const bool keep = w > 0.0f;
  const unsigned mask = __ballot_sync(0xffffffffu, keep);
  const unsigned lane = threadIdx.x & 31u;
  uint32_t base = 0;
  if (mask) {
    const int leader = __ffs(mask) - 1;
    if (int(lane) == leader) base = atomicAdd(out_count, uint32_t(__popc(mask)));
    base = __shfl_sync(0xffffffffu, base, leader);
  }
  if (keep) {
    const uint32_t slot = base + uint32_t(__popc(mask & ((1u << lane) - 1u)));
    if (slot < out_capacity) {
      out[3 * size_t(slot)] = make_float4(a.x, a.y, a.z, w);
      out[3 * size_t(slot) + 1] = make_float4(b.x, b.y, b.z, 0.0f);
      out[3 * size_t(slot) + 2] = make_float4(c.x, c.y, c.z, 0.0f);
    } else {
      w = 0.0f;
    }
  }
  for (int o = 16; o > 0; o >>= 1) w += __shfl_down_sync(0xffffffffu, w, o);
  if (lane == 0 && w != 0.0f) atomicAdd(weight_sum, w);
}

cudaError_t launch_guide_samples(const float4* records, const uint32_t* record_count, uint32_t capacity,
                                 const float4* path_radiance, float4* samples, uint32_t sample_capacity,
                                 uint32_t* sample_count, float* weight_sum, cudaStream_t stream) {
  if (capacity == 0) return cudaSuccess;
  guide_samples_kernel<<<(capacity + 255) / 256, 256, 0, stream>>>(records, record_count, capacity, path_radiance,
                                                                   samples, sample_capacity, sample_count,
                                                                   weight_sum);
  return cudaGetLastError();
}

// ------------------------------------------------------------------------ scratch without allocation
// Scratch of tc_render_no_alloc: [0] the work-queue counter, [1..3] the path, extension-ray and
// shadow-ray counters. Every GPU that loads the library holds these 256 bytes until exit; all
// calls share them, so the entry point clears them at the start of each call, and calls whose
// kernels overlap on the GPU race on them.
static __device__ __align__(256) unsigned long long g_render_scratch[kStaticScratchWords];

cudaError_t render_static_scratch(int device, unsigned long long** out) {
  // Host code must never hand the array's name itself to a kernel: it is only a host-side
  // stand-in. The device address belongs to the CUDA context current now (the one the library
  // module was loaded into), so it is looked up with `device` current and kept by the caller
  // beside the other resources of that context rather than in a process-wide table, which a
  // cudaDeviceReset or a host's own driver context would leave pointing at freed memory.
  int current = 0;
  cudaError_t e = cudaGetDevice(&current);
  if (e != cudaSuccess) return e;
  if (current != device) return cudaErrorInvalidDevice;
  void* ptr = nullptr;
  e = cudaGetSymbolAddress(&ptr, g_render_scratch);
  if (e != cudaSuccess) return e;
  *out = static_cast<unsigned long long*>(ptr);
  return cudaSuccess;
}

// ------------------------------------------------------------------------ resolve
__global__ void resolve_kernel(const double* __restrict__ accum, uint32_t pixels, double inv_samples,
                               float4* __restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= pixels) return;
  const double* a = accum + size_t(3) * i;
  out[i] = make_float4(float(a[0] * inv_samples), float(a[1] * inv_samples), float(a[2] * inv_samples), 1.0f);
}

cudaError_t launch_resolve(const double* accum, uint32_t pixels, double inv_samples, float4* out,
                           cudaStream_t stream) {
  if (pixels == 0) return cudaSuccess;
  resolve_kernel<<<(pixels + 255) / 256, 256, 0, stream>>>(accum, pixels, inv_samples, out);
  return cudaGetLastError();
}

// ------------------------------------------------------------------------ environment tables
// Weights follow environment.rs:245-260: luminance * sin(theta_row_centre) * intensity in FP64.
// Row kernel: one block per row; FP64 block reduction for the row sum, then an FP64 inclusive
// scan written as the normalised conditional CDF (last entry forced to 1).
constexpr int kEnvBlock = 256;

__device__ __forceinline__ double env_weight(const float4 t, double sin_theta, double intensity) {
  const double lum = 0.2126 * double(t.x) + 0.7152 * double(t.y) + 0.0722 * double(t.z);
  return lum * sin_theta * intensity;
}

__device__ double block_sum(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  double total = 0.0;
  if (threadIdx.x == 0) {
    for (int w = 0; w < kEnvBlock / 32; ++w) total += sh[w];
    sh[kEnvBlock / 32] = total;
  }
  __syncthreads();
  total = sh[kEnvBlock / 32];
  __syncthreads();
  return total;
}

// Inclusive scan of one value per thread across the block (FP64); returns the prefix.
__device__ double block_scan(double v, double* sh) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int o = 1; o < 32; o <<= 1) {
    const double n = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += n;
  }
  if (lane == 31) sh[warp] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double run = 0.0;
    for (int w = 0; w < kEnvBlock / 32; ++w) {
      const double t = sh[w];
      sh[w] = run;
      run += t;
    }
  }
  __syncthreads();
  v += sh[warp];
  __syncthreads();
  return v;
}

__global__ void env_rows_kernel(const float4* __restrict__ rgb, uint32_t w, uint32_t h, double intensity,
                                float* __restrict__ conditional, double* __restrict__ row_sums) {
  __shared__ double sh[kEnvBlock / 32 + 1];
  __shared__ double tile_end;
  const uint32_t y = blockIdx.x;
  const double sin_theta = sin(CUDART_PI * (double(y) + 0.5) / double(h));
  const float4* row = rgb + size_t(y) * w;
  double local = 0.0;
  for (uint32_t x = threadIdx.x; x < w; x += kEnvBlock) local += env_weight(row[x], sin_theta, intensity);
  const double total = block_sum(local, sh);
  if (threadIdx.x == 0) row_sums[y] = total;
  float* out = conditional + size_t(y) * w;
  if (!(total > 0.0) || !isfinite(total)) {
    for (uint32_t x = threadIdx.x; x < w; x += kEnvBlock) out[x] = float(double(x + 1) / double(w));
    return;
  }
  double carry = 0.0;
  for (uint32_t base = 0; base < w; base += kEnvBlock) {
    const uint32_t x = base + threadIdx.x;
    const double v = x < w ? env_weight(row[x], sin_theta, intensity) : 0.0;
    const double incl = block_scan(v, sh) + carry;
    if (x < w) out[x] = (x == w - 1) ? 1.0f : float(incl / total);
    // The carry into the next tile is the inclusive value of the tile's last thread.
    if (threadIdx.x == kEnvBlock - 1) tile_end = incl;
    __syncthreads();
    carry = tile_end;
    __syncthreads();
  }
}

__global__ void env_marginal_kernel(const double* __restrict__ row_sums, uint32_t h, float* __restrict__ marginal,
                                    double* __restrict__ total_out) {
  __shared__ double sh[kEnvBlock / 32 + 1];
  double local = 0.0;
  for (uint32_t y = threadIdx.x; y < h; y += kEnvBlock) local += row_sums[y];
  const double total = block_sum(local, sh);
  if (threadIdx.x == 0) *total_out = total;
  if (!(total > 0.0) || !isfinite(total)) {
    for (uint32_t y = threadIdx.x; y < h; y += kEnvBlock) marginal[y] = 0.0f;
    return;
  }
  __shared__ double tile_end;
  double carry = 0.0;
  for (uint32_t base = 0; base < h; base += kEnvBlock) {
    const uint32_t y = base + threadIdx.x;
    const double v = y < h ? row_sums[y] : 0.0;
    const double incl = block_scan(v, sh) + carry;
    if (y < h) marginal[y] = (y == h - 1) ? 1.0f : float(incl / total);
    if (threadIdx.x == kEnvBlock - 1) tile_end = incl;
    __syncthreads();
    carry = tile_end;
    __syncthreads();
  }
}

// Per-texel numerator of the solid-angle density: P(row) * P(column | row) * W * H / (2 pi^2),
// both probabilities taken from the stored FP32 CDFs the sampler inverts.
__global__ void env_pdf_kernel(const float* __restrict__ marginal, const float* __restrict__ conditional,
                               uint32_t w, uint32_t h, const double* __restrict__ total, float* __restrict__ pdf) {
  const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= size_t(w) * h) return;
  const double t = *total;
  if (!(t > 0.0) || !isfinite(t)) {
    pdf[i] = 0.0f;
    return;
  }
  const uint32_t y = uint32_t(i / w), x = uint32_t(i - size_t(y) * w);
  const double py = double(marginal[y]) - (y ? double(marginal[y - 1]) : 0.0);
  const float* row = conditional + size_t(y) * w;
  const double px = double(row[x]) - (x ? double(row[x - 1]) : 0.0);
  const double p = fmax(py, 0.0) * fmax(px, 0.0);
  pdf[i] = float(p * double(w) * double(h) / (2.0 * CUDART_PI * CUDART_PI));
}

// Walker alias tables of the importance distribution (Vose's construction): table y < h is row
// y's distribution over its columns, table h the marginal over rows. The weights are the FP32 CDF
// differences env_pdf_kernel turns into densities, so the sampler draws each texel with exactly the
// probability its density reports. An entry is (probability of keeping the drawn index, as float
// bits; the index taken otherwise). One warp per table: the lanes read and sum the weights, lane 0
// runs the construction (it is sequential) on the table's working set, held in shared memory
// (max(w, h) doubles and 2 x max(w, h) indices) or, for maps too wide for it, in `scratch_q` /
// `scratch_idx` (the same amounts per table).
__global__ void __launch_bounds__(32) env_alias_kernel(const float* __restrict__ marginal,
                                                       const float* __restrict__ conditional, uint32_t w, uint32_t h,
                                                       bool in_shared, double* __restrict__ scratch_q,
                                                       uint32_t* __restrict__ scratch_idx, uint2* __restrict__ cond_alias,
                                                       uint2* __restrict__ marg_alias) {
  extern __shared__ __align__(16) uint8_t env_sm[];
  const uint32_t t = blockIdx.x, lane = threadIdx.x;
  const uint32_t span = max(w, h);
  const bool marg = t == h;
  const uint32_t n = marg ? h : w;
  const float* cdf = marg ? marginal : conditional + size_t(t) * w;
  uint2* out = marg ? marg_alias : cond_alias + size_t(t) * w;
  double* q = in_shared ? reinterpret_cast<double*>(env_sm) : scratch_q + size_t(t) * span;
  uint32_t* small = in_shared ? reinterpret_cast<uint32_t*>(q + span) : scratch_idx + size_t(t) * 2 * span;
  uint32_t* large = small + span;
  double part = 0.0;
  for (uint32_t i = lane; i < n; i += 32) {
    const double p = fmax(double(cdf[i]) - (i ? double(cdf[i - 1]) : 0.0), 0.0);
    q[i] = p;
    part += p;
  }
  for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
  const double sum = part;
  if (!(sum > 0.0) || !isfinite(sum)) {
    for (uint32_t i = lane; i < n; i += 32) out[i] = make_uint2(__float_as_uint(1.0f), i);
    return;
  }
  const double scale = double(n) / sum;
  for (uint32_t i = lane; i < n; i += 32) q[i] *= scale;
  __syncwarp();
  if (lane != 0) return;
  uint32_t ns = 0, nl = 0;
  for (uint32_t i = 0; i < n; ++i) {
    if (q[i] < 1.0) small[ns++] = i;
    else large[nl++] = i;
  }
  while (ns && nl) {
    const uint32_t sm = small[--ns], lg = large[--nl];
    out[sm] = make_uint2(__float_as_uint(float(q[sm])), lg);
    q[lg] = (q[lg] + q[sm]) - 1.0;
    if (q[lg] < 1.0) small[ns++] = lg;
    else large[nl++] = lg;
  }
  // Leftovers hold probability 1 up to rounding.
  while (nl) {
    const uint32_t lg = large[--nl];
    out[lg] = make_uint2(__float_as_uint(1.0f), lg);
  }
  while (ns) {
    const uint32_t sm = small[--ns];
    out[sm] = make_uint2(__float_as_uint(1.0f), sm);
  }
}

cudaError_t launch_env_tables(const float4* rgb, uint32_t w, uint32_t h, float intensity, float* marginal,
                              float* conditional, float* pdf, double* row_sums, double* total_out,
                              double* alias_q, uint32_t* alias_idx, uint2* cond_alias, uint2* marg_alias,
                              cudaStream_t stream) {
  if (w == 0 || h == 0) return cudaSuccess;
  env_rows_kernel<<<h, kEnvBlock, 0, stream>>>(rgb, w, h, double(intensity), conditional, row_sums);
  env_marginal_kernel<<<1, kEnvBlock, 0, stream>>>(row_sums, h, marginal, total_out);
  const size_t n = size_t(w) * h;
  env_pdf_kernel<<<unsigned((n + 255) / 256), 256, 0, stream>>>(marginal, conditional, w, h, total_out, pdf);
  // The working set of one table in shared memory when it fits (maps up to 12,800 texels wide).
  const size_t table_bytes = size_t(std::max(w, h)) * (sizeof(double) + 2 * sizeof(uint32_t));
  const bool in_shared = env_alias_in_shared(w, h);
  if (in_shared) {
    const cudaError_t e =
        cudaFuncSetAttribute(env_alias_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(table_bytes));
    if (e != cudaSuccess) return e;
  }
  env_alias_kernel<<<h + 1, 32, in_shared ? table_bytes : 0, stream>>>(marginal, conditional, w, h, in_shared,
                                                                       alias_q, alias_idx, cond_alias, marg_alias);
  return cudaGetLastError();
}

}  // namespace tcb
