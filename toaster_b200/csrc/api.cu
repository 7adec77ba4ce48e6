// Host runtime and C ABI of the toaster B200 path tracer (see include/toaster_cuda.h).
//
// Ownership follows the reference boundary (crates/toaster-gpu/src/path_tracer.rs:518-849):
// the caller owns host arrays, the context owns every device buffer and one stream, and each
// call is synchronous like dispatch_compute_2d's device.poll(Wait) (dispatch.rs:57).
#include <cuda_runtime.h>
#include <nvjpeg.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <array>
#include <vector>

#include "../../include/toaster_cuda.h"
#include "bvh_build.h"
#include "bvh_device.h"
#include "device_scene.h"
#include "display.h"
#include "guide.h"
#include "layout.h"
#include "refit.h"

static_assert(sizeof(tc_gpu_render_params) == 96, "GpuRenderParams is 96 bytes");
static_assert(sizeof(tc_gpu_camera) == 64, "GpuCamera is 64 bytes");
static_assert(sizeof(tc_gpu_sphere) == 32, "GpuSphere is 32 bytes");
static_assert(sizeof(tc_gpu_triangle) == 64, "GpuTriangle is 64 bytes");
static_assert(sizeof(tc_gpu_triangle_attributes) == 80, "GpuTriangleAttributes is 80 bytes");
static_assert(sizeof(tc_gpu_material) == 48, "GpuMaterial is 48 bytes");
static_assert(sizeof(tc_gpu_light) == 96, "GpuLight is 96 bytes");
static_assert(sizeof(tc_gpu_bvh_node) == 48, "GpuBvhNode is 48 bytes");
static_assert(sizeof(tc_gpu_primitive_ref) == 8, "GpuPrimitiveRef is 8 bytes");

namespace {

// Default dynamic-fetch threshold of the path kernel (tc_render_options.refill_lanes).
constexpr int kDefaultRefillLanes = 1;
// Plain wavefront schedule: default path slots, and the smallest frame (in paths) that the
// automatic schedule gives it (smaller frames run in less time than its per-bounce launches cost).
constexpr uint32_t kWavefrontSlots = 1u << 23;
constexpr uint64_t kWavefrontMinPaths = 1ull << 20;
// Iterations the host runs ahead of the live-slot count it waits for (kWfRing = kWfLag + 1).
constexpr int kWfLag = 4;
constexpr int kWfRing = kWfLag + 1;
// Scenes with at least this many primitives build their hierarchy on the device by default.
constexpr size_t kDeviceBuildMin = 4096;
// Guide training samples the pool keeps across recording batches (48 bytes each: 768 MiB).
constexpr uint32_t kGuidePoolSamples = 1u << 24;

thread_local std::string g_thread_error;

struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
  }
  // Grows to at least `n` bytes (contents are not preserved).
  cudaError_t reserve(size_t n) {
    if (n <= bytes && ptr) return cudaSuccess;
    release();
    if (n == 0) return cudaSuccess;
    cudaError_t e = cudaMalloc(&ptr, n);
    if (e == cudaSuccess) bytes = n;
    else ptr = nullptr;
    return e;
  }
  template <class T>
  T* as() const { return static_cast<T*>(ptr); }
};

}  // namespace

struct tc_context {
  int device = 0;
  int sm_count = 0;
  cudaStream_t stream = nullptr;        // stream used by every call
  cudaStream_t own_stream = nullptr;    // the context's own stream
  cudaEvent_t ev_begin = nullptr, ev_kernel0 = nullptr, ev_kernel1 = nullptr, ev_end = nullptr;
  std::string error;

  // Scene
  bool has_scene = false;
  tcb::DevScene scene{};
  DevBuf pairs, prims, materials, lights, attributes, texels;
  DevBuf env_rgb, env_marginal, env_conditional, env_pdf, env_row_sums, env_total;
  DevBuf env_alias_cond, env_alias_marg, env_alias_q, env_alias_idx;  // alias tables and their build scratch
  uint32_t sphere_count = 0, triangle_count = 0, material_count = 0, light_count = 0, bvh_prims = 0;
  uint32_t bvh_depth = 0;
  size_t pair_count = 0;
  bool any_attr = false;
  // Geometry refit (tc_update_geometry): the root record, the scene-order geometry the prim
  // records are rewritten from, and pair-node indices grouped by depth.
  DevBuf root_buf, raw_spheres, raw_triangles, refit_nodes;
  std::vector<uint32_t> refit_levels;
  bool raw_spheres_valid = false, raw_triangles_valid = false;
  // Display conversion output (packed RGBA8) and the job table of batched launches.
  DevBuf display, batch_jobs;
  // Device hierarchy build (tc_set_hierarchy_build): mode, builder, triangle attribute flags and
  // its status word.
  int build_mode = 0;
  bool device_built = false;
  tcb::DeviceBvhBuilder builder;
  DevBuf attr_flags, build_status;
  // JPEG frames (tc_encode_jpeg): encoder created on first use, RGB8 input on the device.
  nvjpegHandle_t jpeg = nullptr;
  nvjpegEncoderState_t jpeg_state = nullptr;
  nvjpegEncoderParams_t jpeg_params = nullptr;
  DevBuf jpeg_rgb;

  // Accumulation state (progressive contract of path_tracer.rs:900-923)
  uint32_t width = 0, height = 0, accumulated = 0;
  bool has_moments = false;
  DevBuf accum, accum_sq, image, work_counter, counters;

  // Parity scratch
  DevBuf ray_buf, prim_buf, t_buf;

  // Path guiding
  bool has_guide = false;
  tcb::GuideDevice guide;
  DevBuf g_params, g_m, g_v, g_grad, g_images, g_biases, g_status, g_in, g_out;
  // Guided wavefront buffers (two state buffers, queries, decoded mixtures, round counters).
  DevBuf w_state_a, w_state_b, w_query, w_mix, w_counts, w_prefix;
  // Recorded training data: the records of the last recording batch, and the sample pool every
  // recording batch appends its positive-weight samples to (guide_record = 1 starts a new pool):
  // rec_samples holds kGuidePoolSamples samples, rec_wsum their (count, weight sum).
  DevBuf rec_records, rec_count, rec_path_rad, rec_samples, rec_wsum, wf_rec_ref;
  uint32_t rec_capacity = 0;
  bool has_records = false;

  tc_stats stats{};

  // tc_render_no_alloc: device address of the library's static scratch array in this context's
  // CUDA context, looked up by the first such call on the context.
  unsigned long long* static_scratch = nullptr;

  // Plain wavefront schedule: per-path state and queues for wf_capacity slots, and a pinned
  // ring of live-slot counts with one event per entry (the host's drain check).
  uint32_t wf_capacity = 0;
  DevBuf wf_state, wf_ray_o, wf_ray_d, wf_thr, wf_rad, wf_rng, wf_hit, wf_nee, wf_shadow_q, wf_ext_q, wf_mat_q, wf_q;
  DevBuf wf_ext_key, wf_shadow_key, wf_sort_counts, wf_sorted;
  uint32_t* wf_live_host = nullptr;
  unsigned long long* wf_work_host = nullptr;  // the work counter, read back beside each live count
  cudaEvent_t wf_events[kWfRing] = {};
  // Phase timing (tc_render_options.phase_timing): kWfMarks events per iteration of the last
  // wavefront render, wf_marks_used iterations of them recorded.
  std::vector<std::array<cudaEvent_t, tcb::kWfMarks>> wf_marks;
  uint32_t wf_marks_used = 0;
  bool wf_marks_guided = false;

  // Triangle test of the next upload (tc_set_triangle_test) and, for the watertight test, the
  // vertex records of the uploaded scene in leaf order.
  int triangle_test = TC_TRIANGLE_MOLLER_TRUMBORE;
  DevBuf tri_verts;
};

namespace {

int fail(tc_context* ctx, int code, const std::string& msg) {
  if (ctx) ctx->error = msg;
  g_thread_error = msg;
  return code;
}

int cuda_fail(tc_context* ctx, cudaError_t e, const char* what) {
  return fail(ctx, TC_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define TC_CUDA(ctx, call)                                     \
  do {                                                         \
    cudaError_t _e = (call);                                   \
    if (_e != cudaSuccess) return cuda_fail((ctx), _e, #call); \
  } while (0)

template <class T>
cudaError_t upload(DevBuf& buf, const T* src, size_t count, cudaStream_t stream) {
  const size_t bytes = sizeof(T) * count;
  if (bytes == 0) return cudaSuccess;
  cudaError_t e = buf.reserve(bytes);
  if (e != cudaSuccess) return e;
  return cudaMemcpyAsync(buf.ptr, src, bytes, cudaMemcpyHostToDevice, stream);
}

// Walker alias table (Vose's construction) over light weights, built in double precision.
void build_alias(const std::vector<double>& w, std::vector<float>& prob, std::vector<uint32_t>& alias) {
  const size_t n = w.size();
  prob.assign(n, 1.0f);
  alias.resize(n);
  for (size_t i = 0; i < n; ++i) alias[i] = uint32_t(i);
  double total = 0.0;
  for (double x : w) total += x;
  if (n == 0 || !(total > 0.0)) return;
  std::vector<double> q(n);
  std::vector<uint32_t> small, large;
  for (size_t i = 0; i < n; ++i) {
    q[i] = w[i] * double(n) / total;
    (q[i] < 1.0 ? small : large).push_back(uint32_t(i));
  }
  while (!small.empty() && !large.empty()) {
    const uint32_t s = small.back(), l = large.back();
    small.pop_back();
    prob[s] = float(q[s]);
    alias[s] = l;
    q[l] = (q[l] + q[s]) - 1.0;
    if (q[l] < 1.0) {
      large.pop_back();
      small.push_back(l);
    }
  }
  for (uint32_t i : large) prob[i] = 1.0f;
  for (uint32_t i : small) prob[i] = 1.0f;
}

bool finite3(const float* v) { return std::isfinite(v[0]) && std::isfinite(v[1]) && std::isfinite(v[2]); }

// Per-primitive checks shared by uploads and geometry updates (scene_upload.rs:84-98 plus
// finiteness, which the device layout needs).
int validate_geometry(tc_context* ctx, const tc_scene_data* sd, uint32_t n_mat) {
  for (size_t i = 0; i < sd->sphere_count; ++i) {
    const tc_gpu_sphere& s = sd->spheres[i];
    if (s.material_index >= n_mat) return fail(ctx, TC_ERR_INVALID, "sphere " + std::to_string(i) + " references an unknown material");
    if (!std::isfinite(s.center_radius[3]) || !(s.center_radius[3] > 0.0f) || !finite3(s.center_radius))
      return fail(ctx, TC_ERR_INVALID, "sphere " + std::to_string(i) + " must have a finite center and positive radius");
  }
  for (size_t i = 0; i < sd->triangle_count; ++i) {
    const tc_gpu_triangle& t = sd->triangles[i];
    if (t.material_index >= n_mat) return fail(ctx, TC_ERR_INVALID, "triangle " + std::to_string(i) + " references an unknown material");
    if (!finite3(t.v0) || !finite3(t.v1) || !finite3(t.v2))
      return fail(ctx, TC_ERR_INVALID, "triangle " + std::to_string(i) + " vertices must be finite");
  }
  return TC_OK;
}

// Device light records with a Walker alias table over the GpuLight weights (the light
// distribution of light.rs:57-113). Validates kinds, areas and material references.
int pack_lights(tc_context* ctx, const tc_scene_data* sd, uint32_t n_mat, std::vector<tcb::DevLight>& lights) {
  lights.assign(sd->light_count, tcb::DevLight{});
  if (sd->light_count) {
    if (!sd->lights) return fail(ctx, TC_ERR_INVALID, "light pointer is null for a nonzero count");
    std::vector<double> w(sd->light_count);
    double total = 0.0;
    for (size_t i = 0; i < sd->light_count; ++i) {
      w[i] = std::max(0.0, double(sd->lights[i].area_weight_cumulative[1]));
      total += w[i];
    }
    if (!(total > 0.0)) return fail(ctx, TC_ERR_INVALID, "lights have no positive weight");
    std::vector<float> prob;
    std::vector<uint32_t> alias;
    build_alias(w, prob, alias);
    for (size_t i = 0; i < sd->light_count; ++i) {
      const tc_gpu_light& l = sd->lights[i];
      if (l.material_index >= n_mat) return fail(ctx, TC_ERR_INVALID, "light " + std::to_string(i) + " references an unknown material");
      const tc_gpu_material& m = sd->materials[l.material_index];
      tcb::DevLight d{};
      d.kind = l.kind;
      const float area = l.area_weight_cumulative[0];
      if (!(area > 0.0f)) return fail(ctx, TC_ERR_INVALID, "light " + std::to_string(i) + " has no area");
      d.pdf_area = float((w[i] / total) / double(area));
      for (int c = 0; c < 3; ++c) d.emission[c] = m.albedo[c] * m.params[2];
      if (l.kind == 0) {
        float e1[3], e2[3];
        for (int c = 0; c < 3; ++c) {
          d.p0[c] = l.v0[c];
          e1[c] = l.v1[c] - l.v0[c];
          e2[c] = l.v2[c] - l.v0[c];
          d.e1[c] = e1[c];
          d.e2[c] = e2[c];
        }
        const float nx = e1[1] * e2[2] - e2[1] * e1[2], ny = e1[2] * e2[0] - e2[2] * e1[0],
                    nz = e1[0] * e2[1] - e2[0] * e1[1];
        const float inv = 1.0f / std::sqrt(nx * nx + ny * ny + nz * nz);
        d.normal[0] = nx * inv;
        d.normal[1] = ny * inv;
        d.normal[2] = nz * inv;
      } else if (l.kind == 1) {
        for (int c = 0; c < 3; ++c) d.p0[c] = l.center_radius[c];
        d.radius = l.center_radius[3];
      } else {
        return fail(ctx, TC_ERR_INVALID, "light " + std::to_string(i) + " kind must be 0 (triangle) or 1 (sphere)");
      }
      d.alias_prob = prob[i];
      d.alias = alias[i];
      lights[i] = d;
    }
  }
  return TC_OK;
}

// Progressive contract of path_tracer.rs:900-923: accumulated_samples == 0 starts a new image
// (buffers sized and cleared on `st`), otherwise it must equal the samples already held.
int prepare_accumulation(tc_context* ctx, const tc_gpu_render_params* p, bool moments, cudaStream_t st) {
  const uint32_t npix = p->width * p->height;
  if (p->accumulated_samples == 0) {
    if (ctx->width != p->width || ctx->height != p->height || !ctx->accum.ptr) {
      TC_CUDA(ctx, ctx->accum.reserve(sizeof(double) * 3 * npix));
      TC_CUDA(ctx, ctx->image.reserve(sizeof(float4) * npix));
    }
    if (moments) TC_CUDA(ctx, ctx->accum_sq.reserve(sizeof(double) * 3 * npix));
    TC_CUDA(ctx, cudaMemsetAsync(ctx->accum.ptr, 0, sizeof(double) * 3 * npix, st));
    if (moments) TC_CUDA(ctx, cudaMemsetAsync(ctx->accum_sq.ptr, 0, sizeof(double) * 3 * npix, st));
    ctx->width = p->width;
    ctx->height = p->height;
    ctx->accumulated = 0;
    ctx->has_moments = moments;
  } else {
    if (p->width != ctx->width || p->height != ctx->height)
      return fail(ctx, TC_ERR_STATE, "progressive batch changes the image size");
    if (p->accumulated_samples != ctx->accumulated)
      return fail(ctx, TC_ERR_STATE, "accumulated_samples " + std::to_string(p->accumulated_samples) +
                                          " does not match the " + std::to_string(ctx->accumulated) +
                                          " samples held by the context");
    if (moments && !ctx->has_moments)
      return fail(ctx, TC_ERR_STATE, "keep_moments must be set from the first batch of an accumulation");
  }
  if (uint64_t(ctx->accumulated) + p->samples > 0xFFFFFFFFull)
    return fail(ctx, TC_ERR_INVALID, "progressive accumulated sample count overflowed");
  return TC_OK;
}

// Checks shared by every render entry point.
int check_render_params(tc_context* ctx, const tc_gpu_render_params* p) {
  if (!p) return fail(ctx, TC_ERR_INVALID, "render params are null");
  if (!ctx->has_scene) return fail(ctx, TC_ERR_STATE, "render before tc_upload_scene");
  if (p->width == 0 || p->height == 0) return fail(ctx, TC_ERR_INVALID, "render dimensions must be nonzero");
  if (p->samples == 0) return fail(ctx, TC_ERR_INVALID, "sample batch must be greater than zero");
  if (uint64_t(p->width) * p->height > (1ull << 31)) return fail(ctx, TC_ERR_INVALID, "image is too large");
  return TC_OK;
}

// Device hierarchy of a scene: the caller's flat BVH in the reference layout (when given and
// use_given is set) or a fresh median-split build (crates/toaster-bvh/src/bvh.rs:92-154).
int build_hierarchy(tc_context* ctx, const tc_scene_data* sd, bool use_given, tcb::DeviceHierarchy& dh) {
  std::vector<tcb::SphereIn> sph(sd->sphere_count);
  std::vector<uint32_t> sph_mat(sd->sphere_count);
  for (size_t i = 0; i < sd->sphere_count; ++i) {
    const tc_gpu_sphere& s = sd->spheres[i];
    sph[i] = tcb::SphereIn{{s.center_radius[0], s.center_radius[1], s.center_radius[2]}, s.center_radius[3]};
    sph_mat[i] = s.material_index;
  }
  std::vector<tcb::TriangleIn> tri(sd->triangle_count);
  std::vector<uint32_t> tri_mat(sd->triangle_count), tri_flags(sd->triangle_count, 0u);
  for (size_t i = 0; i < sd->triangle_count; ++i) {
    const tc_gpu_triangle& t = sd->triangles[i];
    for (int c = 0; c < 3; ++c) {
      tri[i].v[0][c] = t.v0[c];
      tri[i].v[1][c] = t.v1[c];
      tri[i].v[2][c] = t.v2[c];
    }
    tri_mat[i] = t.material_index;
    if (sd->triangle_attributes) tri_flags[i] = sd->triangle_attributes[i].flags & 3u;
  }
  tcb::FlatHierarchy flat;
  if (use_given && sd->bvh_nodes && sd->bvh_node_count) {
    if (!sd->bvh_primitives || sd->bvh_primitive_count != sd->sphere_count + sd->triangle_count)
      return fail(ctx, TC_ERR_INVALID, "BVH primitive references must cover every sphere and triangle");
    flat.nodes.resize(sd->bvh_node_count);
    for (size_t i = 0; i < sd->bvh_node_count; ++i) {
      const tc_gpu_bvh_node& n = sd->bvh_nodes[i];
      tcb::FlatNode& f = flat.nodes[i];
      for (int c = 0; c < 3; ++c) {
        f.min[c] = n.min[c];
        f.max[c] = n.max[c];
      }
      f.first_or_right = n.first_or_right;
      f.count = n.primitive_count;
    }
    flat.prims.resize(sd->bvh_primitive_count);
    for (size_t i = 0; i < sd->bvh_primitive_count; ++i)
      flat.prims[i] = tcb::PrimRef{sd->bvh_primitives[i].kind, sd->bvh_primitives[i].index};
  } else {
    flat = tcb::build_median_split(sph.data(), sph.size(), tri.data(), tri.size());
  }
  std::string err;
  if (!tcb::to_device_layout(flat, sph.data(), sph_mat.data(), sph.size(), tri.data(), tri_mat.data(),
                             tri_flags.data(), tri.size(), dh, err))
    return fail(ctx, TC_ERR_INVALID, err);
  return TC_OK;
}

}  // namespace

extern "C" {

int tc_abi_version(void) { return TC_ABI_VERSION; }

const char* tc_last_error(const tc_context* ctx) {
  if (ctx) return ctx->error.c_str();
  return g_thread_error.c_str();
}

int tc_record_sizes(uint32_t* out, size_t n) {
  const uint32_t sizes[9] = {uint32_t(sizeof(tc_gpu_render_params)), uint32_t(sizeof(tc_gpu_camera)),
                             uint32_t(sizeof(tc_gpu_sphere)),         uint32_t(sizeof(tc_gpu_triangle)),
                             uint32_t(sizeof(tc_gpu_triangle_attributes)), uint32_t(sizeof(tc_gpu_material)),
                             uint32_t(sizeof(tc_gpu_light)),          uint32_t(sizeof(tc_gpu_bvh_node)),
                             uint32_t(sizeof(tc_gpu_primitive_ref))};
  if (!out || n < 9) return fail(nullptr, TC_ERR_INVALID, "tc_record_sizes needs room for 9 values");
  std::memcpy(out, sizes, sizeof(sizes));
  return TC_OK;
}

int tc_create(int device_ordinal, tc_context** out_ctx) {
  if (!out_ctx) return fail(nullptr, TC_ERR_INVALID, "out_ctx is null");
  *out_ctx = nullptr;
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0)
    return fail(nullptr, TC_ERR_NO_DEVICE, std::string("no CUDA device: ") + cudaGetErrorString(e));
  if (device_ordinal < 0 || device_ordinal >= count)
    return fail(nullptr, TC_ERR_NO_DEVICE, "device ordinal " + std::to_string(device_ordinal) + " out of range");
  cudaDeviceProp prop;
  e = cudaGetDeviceProperties(&prop, device_ordinal);
  if (e != cudaSuccess) return fail(nullptr, TC_ERR_NO_DEVICE, cudaGetErrorString(e));
  if (prop.major != 10)
    return fail(nullptr, TC_ERR_NO_DEVICE,
                std::string("device ") + prop.name + " is not sm_100 (compute capability " +
                    std::to_string(prop.major) + "." + std::to_string(prop.minor) + ")");
  e = cudaSetDevice(device_ordinal);
  if (e != cudaSuccess) return fail(nullptr, TC_ERR_CUDA, cudaGetErrorString(e));
  auto* ctx = new tc_context();
  ctx->device = device_ordinal;
  ctx->sm_count = prop.multiProcessorCount;
  if ((e = cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaEventCreate(&ctx->ev_begin)) != cudaSuccess || (e = cudaEventCreate(&ctx->ev_kernel0)) != cudaSuccess ||
      (e = cudaEventCreate(&ctx->ev_kernel1)) != cudaSuccess || (e = cudaEventCreate(&ctx->ev_end)) != cudaSuccess) {
    std::string msg = std::string("context setup failed: ") + cudaGetErrorString(e);
    tc_destroy(ctx);
    return fail(nullptr, TC_ERR_CUDA, msg);
  }
  ctx->stream = ctx->own_stream;
  if ((e = ctx->work_counter.reserve(sizeof(unsigned long long))) != cudaSuccess ||
      (e = ctx->counters.reserve(4 * sizeof(unsigned long long))) != cudaSuccess) {
    std::string msg = std::string("context allocation failed: ") + cudaGetErrorString(e);
    tc_destroy(ctx);
    return fail(nullptr, TC_ERR_CUDA, msg);
  }
  *out_ctx = ctx;
  return TC_OK;
}

int tc_destroy(tc_context* ctx) {
  if (!ctx) return TC_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->own_stream && ctx->own_stream != ctx->stream) cudaStreamSynchronize(ctx->own_stream);
  if (ctx->ev_begin) cudaEventDestroy(ctx->ev_begin);
  if (ctx->ev_kernel0) cudaEventDestroy(ctx->ev_kernel0);
  if (ctx->ev_kernel1) cudaEventDestroy(ctx->ev_kernel1);
  if (ctx->ev_end) cudaEventDestroy(ctx->ev_end);
  for (cudaEvent_t e : ctx->wf_events)
    if (e) cudaEventDestroy(e);
  for (auto& m : ctx->wf_marks)
    for (cudaEvent_t e : m) cudaEventDestroy(e);
  if (ctx->wf_live_host) cudaFreeHost(ctx->wf_live_host);
  if (ctx->wf_work_host) cudaFreeHost(ctx->wf_work_host);
  if (ctx->jpeg_params) nvjpegEncoderParamsDestroy(ctx->jpeg_params);
  if (ctx->jpeg_state) nvjpegEncoderStateDestroy(ctx->jpeg_state);
  if (ctx->jpeg) nvjpegDestroy(ctx->jpeg);
  if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
  delete ctx;
  return TC_OK;
}

int tc_set_stream(tc_context* ctx, void* stream) {
  if (!ctx) return fail(nullptr, TC_ERR_INVALID, "context is null");
  TC_CUDA(ctx, cudaSetDevice(ctx->device));
  TC_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  ctx->stream = stream ? static_cast<cudaStream_t>(stream) : ctx->own_stream;
  return TC_OK;
}

int tc_upload_scene(tc_context* ctx, const tc_scene_data* sd) {
  if (!ctx) return fail(nullptr, TC_ERR_INVALID, "context is null");
  if (!sd) return fail(ctx, TC_ERR_INVALID, "scene is null");
  TC_CUDA(ctx, cudaSetDevice(ctx->device));
  // Validation mirrors scene_to_gpu_inner (crates/toaster-gpu/src/scene_upload.rs:84-98).
  if (sd->sphere_count == 0 && sd->triangle_count == 0)
    return fail(ctx, TC_ERR_INVALID, "GPU renderer requires at least one object");
  if (sd->material_count == 0 || !sd->materials)
    return fail(ctx, TC_ERR_INVALID, "GPU renderer requires at least one material");
  if ((sd->sphere_count && !sd->spheres) || (sd->triangle_count && !sd->triangles))
    return fail(ctx, TC_ERR_INVALID, "geometry pointer is null for a nonzero count");
  if (sd->triangle_attributes && sd->triangle_attribute_count != sd->triangle_count)
    return fail(ctx, TC_ERR_INVALID, "triangle attribute count must match triangle count");
  if (sd->sphere_count + sd->triangle_count > tcb::kMaxPrimitives)
    return fail(ctx, TC_ERR_INVALID, "too many primitives for GPU");
  const uint32_t n_mat = uint32_t(sd->material_count);
  if (int rc = validate_geometry(ctx, sd, n_mat)) return rc;
  const uint32_t bg = sd->params.background_kind;
  if (bg > 2u) return fail(ctx, TC_ERR_INVALID, "background kind must be 0 (sky), 1 (black) or 2 (environment)");
  const uint32_t ew = sd->params.environment_width, eh = sd->params.environment_height;
  const bool has_env = ew > 0 && eh > 0;
  if (bg == 2u && (!has_env || !sd->environment_pixels))
    return fail(ctx, TC_ERR_INVALID, "environment background requires an environment map");
  if (has_env && sd->environment_pixels && sd->environment_pixel_count != size_t(ew) * eh)
    return fail(ctx, TC_ERR_INVALID, "environment contains " + std::to_string(sd->environment_pixel_count) +
                                         " pixels but " + std::to_string(size_t(ew) * eh) + " were expected");

  // Materials.
  std::vector<tcb::DevMaterial> mats(n_mat);
  for (uint32_t i = 0; i < n_mat; ++i) {
    const tc_gpu_material& m = sd->materials[i];
    if (m.kind > 3u) return fail(ctx, TC_ERR_INVALID, "material " + std::to_string(i) + " has an unknown kind");
    if (m.texture_width && m.texture_height &&
        (!sd->texture_pixels || size_t(m.texture_offset) + size_t(m.texture_width) * m.texture_height > sd->texture_pixel_count))
      return fail(ctx, TC_ERR_INVALID, "material " + std::to_string(i) + " texture lies outside the texture atlas");
    tcb::DevMaterial d{};
    d.kind = m.kind;
    for (int c = 0; c < 3; ++c) {
      d.albedo[c] = m.albedo[c];
      d.emission[c] = m.kind == tcb::kEmissive ? m.albedo[c] * m.params[2] : 0.0f;
    }
    d.roughness = std::min(std::max(m.params[0], 0.0f), 1.0f);
    d.ior = m.params[1];
    if (m.kind == tcb::kDielectric && !(d.ior > 0.0f))
      return fail(ctx, TC_ERR_INVALID, "material " + std::to_string(i) + ": dielectric ior must be positive");
    d.tex_offset = m.texture_offset;
    d.tex_width = m.texture_width;
    d.tex_height = m.texture_height;
    mats[i] = d;
  }

  // Lights: alias table over the GpuLight weights (light.rs:57-113 distribution).
  std::vector<tcb::DevLight> lights;
  if (int rc = pack_lights(ctx, sd, n_mat, lights)) return rc;

  cudaStream_t st = ctx->stream;
  bool any_attr = false;
  if (sd->triangle_attributes)
    for (size_t i = 0; i < sd->triangle_count; ++i) any_attr |= (sd->triangle_attributes[i].flags & 3u) != 0u;

  // Hierarchy: the caller's (reference layout), or the median-split build, on the device
  // (tc_set_hierarchy_build) or on the host. A device build that meets a degenerate node falls
  // back to the host build, which makes such nodes leaves.
  const size_t n_prims = sd->sphere_count + sd->triangle_count;
  const bool given = sd->bvh_nodes && sd->bvh_node_count;
  const bool on_device = !given && (ctx->build_mode == 2 || (ctx->build_mode == 0 && n_prims >= kDeviceBuildMin));
  bool built = false;
  uint32_t pair_count = 0, prim_count = 0, depth = 0;
  if (on_device) {
    TC_CUDA(ctx, ctx->builder.plan(uint32_t(sd->sphere_count), uint32_t(sd->triangle_count)));
    TC_CUDA(ctx, upload(ctx->raw_spheres, sd->spheres, sd->sphere_count, st));
    TC_CUDA(ctx, upload(ctx->raw_triangles, sd->triangles, sd->triangle_count, st));
    const uint32_t* flags = nullptr;
    if (any_attr) {
      std::vector<uint32_t> f(sd->triangle_count);
      for (size_t i = 0; i < f.size(); ++i) f[i] = sd->triangle_attributes[i].flags & 3u;
      TC_CUDA(ctx, upload(ctx->attr_flags, f.data(), f.size(), st));
      TC_CUDA(ctx, cudaStreamSynchronize(st));
      flags = ctx->attr_flags.as<uint32_t>();
    }
    TC_CUDA(ctx, ctx->pairs.reserve(sizeof(tcb::PairNode) * std::max<size_t>(ctx->builder.pair_count(), 1)));
    TC_CUDA(ctx, ctx->prims.reserve(sizeof(tcb::PrimRecord) * n_prims));
    TC_CUDA(ctx, ctx->root_buf.reserve(sizeof(tcb::ChildRec)));
    TC_CUDA(ctx, ctx->build_status.reserve(sizeof(uint32_t)));
    TC_CUDA(ctx, cudaMemsetAsync(ctx->build_status.ptr, 0, sizeof(uint32_t), st));
    TC_CUDA(ctx, ctx->builder.build(ctx->raw_spheres.as<tc_gpu_sphere>(), ctx->raw_triangles.as<tc_gpu_triangle>(),
                                    flags, ctx->pairs.as<tcb::PairNode>(), ctx->root_buf.as<tcb::ChildRec>(),
                                    ctx->prims.as<tcb::PrimRecord>(), ctx->build_status.as<uint32_t>(), st));
    uint32_t degenerate = 0;
    TC_CUDA(ctx, cudaMemcpyAsync(&degenerate, ctx->build_status.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    TC_CUDA(ctx, cudaStreamSynchronize(st));
    if (!degenerate) {
      built = true;
      pair_count = ctx->builder.pair_count();
      prim_count = uint32_t(n_prims);
      depth = ctx->builder.depth();
      const size_t refit_count = ctx->builder.refit_levels().back();
      TC_CUDA(ctx, ctx->refit_nodes.reserve(sizeof(uint32_t) * std::max<size_t>(refit_count, 1)));
      if (refit_count)
        TC_CUDA(ctx, cudaMemcpyAsync(ctx->refit_nodes.ptr, ctx->builder.refit_nodes(), sizeof(uint32_t) * refit_count,
                                     cudaMemcpyDeviceToDevice, st));
      ctx->refit_levels = ctx->builder.refit_levels();
    }
  }
  if (!built) {
    tcb::DeviceHierarchy dh;
    if (int rc = build_hierarchy(ctx, sd, true, dh)) return rc;
    TC_CUDA(ctx, upload(ctx->pairs, dh.pairs.data(), dh.pairs.size(), st));
    TC_CUDA(ctx, upload(ctx->prims, dh.prims.data(), dh.prims.size(), st));
    TC_CUDA(ctx, upload(ctx->root_buf, &dh.root, 1, st));
    // Pair nodes grouped by depth, root first, for the bottom-up refit.
    std::vector<uint32_t> order, offsets{0u};
    if (!(dh.root.link & tcb::kLeafBit)) {
      order.push_back(dh.root.link);
      size_t begin = 0;
      while (begin < order.size()) {
        const size_t end = order.size();
        offsets.push_back(uint32_t(end));
        for (size_t i = begin; i < end; ++i)
          for (const tcb::ChildRec& c : dh.pairs[order[i]].child)
            if (!(c.link & tcb::kLeafBit)) order.push_back(c.link);
        begin = end;
      }
    }
    TC_CUDA(ctx, upload(ctx->refit_nodes, order.data(), order.size(), st));
    ctx->refit_levels = std::move(offsets);
    pair_count = uint32_t(dh.pairs.size());
    prim_count = uint32_t(dh.prims.size());
    depth = dh.depth;
  }
  TC_CUDA(ctx, upload(ctx->materials, mats.data(), mats.size(), st));
  TC_CUDA(ctx, upload(ctx->lights, lights.data(), lights.size(), st));
  if (any_attr) TC_CUDA(ctx, upload(ctx->attributes, sd->triangle_attributes, sd->triangle_count, st));
  if (sd->texture_pixels && sd->texture_pixel_count)
    TC_CUDA(ctx, upload(ctx->texels, sd->texture_pixels, sd->texture_pixel_count, st));

  tcb::DevScene& s = ctx->scene;
  s = tcb::DevScene{};
  s.pairs = ctx->pairs.as<tcb::PairNode>();
  s.prims = ctx->prims.as<tcb::PrimRecord>();
  s.root = ctx->root_buf.as<tcb::ChildRec>();
  s.materials = ctx->materials.as<tcb::DevMaterial>();
  s.material_count = n_mat;
  s.lights = sd->light_count ? ctx->lights.as<tcb::DevLight>() : nullptr;
  s.light_count = uint32_t(sd->light_count);
  s.attributes = any_attr ? ctx->attributes.as<float4>() : nullptr;
  s.texels = (sd->texture_pixels && sd->texture_pixel_count) ? ctx->texels.as<uint32_t>() : nullptr;
  s.background = bg;
  if (has_env && sd->environment_pixels) {
    const size_t n = size_t(ew) * eh;
    TC_CUDA(ctx, upload(ctx->env_rgb, reinterpret_cast<const float4*>(sd->environment_pixels), n, st));
    TC_CUDA(ctx, ctx->env_marginal.reserve(sizeof(float) * eh));
    TC_CUDA(ctx, ctx->env_conditional.reserve(sizeof(float) * n));
    TC_CUDA(ctx, ctx->env_pdf.reserve(sizeof(float) * n));
    TC_CUDA(ctx, ctx->env_row_sums.reserve(sizeof(double) * eh));
    TC_CUDA(ctx, ctx->env_total.reserve(sizeof(double)));
    const size_t span = std::max<size_t>(ew, eh);
    TC_CUDA(ctx, ctx->env_alias_cond.reserve(sizeof(uint2) * n));
    TC_CUDA(ctx, ctx->env_alias_marg.reserve(sizeof(uint2) * eh));
    if (!tcb::env_alias_in_shared(ew, eh)) {
      TC_CUDA(ctx, ctx->env_alias_q.reserve(sizeof(double) * span * (size_t(eh) + 1)));
      TC_CUDA(ctx, ctx->env_alias_idx.reserve(2 * sizeof(uint32_t) * span * (size_t(eh) + 1)));
    }
    TC_CUDA(ctx, tcb::launch_env_tables(ctx->env_rgb.as<float4>(), ew, eh, sd->params.environment_intensity,
                                        ctx->env_marginal.as<float>(), ctx->env_conditional.as<float>(),
                                        ctx->env_pdf.as<float>(), ctx->env_row_sums.as<double>(),
                                        ctx->env_total.as<double>(), ctx->env_alias_q.as<double>(),
                                        ctx->env_alias_idx.as<uint32_t>(), ctx->env_alias_cond.as<uint2>(),
                                        ctx->env_alias_marg.as<uint2>(), st));
    double total = 0.0;
    TC_CUDA(ctx, cudaMemcpyAsync(&total, ctx->env_total.ptr, sizeof(double), cudaMemcpyDeviceToHost, st));
    TC_CUDA(ctx, cudaStreamSynchronize(st));
    s.env_rgb = ctx->env_rgb.as<float4>();
    s.env_alias_marg = ctx->env_alias_marg.as<uint2>();
    s.env_alias_cond = ctx->env_alias_cond.as<uint2>();
    s.env_pdf = ctx->env_pdf.as<float>();
    s.env_width = ew;
    s.env_height = eh;
    s.env_intensity = sd->params.environment_intensity;
    float rot = std::fmod(sd->params.environment_rotation_degrees, 360.0f);
    if (rot < 0.0f) rot += 360.0f;
    s.env_rotation_turns = rot / 360.0f;
    s.env_sampleable = (total > 0.0 && std::isfinite(total)) ? 1u : 0u;
  }
  for (int c = 0; c < 3; ++c) {
    s.cam_origin[c] = sd->camera.origin[c];
    s.cam_lower_left[c] = sd->camera.lower_left_corner[c];
    s.cam_horizontal[c] = sd->camera.horizontal[c];
    s.cam_vertical[c] = sd->camera.vertical[c];
  }
  const bool raw_tris_on_device = built && on_device;
  if (ctx->triangle_test == TC_TRIANGLE_WATERTIGHT && sd->triangle_count) {
    // Vertex records for the watertight test, gathered in leaf order from the scene's triangles.
    if (!raw_tris_on_device) TC_CUDA(ctx, upload(ctx->raw_triangles, sd->triangles, sd->triangle_count, st));
    TC_CUDA(ctx, ctx->tri_verts.reserve(3 * sizeof(float4) * size_t(prim_count)));
    TC_CUDA(ctx, tcb::launch_triangle_vertices(ctx->prims.as<tcb::PrimRecord>(), prim_count, ctx->raw_triangles.ptr,
                                               ctx->tri_verts.as<float4>(), st));
    s.tri_verts = ctx->tri_verts.as<float4>();
  }
  TC_CUDA(ctx, cudaStreamSynchronize(st));
  ctx->has_scene = true;
  ctx->sphere_count = uint32_t(sd->sphere_count);
  ctx->triangle_count = uint32_t(sd->triangle_count);
  ctx->material_count = n_mat;
  ctx->light_count = uint32_t(sd->light_count);
  ctx->bvh_prims = prim_count;
  ctx->bvh_depth = depth;
  ctx->stats.bvh_depth = depth;
  ctx->any_attr = any_attr;
  ctx->pair_count = pair_count;
  ctx->device_built = built && on_device;
  ctx->raw_spheres_valid = ctx->device_built;
  ctx->raw_triangles_valid = ctx->device_built || ctx->scene.tri_verts != nullptr;
  return TC_OK;
}

int tc_set_triangle_test(tc_context* ctx, int test) {
  if (!ctx) return fail(nullptr, TC_ERR_INVALID, "context is null");
  if (test != TC_TRIANGLE_MOLLER_TRUMBORE && test != TC_TRIANGLE_WATERTIGHT)
    return fail(ctx, TC_ERR_INVALID, "triangle test must be 0 (Moller-Trumbore) or 1 (watertight)");
  ctx->triangle_test = test;
  return TC_OK;
}

int tc_set_hierarchy_build(tc_context* ctx, int mode) {
  if (!ctx) return fail(nullptr, TC_ERR_INVALID, "context is null");
  if (mode < 0 || mode > 2) return fail(ctx, TC_ERR_INVALID, "hierarchy build mode must be 0 (auto), 1 (host) or 2 (device)");
  ctx->build_mode = mode;
  return TC_OK;
}

int tc_update_geometry(tc_context* ctx, const tc_scene_data* sd, const tc_scene_changes* changes) {
  if (!ctx) return fail(nullptr, TC_ERR_INVALID, "context is null");
  if (!sd || !changes) return fail(ctx, TC_ERR_INVALID, "scene or change set is null");
  if (!ctx->has_scene) return fail(ctx, TC_ERR_STATE, "tc_update_geometry before tc_upload_scene");
  // Counts are fixed for a render session (path_tracer.rs:639-653).
  if (sd->sphere_count != ctx->sphere_count || sd->triangle_count != ctx->triangle_count ||
      sd->material_count != ctx->material_count || sd->light_count != ctx->light_count ||
      (sd->triangle_attributes && sd->triangle_attribute_count != sd->triangle_count))
    return fail(ctx, TC_ERR_INVALID,
                "evaluated scenes must preserve GPU geometry, material, light, and BVH primitive counts");
  if (!sd->materials) return fail(ctx, TC_ERR_INVALID, "GPU renderer requires at least one material");
  if ((sd->sphere_count && !sd->spheres) || (sd->triangle_count && !sd->triangles))
    return fail(ctx, TC_ERR_INVALID, "geometry pointer is null for a nonzero count");
  const bool geometry = changes->spheres || changes->triangles;
  if (geometry)
    if (int rc = validate_geometry(ctx, sd, ctx->material_count)) return rc;
  std::vector<tcb::DevLight> lights;
  if (changes->emissive_geometry)
    if (int rc = pack_lights(ctx, sd, ctx->material_count, lights)) return rc;
  TC_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  if (geometry) {
    if (ctx->sphere_count && (changes->spheres || !ctx->raw_spheres_valid)) {
      TC_CUDA(ctx, upload(ctx->raw_spheres, sd->spheres, sd->sphere_count, st));
      ctx->raw_spheres_valid = true;
    }
    if (ctx->triangle_count && (changes->triangles || !ctx->raw_triangles_valid)) {
      TC_CUDA(ctx, upload(ctx->raw_triangles, sd->triangles, sd->triangle_count, st));
      ctx->raw_triangles_valid = true;
    }
    if (changes->triangles && ctx->any_attr && sd->triangle_attributes)
      TC_CUDA(ctx, upload(ctx->attributes, sd->triangle_attributes, sd->triangle_count, st));
    tcb::RefitPlan plan;
    plan.nodes = ctx->refit_nodes.as<uint32_t>();
    plan.level_offsets = ctx->refit_levels;
    TC_CUDA(ctx, tcb::launch_refit(plan, ctx->pairs.as<tcb::PairNode>(), ctx->root_buf.as<tcb::ChildRec>(),
                                   ctx->prims.as<tcb::PrimRecord>(), ctx->bvh_prims,
                                   ctx->raw_spheres.as<tc_gpu_sphere>(), ctx->raw_triangles.as<tc_gpu_triangle>(), st));
    if (ctx->scene.tri_verts && changes->triangles)
      TC_CUDA(ctx, tcb::launch_triangle_vertices(ctx->prims.as<tcb::PrimRecord>(), ctx->bvh_prims,
                                                 ctx->raw_triangles.ptr, ctx->tri_verts.as<float4>(), st));
  }
  if (changes->emissive_geometry && !lights.empty())
    TC_CUDA(ctx, upload(ctx->lights, lights.data(), lights.size(), st));
  if (changes->camera) {
    tcb::DevScene& s = ctx->scene;
    for (int c = 0; c < 3; ++c) {
      s.cam_origin[c] = sd->camera.origin[c];
      s.cam_lower_left[c] = sd->camera.lower_left_corner[c];
      s.cam_horizontal[c] = sd->camera.horizontal[c];
      s.cam_vertical[c] = sd->camera.vertical[c];
    }
  }
  TC_CUDA(ctx, cudaStreamSynchronize(st));
  return TC_OK;
}

int tc_set_camera(tc_context* ctx, const tc_gpu_camera* cam) {
  if (!ctx) return fail(nullptr, TC_ERR_INVALID, "context is null");
  if (!cam) return fail(ctx, TC_ERR_INVALID, "camera is null");
  if (!ctx->has_scene) return fail(ctx, TC_ERR_STATE, "tc_set_camera before tc_upload_scene");
  for (int c = 0; c < 3; ++c) {
    ctx->scene.cam_origin[c] = cam->origin[c];
    ctx->scene.cam_lower_left[c] = cam->lower_left_corner[c];
    ctx->scene.cam_horizontal[c] = cam->horizontal[c];
    ctx->scene.cam_vertical[c] = cam->vertical[c];
  }
  return TC_OK;
}

// A render as a wavefront (tcb::WavefrontLaunch): plain or guided (the diffuse queue inferred
// between logic and shade), recording training records when L.g.records is set. Iterations of
// logic, shade and trace launches until no slot holds a path and no work is left. The host waits, kWfLag iterations
// behind the last one it enqueued, for the live-slot count of an earlier iteration, so the GPU
// always has queued work; the iterations launched after the last path finished find nothing to do.
static int run_wavefront(tc_context* ctx, const tcb::RenderLaunch& L, uint32_t slots, uint32_t max_bounces,
                         int refill_lanes, bool moments, bool guided, bool sort_rays, bool phase_timing,
                         cudaStream_t st) {
  const uint64_t items = L.total_items;
  const uint32_t cap = uint32_t(std::max<uint64_t>(32, std::min<uint64_t>(slots, items)));
  if (cap != ctx->wf_capacity) {
    ctx->wf_capacity = 0;
    const size_t n = cap;
    TC_CUDA(ctx, ctx->wf_state.reserve(sizeof(uint32_t) * n));
    TC_CUDA(ctx, ctx->wf_ray_o.reserve(sizeof(float4) * n));
    TC_CUDA(ctx, ctx->wf_ray_d.reserve(sizeof(float4) * n));
    TC_CUDA(ctx, ctx->wf_thr.reserve(sizeof(float4) * n));
    TC_CUDA(ctx, ctx->wf_rad.reserve(sizeof(float4) * n));
    TC_CUDA(ctx, ctx->wf_rng.reserve(sizeof(uint4) * n));
    TC_CUDA(ctx, ctx->wf_hit.reserve(sizeof(uint4) * n));
    TC_CUDA(ctx, ctx->wf_nee.reserve(2 * sizeof(float4) * n));
    TC_CUDA(ctx, ctx->wf_shadow_q.reserve(4 * sizeof(float4) * n));  // two shadow rays per slot
    TC_CUDA(ctx, ctx->wf_ext_q.reserve(sizeof(uint32_t) * n));
    TC_CUDA(ctx, ctx->wf_mat_q.reserve(3 * sizeof(uint32_t) * n));
    TC_CUDA(ctx, ctx->wf_q.reserve(sizeof(uint32_t) * tcb::kWfCounters));
    ctx->wf_capacity = cap;
  }
  if (!ctx->wf_live_host) {
    TC_CUDA(ctx, cudaHostAlloc(reinterpret_cast<void**>(&ctx->wf_live_host), sizeof(uint32_t) * kWfRing,
                               cudaHostAllocDefault));
    TC_CUDA(ctx, cudaHostAlloc(reinterpret_cast<void**>(&ctx->wf_work_host), sizeof(unsigned long long) * kWfRing,
                               cudaHostAllocDefault));
    for (cudaEvent_t& e : ctx->wf_events) TC_CUDA(ctx, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  tcb::WavefrontLaunch w{};
  w.r = L;
  w.capacity = cap;
  w.state = ctx->wf_state.as<uint32_t>();
  w.ray_o = ctx->wf_ray_o.as<float4>();
  w.ray_d = ctx->wf_ray_d.as<float4>();
  w.thr = ctx->wf_thr.as<float4>();
  w.rad = ctx->wf_rad.as<float4>();
  w.rng = ctx->wf_rng.as<uint4>();
  w.hit = ctx->wf_hit.as<uint4>();
  w.nee = ctx->wf_nee.as<float4>();
  w.shadow_q = ctx->wf_shadow_q.as<float4>();
  w.ext_q = ctx->wf_ext_q.as<uint32_t>();
  w.mat_q = ctx->wf_mat_q.as<uint32_t>();
  w.q = ctx->wf_q.as<uint32_t>();
  w.refill_lanes = refill_lanes;
  w.prim_count = ctx->bvh_prims;
  if (sort_rays) {
    TC_CUDA(ctx, ctx->wf_ext_key.reserve(sizeof(uint32_t) * size_t(cap)));
    TC_CUDA(ctx, ctx->wf_shadow_key.reserve(2 * sizeof(uint32_t) * size_t(cap)));
    TC_CUDA(ctx, ctx->wf_sort_counts.reserve(sizeof(uint32_t) * size_t(tcb::kWfSortBins) * tcb::kWfSortBlocks));
    TC_CUDA(ctx, ctx->wf_sorted.reserve(3 * sizeof(uint32_t) * size_t(cap)));
    w.ext_key = ctx->wf_ext_key.as<uint32_t>();
    w.shadow_key = ctx->wf_shadow_key.as<uint32_t>();
    w.sort_counts = ctx->wf_sort_counts.as<uint32_t>();
    w.sorted = ctx->wf_sorted.as<uint32_t>();
  }
  if (L.g.records) {
    TC_CUDA(ctx, ctx->wf_rec_ref.reserve(sizeof(uint2) * size_t(cap)));
    w.rec_ref = ctx->wf_rec_ref.as<uint2>();
  }
  if (guided) {
    // The diffuse queue's inference queries and decoded mixtures, one entry per slot.
    TC_CUDA(ctx, ctx->w_query.reserve(sizeof(float4) * 2 * size_t(cap)));
    TC_CUDA(ctx, ctx->w_mix.reserve(sizeof(float4) * tcb::kGuideDecodedF4 * size_t(cap)));
    w.query = ctx->w_query.as<float4>();
    w.r.g.in_mix = ctx->w_mix.as<float4>();
  }
  TC_CUDA(ctx, cudaMemsetAsync(w.state, 0, sizeof(uint32_t) * cap, st));
  // Every iteration advances each live path by one vertex and refills every free slot, so the
  // frame drains in at most (waves + 1) x (bounces + 2) iterations; the bound only guards the loop.
  const uint64_t bound = 2 * ((items + cap - 1) / cap + 1) * (uint64_t(max_bounces) + 2) + 2 * kWfRing;
  for (uint64_t it = 0;; ++it) {
    if (it > bound) return fail(ctx, TC_ERR_DEVICE_STATUS, "wavefront render did not drain its paths");
    TC_CUDA(ctx, cudaMemsetAsync(w.q, 0, sizeof(uint32_t) * tcb::kWfCounters, st));
    const cudaEvent_t* marks = nullptr;
    ctx->wf_marks_guided = guided;
    if (phase_timing) {
      if (ctx->wf_marks.size() <= ctx->wf_marks_used) {
        std::array<cudaEvent_t, tcb::kWfMarks> m{};
        for (cudaEvent_t& e : m) TC_CUDA(ctx, cudaEventCreate(&e));
        ctx->wf_marks.push_back(m);
      }
      marks = ctx->wf_marks[ctx->wf_marks_used++].data();
    }
    TC_CUDA(ctx, tcb::launch_wavefront_iteration(w, moments, ctx->sm_count, st, guided ? &ctx->guide : nullptr,
                                                 marks));
    ctx->stats.kernel_launches += (guided ? 4u : 3u) + (sort_rays ? 3u : 0u);
    ctx->stats.wf_iterations += 1;
    const int k = int(it % kWfRing);
    TC_CUDA(ctx, cudaMemcpyAsync(ctx->wf_live_host + k, w.q + tcb::kWfLive, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                 st));
    TC_CUDA(ctx, cudaMemcpyAsync(ctx->wf_work_host + k, L.work_counter, sizeof(unsigned long long),
                                 cudaMemcpyDeviceToHost, st));
    TC_CUDA(ctx, cudaEventRecord(ctx->wf_events[k], st));
    if (it >= uint64_t(kWfLag)) {
      const int j = int((it - kWfLag) % kWfRing);
      TC_CUDA(ctx, cudaEventSynchronize(ctx->wf_events[j]));
      if (ctx->wf_live_host[j] == 0) break;
      if (ctx->wf_work_host[j] >= items) w.work_done = 1u;
    }
  }
  return TC_OK;
}

// Everything a render puts on `st` without synchronising the host: accumulation setup, the path
// kernel (or the guided wavefront's rounds) and the counter readback into `counters_host`.
// `timing` records the context's events around the kernels (left out while capturing a graph).
// frame_index_dev / camera_dev, when set, make the kernels read those per-frame values from
// device memory. On success ctx->accumulated is advanced.
static int append_training_samples(tc_context* ctx, bool fresh, cudaStream_t st);

static int enqueue_render(tc_context* ctx, const tc_gpu_render_params* p, const tc_render_options& o, cudaStream_t st,
                          bool timing, const uint32_t* frame_index_dev, const float* camera_dev,
                          unsigned long long* counters_host) {
  const bool moments = o.keep_moments != 0;
  const uint32_t npix = p->width * p->height;
  const int block = o.block_size ? int(o.block_size) : 128;
  if (block % 32 != 0 || block < 32 || block > 256)
    return fail(ctx, TC_ERR_INVALID, "block_size must be a multiple of 32 in [32, 256]");
  if (o.guide_record > 2)
    return fail(ctx, TC_ERR_INVALID, "guide_record must be 0, 1 (start a new sample pool) or 2 (add to the pool)");
  if (o.guiding && !ctx->has_guide) return fail(ctx, TC_ERR_STATE, "guided rendering needs tc_guide_set_params first");
  if (!(o.guide_fraction >= 0.0f && o.guide_fraction < 1.0f))
    return fail(ctx, TC_ERR_INVALID, "guide_fraction must be in [0, 1)");
  if (o.short_stack > 16) return fail(ctx, TC_ERR_INVALID, "short_stack must be at most 16 entries");
  if (o.refill_lanes > 32) return fail(ctx, TC_ERR_INVALID, "refill_lanes must be at most 32");
  if (timing) TC_CUDA(ctx, cudaEventRecord(ctx->ev_begin, st));
  if (int rc = prepare_accumulation(ctx, p, moments, st)) return rc;
  ctx->stats.kernel_launches = 0;
  ctx->stats.wf_iterations = 0;
  ctx->stats.trace_ms = ctx->stats.logic_ms = ctx->stats.shade_ms = ctx->stats.guide_ms = 0.0f;
  ctx->wf_marks_used = 0;

  tcb::RenderLaunch L{};
  L.f.scene = ctx->scene;
  L.f.width = p->width;
  L.f.height = p->height;
  L.f.samples = p->samples;
  L.f.max_bounces = p->max_bounces;
  L.f.frame_index = p->frame_index;
  L.f.sample_base = ctx->accumulated;
  L.f.samples_per_item = std::min<uint32_t>(o.samples_per_item ? o.samples_per_item : 1u, p->samples);
  L.f.items_per_pixel = (p->samples + L.f.samples_per_item - 1) / L.f.samples_per_item;
  L.f.frame_index_dev = frame_index_dev;
  L.f.camera_dev = camera_dev;
  L.total_items = uint64_t(npix) * L.f.items_per_pixel;
  L.f.accum = ctx->accum.as<double>();
  L.f.accum_sq = moments ? ctx->accum_sq.as<double>() : nullptr;
  L.work_counter = ctx->work_counter.as<unsigned long long>();
  L.counters = ctx->counters.as<unsigned long long>();
  L.short_stack = int(o.short_stack);
  L.min_active = int(o.refill_lanes ? o.refill_lanes : kDefaultRefillLanes);
  TC_CUDA(ctx, cudaMemsetAsync(ctx->work_counter.ptr, 0, sizeof(unsigned long long), st));
  TC_CUDA(ctx, cudaMemsetAsync(ctx->counters.ptr, 0, 4 * sizeof(unsigned long long), st));
  const int mode = o.guiding ? tcb::kModeGuided : (o.guide_record ? tcb::kModeRecord : tcb::kModePlain);
  int per_sm = tcb::render_max_blocks_per_sm(block, moments, mode, L.short_stack, L.min_active);
  if (per_sm <= 0) return fail(ctx, TC_ERR_CUDA, "render kernel cannot be resident with this block size");
  // The persistent grid fills every SM; a frame with fewer work items than that needs fewer blocks
  // (guided rounds size their work on the device, so they keep the full grid).
  int grid = per_sm * ctx->sm_count;
  if (mode != tcb::kModeGuided)
    grid = int(std::max<uint64_t>(1, std::min<uint64_t>(uint64_t(grid), (L.total_items + block - 1) / block)));
  if (o.guide_record) {
    // One record per diffuse scatter and per environment shadow ray, at most two per bounce
    // (capped at 2^27 records, 8 GiB; records past the cap are dropped), and the final radiance
    // of every path of the batch.
    const uint64_t paths = uint64_t(npix) * p->samples;
    if (paths > (1ull << 31)) return fail(ctx, TC_ERR_INVALID, "too many paths to record in one batch");
    ctx->rec_capacity =
        uint32_t(std::min<uint64_t>(2 * uint64_t(std::max<uint32_t>(p->max_bounces, 1)) * paths, uint64_t(1) << 27));
    TC_CUDA(ctx, ctx->rec_records.reserve(sizeof(float4) * 4 * size_t(ctx->rec_capacity)));
    TC_CUDA(ctx, ctx->rec_count.reserve(sizeof(uint32_t)));
    TC_CUDA(ctx, ctx->rec_path_rad.reserve(sizeof(float4) * size_t(paths)));
    TC_CUDA(ctx, cudaMemsetAsync(ctx->rec_count.ptr, 0, sizeof(uint32_t), st));
    L.g.records = ctx->rec_records.as<float4>();
    L.g.record_count = ctx->rec_count.as<uint32_t>();
    L.g.record_capacity = ctx->rec_capacity;
    L.g.path_radiance = ctx->rec_path_rad.as<float4>();
  }
  // Plain and guided renders called directly (not captured into a graph) may run as a wavefront.
  const bool direct = !camera_dev && !frame_index_dev;
  const bool wf_mode = mode == tcb::kModePlain || mode == tcb::kModeGuided || mode == tcb::kModeRecord;
  if (o.schedule > TC_SCHEDULE_WAVEFRONT) return fail(ctx, TC_ERR_INVALID, "schedule must be 0 (auto), 1 or 2");
  if (o.schedule == TC_SCHEDULE_WAVEFRONT && wf_mode && !direct)
    return fail(ctx, TC_ERR_INVALID, "the wavefront schedule renders direct calls only, not captured frames");
  const bool wavefront =
      wf_mode && direct && p->max_bounces > 0 && p->max_bounces <= tcb::kWfDepthMask &&
      (o.schedule == TC_SCHEDULE_WAVEFRONT ||
       (o.schedule == TC_SCHEDULE_AUTO && uint64_t(npix) * p->samples >= kWavefrontMinPaths));
  if (ctx->scene.tri_verts && !wavefront)
    return fail(ctx, TC_ERR_INVALID,
                "the watertight triangle test is traced by tc_trace_closest and by plain wavefront renders only");
  if (o.guiding && o.guide_record && !wavefront)
    return fail(ctx, TC_ERR_INVALID, "guided renders record training samples on the wavefront schedule only");
  if (timing) TC_CUDA(ctx, cudaEventRecord(ctx->ev_kernel0, st));
  if (wavefront) {
    L.total_items = uint64_t(npix) * p->samples;  // one path per work item
    L.g.guide_fraction = o.guide_fraction > 0.0f ? o.guide_fraction : 0.5f;
    if (o.ray_sort > 2) return fail(ctx, TC_ERR_INVALID, "ray_sort must be 0 (default), 1 (off) or 2 (on)");
    if (int rc = run_wavefront(ctx, L, o.wave_paths ? o.wave_paths : kWavefrontSlots, p->max_bounces,
                               int(o.refill_lanes), moments, mode == tcb::kModeGuided, o.ray_sort == 2,
                               timing && o.phase_timing != 0, st))
      return rc;
  } else if (mode != tcb::kModeGuided) {
    TC_CUDA(ctx, tcb::launch_render(L, block, grid, moments, st, mode));
    ctx->stats.kernel_launches = 1;
  } else {
    // Wavefront: waves of whole samples per pixel; within a wave, rounds of (path kernel ->
    // suspended diffuse vertices -> tensor-core inference of their mixtures -> resume). Counts
    // stay on the device, so the rounds need no host synchronisation.
    const uint32_t wave_cap = o.wave_paths ? o.wave_paths : (1u << 23);
    L.g.guide_fraction = o.guide_fraction > 0.0f ? o.guide_fraction : 0.5f;
    const uint32_t wave_spp = std::max<uint32_t>(1u, std::min<uint32_t>(p->samples, wave_cap / npix));
    const uint32_t cap = wave_spp * npix;
    const uint32_t rounds = p->max_bounces > 1 ? p->max_bounces - 1 : 0;
    TC_CUDA(ctx, ctx->w_state_a.reserve(sizeof(float4) * 6 * size_t(cap)));
    TC_CUDA(ctx, ctx->w_state_b.reserve(sizeof(float4) * 6 * size_t(cap)));
    TC_CUDA(ctx, ctx->w_query.reserve(sizeof(float4) * 2 * size_t(cap)));
    TC_CUDA(ctx, ctx->w_mix.reserve(sizeof(float4) * tcb::kGuideDecodedF4 * size_t(cap)));
    TC_CUDA(ctx, ctx->w_counts.reserve(sizeof(uint32_t) * (rounds + 2)));
    float4* state_in = ctx->w_state_a.as<float4>();
    float4* state_out = ctx->w_state_b.as<float4>();
    uint32_t* counts = ctx->w_counts.as<uint32_t>();
    for (uint32_t first = 0; first < p->samples; first += wave_spp) {
      const uint32_t ws = std::min(wave_spp, p->samples - first);
      TC_CUDA(ctx, cudaMemsetAsync(counts, 0, sizeof(uint32_t) * (rounds + 2), st));
      tcb::RenderLaunch R = L;
      R.total_items = uint64_t(npix) * ws;
      R.g.capacity = cap;
      R.g.out_query = ctx->w_query.as<float4>();
      R.g.wave_first_sample = ctx->accumulated + first;
      R.g.wave_spp = ws;
      R.g.resume = 0;
      R.g.out_state = state_out;
      R.g.out_count = counts;
      TC_CUDA(ctx, cudaMemsetAsync(ctx->work_counter.ptr, 0, sizeof(unsigned long long), st));
      TC_CUDA(ctx, tcb::launch_render(R, block, grid, moments, st, mode));
      ctx->stats.kernel_launches += 1 + 2 * rounds;
      for (uint32_t r = 0; r < rounds; ++r) {
        std::swap(state_in, state_out);
        TC_CUDA(ctx, tcb::guide_launch_infer(ctx->guide, ctx->w_query.as<float4>(), cap, ctx->w_mix.as<float4>(),
                                             ctx->sm_count, st, counts + r));
        R.g.resume = 1;
        R.g.in_state = state_in;
        R.g.in_count = counts + r;
        R.g.in_mix = ctx->w_mix.as<float4>();
        R.g.out_state = state_out;
        R.g.out_count = counts + r + 1;
        TC_CUDA(ctx, cudaMemsetAsync(ctx->work_counter.ptr, 0, sizeof(unsigned long long), st));
        TC_CUDA(ctx, tcb::launch_render(R, block, grid, moments, st, mode));
      }
    }
  }
  if (o.guide_record) {
    if (int rc = append_training_samples(ctx, o.guide_record == 1, st)) return rc;
    ctx->stats.kernel_launches += 1;
  }
  if (timing) TC_CUDA(ctx, cudaEventRecord(ctx->ev_kernel1, st));
  if (counters_host)
    TC_CUDA(ctx, cudaMemcpyAsync(counters_host, ctx->counters.ptr, 4 * sizeof(unsigned long long),
                                 cudaMemcpyDeviceToHost, st));
  if (timing) TC_CUDA(ctx, cudaEventRecord(ctx->ev_end, st));
  ctx->accumulated += p->samples;
  if (o.guide_record) ctx->has_records = true;
  return TC_OK;
}

// The wavefront-only statistics, zeroed by the calls that do not run the wavefront schedule.
static void clear_phase_stats(tc_stats& st) {
  st.trace_ms = st.logic_ms = st.shade_ms = st.guide_ms = 0.0f;
  st.wf_iterations = 0;
}

// Counters of a finished render into the context's statistics; fails when paths went missing.
static int finish_render_stats(tc_context* ctx, const unsigned long long* counters, uint64_t expected_paths,
                               bool timing) {
  ctx->stats.paths = counters[0];
  ctx->stats.extension_rays = counters[1];
  ctx->stats.shadow_rays = counters[2];
  ctx->stats.rays = counters[1] + counters[2];
  if (timing) {
    cudaEventElapsedTime(&ctx->stats.kernel_ms, ctx->ev_kernel0, ctx->ev_kernel1);
    cudaEventElapsedTime(&ctx->stats.total_ms, ctx->ev_begin, ctx->ev_end);
    // Phase timing, per iteration: marks 0-1 logic, 1-2 inference, 2-3 shading, 3-4 tracing
    // (plain renders leave mark 2 out: shading is 1-3).
    auto span = [&](uint32_t i, int a, int b) {
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, ctx->wf_marks[i][a], ctx->wf_marks[i][b]);
      return ms;
    };
    for (uint32_t i = 0; i < ctx->wf_marks_used; ++i) {
      ctx->stats.logic_ms += span(i, 0, 1);
      if (ctx->wf_marks_guided) {
        ctx->stats.guide_ms += span(i, 1, 2);
        ctx->stats.shade_ms += span(i, 2, 3);
      } else {
        ctx->stats.shade_ms += span(i, 1, 3);
      }
      ctx->stats.trace_ms += span(i, 3, 4);
    }
  }
  if (counters[0] != expected_paths)
    return fail(ctx, TC_ERR_DEVICE_STATUS, "path kernel completed " + std::to_string(counters[0]) + " of " +
                                                std::to_string(expected_paths) + " paths");
  return TC_OK;
}

int tc_render(tc_context* ctx, const tc_gpu_render_params* p, const tc_render_options* opt) {
  if (!ctx) return fail(nullptr, TC_ERR_INVALID, "context is null");
  if (int rc = check_render_params(ctx, p)) return rc;
  TC_CUDA(ctx, cudaSetDevice(ctx->device));
  tc_render_options o{};
  if (opt) o = *opt;
  unsigned long long counters[4] = {0, 0, 0, 0};
  if (int rc = enqueue_render(ctx, p, o, ctx->stream, true, nullptr, nullptr, counters)) return rc;
  TC_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return finish_render_stats(ctx, counters, uint64_t(p->width) * p->height * p->samples, true);
}

static int render_batch_shared(tc_context* lead, tc_context* const* contexts, const tc_gpu_render_params* params,
                               const std::vector<size_t>& idx, const tc_render_options& o, int block, cudaStream_t st,
                               unsigned long long* counters_host, uint64_t* paths_out, uint32_t* launches_out);

int tc_render_batch(tc_context* const* contexts, const tc_gpu_render_params* params, size_t n,
                    const tc_render_options* opt) {
  if (!contexts || !params || n == 0) return fail(nullptr, TC_ERR_INVALID, "batch is empty or null");
  tc_context* lead = contexts[0];
  if (!lead) return fail(nullptr, TC_ERR_INVALID, "context 0 of the batch is null");
  tc_render_options o{};
  if (opt) o = *opt;
  if (o.keep_moments || o.guide_record)
    return fail(lead, TC_ERR_INVALID, "batched frames do not keep moments or record training samples");
  if (o.guiding && !(o.guide_fraction >= 0.0f && o.guide_fraction < 1.0f))
    return fail(lead, TC_ERR_INVALID, "guide_fraction must be in [0, 1)");
  const int block = o.block_size ? int(o.block_size) : 128;
  if (block % 32 != 0 || block < 32 || block > 256)
    return fail(lead, TC_ERR_INVALID, "block_size must be a multiple of 32 in [32, 256]");
  if (o.short_stack > 16) return fail(lead, TC_ERR_INVALID, "short_stack must be at most 16 entries");
  if (o.refill_lanes > 32) return fail(lead, TC_ERR_INVALID, "refill_lanes must be at most 32");
  for (size_t i = 0; i < n; ++i) {
    tc_context* c = contexts[i];
    if (!c) return fail(lead, TC_ERR_INVALID, "context " + std::to_string(i) + " of the batch is null");
    if (c->device != lead->device) return fail(lead, TC_ERR_INVALID, "batched contexts must share one device");
    if (c->scene.tri_verts)
      return fail(lead, TC_ERR_INVALID, "batched frames use the Moller-Trumbore triangle test");
    for (size_t j = 0; j < i; ++j)
      if (contexts[j] == c) return fail(lead, TC_ERR_INVALID, "a context appears twice in the batch");
    if (int rc = check_render_params(c, &params[i])) {
      lead->error = "frame " + std::to_string(i) + ": " + c->error;
      return rc;
    }
    if (o.guiding && !c->has_guide)
      return fail(lead, TC_ERR_STATE, "frame " + std::to_string(i) + ": guided rendering needs tc_guide_set_params first");
  }
  // Frames of at least kWavefrontMinPaths paths fill the GPU on their own: with the automatic
  // schedule each of them gets its own wavefront call (on the batch's stream, into its own
  // context's buffers), and the other frames share one batched launch of the path kernel, where
  // batching pays (frames too small to fill the SMs). TC_SCHEDULE_MEGAKERNEL puts every frame in
  // the batched launch, TC_SCHEDULE_WAVEFRONT every frame the wavefront can take (1 to
  // kWfDepthMask bounces) in its own call.
  if (o.schedule > TC_SCHEDULE_WAVEFRONT) return fail(lead, TC_ERR_INVALID, "schedule must be 0 (auto), 1 or 2");
  std::vector<size_t> own, shared;
  for (size_t i = 0; i < n; ++i) {
    const uint64_t fp = uint64_t(params[i].width) * params[i].height * params[i].samples;
    const bool wf_ok = params[i].max_bounces > 0 && params[i].max_bounces <= tcb::kWfDepthMask;
    const bool wf = wf_ok && (o.schedule == TC_SCHEDULE_WAVEFRONT ||
                              (o.schedule == TC_SCHEDULE_AUTO && fp >= kWavefrontMinPaths));
    (wf ? own : shared).push_back(i);
  }
  for (size_t i : shared)
    if (o.guiding && params[i].samples != params[shared[0]].samples)
      return fail(lead, TC_ERR_INVALID, "guided frames of one batched launch must share one sample count");
  TC_CUDA(lead, cudaSetDevice(lead->device));
  cudaStream_t st = lead->stream;
  TC_CUDA(lead, cudaEventRecord(lead->ev_begin, st));
  for (size_t i = 0; i < n; ++i) {
    tc_context* c = contexts[i];
    if (c != lead) {  // the batch writes this context's buffers: order after its own stream
      TC_CUDA(lead, cudaEventRecord(c->ev_begin, c->stream));
      TC_CUDA(lead, cudaStreamWaitEvent(st, c->ev_begin, 0));
    }
  }
  TC_CUDA(lead, cudaEventRecord(lead->ev_kernel0, st));
  uint32_t launches = 0;
  unsigned long long counters[4] = {0, 0, 0, 0};
  uint64_t paths = 0;
  if (!shared.empty())
    if (int rc = render_batch_shared(lead, contexts, params, shared, o, block, st, counters, &paths, &launches))
      return rc;
  // Own wavefront calls after the shared launch (whose counters are already on their way to the host).
  std::vector<std::array<unsigned long long, 4>> own_counters(own.size());
  for (size_t k = 0; k < own.size(); ++k) {
    const size_t i = own[k];
    tc_context* c = contexts[i];
    tc_render_options oi = o;
    oi.schedule = TC_SCHEDULE_WAVEFRONT;
    if (int rc = enqueue_render(c, &params[i], oi, st, false, nullptr, nullptr, own_counters[k].data())) {
      if (c != lead) lead->error = "frame " + std::to_string(i) + ": " + c->error;
      return rc;
    }
    launches += c->stats.kernel_launches;
  }
  TC_CUDA(lead, cudaEventRecord(lead->ev_kernel1, st));
  TC_CUDA(lead, cudaEventRecord(lead->ev_end, st));
  TC_CUDA(lead, cudaStreamSynchronize(st));
  if (counters[0] != paths)
    return fail(lead, TC_ERR_DEVICE_STATUS, "batched path kernel completed " + std::to_string(counters[0]) + " of " +
                                                std::to_string(paths) + " paths");
  for (size_t k = 0; k < own.size(); ++k) {
    const size_t i = own[k];
    const uint64_t fp = uint64_t(params[i].width) * params[i].height * params[i].samples;
    if (own_counters[k][0] != fp)
      return fail(lead, TC_ERR_DEVICE_STATUS, "frame " + std::to_string(i) + ": path kernel completed " +
                                                  std::to_string(own_counters[k][0]) + " of " + std::to_string(fp) +
                                                  " paths");
    for (int j = 0; j < 4; ++j) counters[j] += own_counters[k][j];
  }
  for (size_t i : shared) contexts[i]->accumulated += params[i].samples;
  lead->stats.paths = counters[0];
  lead->stats.extension_rays = counters[1];
  lead->stats.shadow_rays = counters[2];
  lead->stats.rays = counters[1] + counters[2];
  lead->stats.kernel_launches = launches;
  clear_phase_stats(lead->stats);
  cudaEventElapsedTime(&lead->stats.kernel_ms, lead->ev_kernel0, lead->ev_kernel1);
  cudaEventElapsedTime(&lead->stats.total_ms, lead->ev_begin, lead->ev_end);
  return TC_OK;
}

// The batched launch over the frames `idx` of a batch (validated by tc_render_batch): one
// persistent path-kernel launch over all their work items (guided: the suspend -> per-frame
// inference -> resume rounds). Enqueues on `st`, copies the launch's counters to `counters_host`
// (stream-ordered), returns the frames' path count and the kernel launches.
static int render_batch_shared(tc_context* lead, tc_context* const* contexts, const tc_gpu_render_params* params,
                               const std::vector<size_t>& idx, const tc_render_options& o, int block, cudaStream_t st,
                               unsigned long long* counters_host, uint64_t* paths_out, uint32_t* launches_out) {
  const size_t n = idx.size();
  std::vector<tcb::FrameJob> jobs(n);
  uint64_t items = 0, paths = 0;
  for (size_t k = 0; k < n; ++k) {
    const size_t i = idx[k];
    tc_context* c = contexts[i];
    const tc_gpu_render_params* p = &params[i];
    if (int rc = prepare_accumulation(c, p, false, st)) {
      lead->error = "frame " + std::to_string(i) + ": " + c->error;
      return rc;
    }
    tcb::FrameJob& J = jobs[k];
    J = tcb::FrameJob{};
    J.scene = c->scene;
    J.accum = c->accum.as<double>();
    J.accum_sq = nullptr;
    J.item_begin = items;
    J.width = p->width;
    J.height = p->height;
    J.samples = p->samples;
    J.max_bounces = p->max_bounces;
    J.frame_index = p->frame_index;
    J.sample_base = c->accumulated;
    J.samples_per_item = std::min<uint32_t>(o.samples_per_item ? o.samples_per_item : 1u, p->samples);
    J.items_per_pixel = (p->samples + J.samples_per_item - 1) / J.samples_per_item;
    items += uint64_t(p->width) * p->height * J.items_per_pixel;
    paths += uint64_t(p->width) * p->height * p->samples;
  }
  // Guided: waves of whole samples per pixel over all frames; frame i owns the region
  // [ws * pix_begin_i, ws * (pix_begin_i + pixels_i)) of the wave's suspended-path buffers.
  uint64_t total_pix = 0;
  for (size_t k = 0; k < n; ++k) {
    jobs[k].pix_begin = uint32_t(total_pix);
    total_pix += uint64_t(params[idx[k]].width) * params[idx[k]].height;
  }
  const uint32_t spp = params[idx[0]].samples;  // guided batched frames share it
  uint32_t ws = 0, rounds = 0;
  if (o.guiding) {
    const uint32_t wave_cap = o.wave_paths ? o.wave_paths : (1u << 23);
    ws = uint32_t(std::max<uint64_t>(1, std::min<uint64_t>(spp, wave_cap / total_pix)));
    if (uint64_t(ws) * total_pix > (1ull << 31)) return fail(lead, TC_ERR_INVALID, "batched guided frames are too large");
    for (size_t k = 0; k < n; ++k) {
      const tc_gpu_render_params& pk = params[idx[k]];
      jobs[k].wave_offset = ws * jobs[k].pix_begin;
      jobs[k].wave_capacity = ws * pk.width * pk.height;
      rounds = std::max(rounds, pk.max_bounces > 1 ? pk.max_bounces - 1 : 0u);
    }
  }
  TC_CUDA(lead, upload(lead->batch_jobs, jobs.data(), jobs.size(), st));
  tcb::RenderLaunch L{};
  L.jobs = lead->batch_jobs.as<tcb::FrameJob>();
  L.job_count = uint32_t(n);
  L.total_items = items;
  L.work_counter = lead->work_counter.as<unsigned long long>();
  L.counters = lead->counters.as<unsigned long long>();
  L.short_stack = int(o.short_stack);
  L.min_active = int(o.refill_lanes ? o.refill_lanes : kDefaultRefillLanes);
  TC_CUDA(lead, cudaMemsetAsync(lead->work_counter.ptr, 0, sizeof(unsigned long long), st));
  TC_CUDA(lead, cudaMemsetAsync(lead->counters.ptr, 0, 4 * sizeof(unsigned long long), st));
  const int per_sm = tcb::render_batch_max_blocks_per_sm(block, o.guiding != 0);
  if (per_sm <= 0) return fail(lead, TC_ERR_CUDA, "batched render kernel cannot be resident with this block size");
  const int grid = per_sm * lead->sm_count;
  uint32_t launches = 0;
  if (!o.guiding) {
    TC_CUDA(lead, tcb::launch_render_batch(L, block, grid, st));
    launches = 1;
  } else {
    // Rounds of (batched path kernel -> each frame's network infers its frame's queries -> prefix
    // of the per-frame counts -> batched resume), as the single-frame guided wavefront does.
    const size_t cap = size_t(ws) * total_pix;
    TC_CUDA(lead, lead->w_state_a.reserve(sizeof(float4) * 6 * cap));
    TC_CUDA(lead, lead->w_state_b.reserve(sizeof(float4) * 6 * cap));
    TC_CUDA(lead, lead->w_query.reserve(sizeof(float4) * 2 * cap));
    TC_CUDA(lead, lead->w_mix.reserve(sizeof(float4) * tcb::kGuideDecodedF4 * cap));
    TC_CUDA(lead, lead->w_counts.reserve(sizeof(uint32_t) * (rounds + 1) * n));
    TC_CUDA(lead, lead->w_prefix.reserve(sizeof(uint32_t) * std::max<size_t>(rounds, 1) * (n + 1)));
    float4* state_in = lead->w_state_a.as<float4>();
    float4* state_out = lead->w_state_b.as<float4>();
    uint32_t* counts = lead->w_counts.as<uint32_t>();
    uint32_t* prefix = lead->w_prefix.as<uint32_t>();
    float4* query = lead->w_query.as<float4>();
    float4* mix = lead->w_mix.as<float4>();
    L.g.guide_fraction = o.guide_fraction > 0.0f ? o.guide_fraction : 0.5f;
    L.g.capacity = uint32_t(cap);
    L.g.out_query = query;
    for (uint32_t first = 0; first < spp; first += ws) {
      const uint32_t wsz = std::min(ws, spp - first);
      TC_CUDA(lead, cudaMemsetAsync(counts, 0, sizeof(uint32_t) * (rounds + 1) * n, st));
      tcb::RenderLaunch R = L;
      R.total_items = uint64_t(wsz) * total_pix;
      R.g.wave_first_sample = first;
      R.g.wave_spp = wsz;
      R.g.resume = 0;
      R.g.out_state = state_out;
      R.g.job_out_count = counts;
      TC_CUDA(lead, cudaMemsetAsync(lead->work_counter.ptr, 0, sizeof(unsigned long long), st));
      TC_CUDA(lead, tcb::launch_render_batch(R, block, grid, st, true));
      launches += 1 + rounds * uint32_t(n + 2);
      for (uint32_t r = 0; r < rounds; ++r) {
        std::swap(state_in, state_out);
        for (size_t k = 0; k < n; ++k)
          TC_CUDA(lead, tcb::guide_launch_infer(contexts[idx[k]]->guide, query + 2 * size_t(jobs[k].wave_offset),
                                                jobs[k].wave_capacity,
                                                mix + size_t(tcb::kGuideDecodedF4) * jobs[k].wave_offset,
                                                lead->sm_count, st, counts + size_t(r) * n + k));
        uint32_t* pre = prefix + size_t(r) * (n + 1);
        TC_CUDA(lead, tcb::launch_job_prefix(counts + size_t(r) * n, L.jobs, uint32_t(n), pre, st));
        R.g.resume = 1;
        R.g.in_state = state_in;
        R.g.in_job_prefix = pre;
        R.g.in_mix = mix;
        R.g.out_state = state_out;
        R.g.job_out_count = counts + size_t(r + 1) * n;
        TC_CUDA(lead, cudaMemsetAsync(lead->work_counter.ptr, 0, sizeof(unsigned long long), st));
        TC_CUDA(lead, tcb::launch_render_batch(R, block, grid, st, true));
      }
    }
  }
  TC_CUDA(lead, cudaMemcpyAsync(counters_host, lead->counters.ptr, 4 * sizeof(unsigned long long),
                               cudaMemcpyDeviceToHost, st));
  *paths_out = paths;
  *launches_out = launches;
  return TC_OK;
}

// ------------------------------------------------------------------------ autotuner
int tc_autotune(tc_context* ctx, const tc_gpu_render_params* params, const tc_render_options* base,
                uint32_t probe_samples, tc_tune_result* out) {
  if (!ctx) return fail(nullptr, TC_ERR_INVALID, "context is null");
  if (!out) return fail(ctx, TC_ERR_INVALID, "result pointer is null");
  if (int rc = check_render_params(ctx, params)) return rc;
  tc_render_options b{};
  if (base) b = *base;
  if (b.guide_record || b.keep_moments)
    return fail(ctx, TC_ERR_INVALID, "the autotuner times plain or guided renders only");
  TC_CUDA(ctx, cudaSetDevice(ctx->device));
  tc_gpu_render_params p = *params;
  p.accumulated_samples = 0;
  p.samples = probe_samples ? probe_samples : std::min<uint32_t>(params->samples, 4u);
  // Coordinate search over the launch shape, one knob at a time in this order, each stage keeping
  // the fastest value so far: (plain) schedule, then block size, dynamic-fetch threshold (refill
  // lanes) and shared short-stack entries of the megakernel, or the trace launch's refill lanes of
  // the wavefront; last the wavefront's path slots (guided or plain wavefront) or the
  // megakernel's samples per work item.
  tc_render_options best = b;
  if (!best.block_size) best.block_size = 128;
  if (!best.refill_lanes) best.refill_lanes = kDefaultRefillLanes;
  if (!best.samples_per_item) best.samples_per_item = 1;

  float best_ms = -1.0f;
  uint32_t tried = 0;
  auto time_shape = [&](const tc_render_options& o, float& ms) -> int {
    // One untimed run sizes the buffers and warms the caches, then one timed run.
    unsigned long long counters[4] = {0, 0, 0, 0};
    if (int rc = enqueue_render(ctx, &p, o, ctx->stream, false, nullptr, nullptr, counters)) return rc;
    if (int rc = enqueue_render(ctx, &p, o, ctx->stream, true, nullptr, nullptr, counters)) return rc;
    TC_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (int rc = finish_render_stats(ctx, counters, uint64_t(p.width) * p.height * p.samples, true)) return rc;
    ms = ctx->stats.kernel_ms;
    ++tried;
    return TC_OK;
  };
  if (int rc = time_shape(best, best_ms)) return rc;
  auto stage = [&](uint32_t tc_render_options::*field, std::initializer_list<uint32_t> values) -> int {
    for (uint32_t v : values) {
      if (best.*field == v) continue;
      tc_render_options o = best;
      o.*field = v;
      float ms = 0.0f;
      if (int rc = time_shape(o, ms)) return rc;
      if (ms < best_ms) {
        best_ms = ms;
        best = o;
      }
    }
    return TC_OK;
  };
  const bool can_wavefront = p.max_bounces > 0 && !ctx->scene.tri_verts;
  // The schedule the automatic choice takes for this probe, so the result names a concrete one.
  if (best.schedule == TC_SCHEDULE_AUTO)
    best.schedule = can_wavefront && uint64_t(p.width) * p.height * p.samples >= kWavefrontMinPaths
                        ? TC_SCHEDULE_WAVEFRONT
                        : TC_SCHEDULE_MEGAKERNEL;
  if (can_wavefront)
    if (int rc = stage(&tc_render_options::schedule, {TC_SCHEDULE_MEGAKERNEL, TC_SCHEDULE_WAVEFRONT})) return rc;
  const bool wavefront = best.schedule == TC_SCHEDULE_WAVEFRONT;
  if (!wavefront)
    if (int rc = stage(&tc_render_options::block_size, {64u, 128u, 256u})) return rc;
  if (int rc = stage(&tc_render_options::refill_lanes, {1u, 12u, 20u, 28u})) return rc;
  if (!wavefront)
    if (int rc = stage(&tc_render_options::short_stack, {0u, 8u, 16u})) return rc;
  if (wavefront) {
    if (int rc = stage(&tc_render_options::wave_paths, {1u << 21, 1u << 22, 1u << 23})) return rc;
  } else if (b.guiding) {
    if (int rc = stage(&tc_render_options::wave_paths, {1u << 21, 1u << 22, 1u << 23})) return rc;
  } else {
    if (int rc = stage(&tc_render_options::samples_per_item, {1u, 2u, 4u})) return rc;
  }
  out->best = best;
  out->best_kernel_ms = best_ms;
  out->best_mpaths_per_s = best_ms > 0.0f ? float(double(p.width) * p.height * p.samples / (1e3 * double(best_ms))) : 0.0f;
  out->candidates = tried;
  out->probe_samples = p.samples;
  return TC_OK;
}

// ------------------------------------------------------------------------ animation frames
// One captured CUDA graph per animation: pinned staging -> device geometry, refit, render (plain
// or guided wavefront), display conversion and the RGBA8 readback. A frame only rewrites the
// pinned staging (geometry, camera, frame index) and replays the graph.
struct tc_animation {
  tc_context* ctx = nullptr;
  tc_gpu_render_params params{};
  tc_render_options options{};
  float exposure = 0.0f;
  bool update_lights = false;
  bool rebuild = false;                     // per-frame median-split build instead of a refit
  size_t npix = 0;
  tc_gpu_sphere* h_spheres = nullptr;       // pinned staging
  tc_gpu_triangle* h_triangles = nullptr;
  tcb::DevLight* h_lights = nullptr;
  tc_gpu_triangle_attributes* h_attrs = nullptr;
  uint32_t* h_attr_flags = nullptr;         // rebuild mode: the build's triangle attribute flags
  uint32_t* h_status = nullptr;             // rebuild mode: the device build's status word
  float* h_frame = nullptr;                 // camera (16 floats) then the frame index (uint32)
  uint8_t* h_rgba = nullptr;                // pinned output
  unsigned long long* h_counters = nullptr;
  DevBuf d_frame, d_rgba;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

static void animation_free(tc_animation* a) {
  if (!a) return;
  if (a->ctx) cudaSetDevice(a->ctx->device);
  if (a->exec) cudaGraphExecDestroy(a->exec);
  if (a->graph) cudaGraphDestroy(a->graph);
  for (void* h : {static_cast<void*>(a->h_spheres), static_cast<void*>(a->h_triangles), static_cast<void*>(a->h_lights),
                  static_cast<void*>(a->h_attrs), static_cast<void*>(a->h_attr_flags), static_cast<void*>(a->h_status),
                  static_cast<void*>(a->h_frame), static_cast<void*>(a->h_rgba), static_cast<void*>(a->h_counters)})
    if (h) cudaFreeHost(h);
  delete a;
}

// Copies one evaluated frame into the pinned staging.
static int animation_stage(tc_animation* a, const tc_scene_data* sd, uint32_t frame_index) {
  tc_context* ctx = a->ctx;
  if (sd->sphere_count != ctx->sphere_count || sd->triangle_count != ctx->triangle_count ||
      sd->material_count != ctx->material_count || sd->light_count != ctx->light_count)
    return fail(ctx, TC_ERR_INVALID,
                "evaluated scenes must preserve GPU geometry, material, light, and BVH primitive counts");
  if ((sd->sphere_count && !sd->spheres) || (sd->triangle_count && !sd->triangles) || !sd->materials)
    return fail(ctx, TC_ERR_INVALID, "frame geometry or material pointer is null");
  if (int rc = validate_geometry(ctx, sd, ctx->material_count)) return rc;
  if (sd->sphere_count) std::memcpy(a->h_spheres, sd->spheres, sizeof(tc_gpu_sphere) * sd->sphere_count);
  if (sd->triangle_count) std::memcpy(a->h_triangles, sd->triangles, sizeof(tc_gpu_triangle) * sd->triangle_count);
  if (a->h_attrs && sd->triangle_attributes) {
    std::memcpy(a->h_attrs, sd->triangle_attributes, sizeof(tc_gpu_triangle_attributes) * sd->triangle_count);
    if (a->h_attr_flags)
      for (size_t i = 0; i < sd->triangle_count; ++i) a->h_attr_flags[i] = sd->triangle_attributes[i].flags & 3u;
  }
  if (a->update_lights && sd->light_count) {
    std::vector<tcb::DevLight> lights;
    if (int rc = pack_lights(ctx, sd, ctx->material_count, lights)) return rc;
    std::memcpy(a->h_lights, lights.data(), sizeof(tcb::DevLight) * lights.size());
  }
  const tc_gpu_camera& c = sd->camera;
  for (int k = 0; k < 4; ++k) {
    a->h_frame[k] = c.origin[k];
    a->h_frame[4 + k] = c.lower_left_corner[k];
    a->h_frame[8 + k] = c.horizontal[k];
    a->h_frame[12 + k] = c.vertical[k];
  }
  std::memcpy(a->h_frame + 16, &frame_index, sizeof(uint32_t));
  return TC_OK;
}

// Enqueues the device work of one frame (what the graph holds).
static int animation_enqueue(tc_animation* a, cudaStream_t st) {
  tc_context* ctx = a->ctx;
  TC_CUDA(ctx, cudaMemcpyAsync(a->d_frame.ptr, a->h_frame, 20 * sizeof(float), cudaMemcpyHostToDevice, st));
  if (a->update_lights && ctx->light_count)
    TC_CUDA(ctx, cudaMemcpyAsync(ctx->lights.ptr, a->h_lights, sizeof(tcb::DevLight) * ctx->light_count,
                                 cudaMemcpyHostToDevice, st));
  if (a->h_attrs)
    TC_CUDA(ctx, cudaMemcpyAsync(ctx->attributes.ptr, a->h_attrs,
                                 sizeof(tc_gpu_triangle_attributes) * ctx->triangle_count, cudaMemcpyHostToDevice, st));
  if (ctx->sphere_count)
    TC_CUDA(ctx, cudaMemcpyAsync(ctx->raw_spheres.ptr, a->h_spheres, sizeof(tc_gpu_sphere) * ctx->sphere_count,
                                 cudaMemcpyHostToDevice, st));
  if (ctx->triangle_count)
    TC_CUDA(ctx, cudaMemcpyAsync(ctx->raw_triangles.ptr, a->h_triangles, sizeof(tc_gpu_triangle) * ctx->triangle_count,
                                 cudaMemcpyHostToDevice, st));
  if (a->rebuild) {
    // The frame's own median-split hierarchy, built on the device into the same buffers.
    if (a->h_attr_flags)
      TC_CUDA(ctx, cudaMemcpyAsync(ctx->attr_flags.ptr, a->h_attr_flags, sizeof(uint32_t) * ctx->triangle_count,
                                   cudaMemcpyHostToDevice, st));
    TC_CUDA(ctx, cudaMemsetAsync(ctx->build_status.ptr, 0, sizeof(uint32_t), st));
    TC_CUDA(ctx, ctx->builder.build(ctx->raw_spheres.as<tc_gpu_sphere>(), ctx->raw_triangles.as<tc_gpu_triangle>(),
                                    a->h_attr_flags ? ctx->attr_flags.as<uint32_t>() : nullptr,
                                    ctx->pairs.as<tcb::PairNode>(), ctx->root_buf.as<tcb::ChildRec>(),
                                    ctx->prims.as<tcb::PrimRecord>(), ctx->build_status.as<uint32_t>(), st));
    TC_CUDA(ctx, cudaMemcpyAsync(a->h_status, ctx->build_status.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  } else {
    tcb::RefitPlan plan;
    plan.nodes = ctx->refit_nodes.as<uint32_t>();
    plan.level_offsets = ctx->refit_levels;
    TC_CUDA(ctx, tcb::launch_refit(plan, ctx->pairs.as<tcb::PairNode>(), ctx->root_buf.as<tcb::ChildRec>(),
                                   ctx->prims.as<tcb::PrimRecord>(), ctx->bvh_prims,
                                   ctx->raw_spheres.as<tc_gpu_sphere>(), ctx->raw_triangles.as<tc_gpu_triangle>(), st));
  }
  const float* cam = a->d_frame.as<float>();
  const uint32_t* fi = reinterpret_cast<const uint32_t*>(cam + 16);
  if (int rc = enqueue_render(ctx, &a->params, a->options, st, false, fi, cam, a->h_counters)) return rc;
  TC_CUDA(ctx, tcb::launch_display_from_sums(ctx->accum.as<double>(), uint32_t(a->npix), 1.0 / double(a->params.samples),
                                             a->exposure, a->d_rgba.as<uint32_t>(), st));
  TC_CUDA(ctx, cudaMemcpyAsync(a->h_rgba, a->d_rgba.ptr, 4 * a->npix, cudaMemcpyDeviceToHost, st));
  return TC_OK;
}

int tc_animation_create(tc_context* ctx, const tc_scene_data* first_frame, const tc_gpu_render_params* params,
                        const tc_render_options* options, float exposure_stops, uint32_t flags,
                        tc_animation** out) {
  if (!ctx) return fail(nullptr, TC_ERR_INVALID, "context is null");
  if (!out || !first_frame) return fail(ctx, TC_ERR_INVALID, "first frame or output pointer is null");
  *out = nullptr;
  if (int rc = check_render_params(ctx, params)) return rc;
  if (!std::isfinite(exposure_stops)) return fail(ctx, TC_ERR_INVALID, "exposure must be finite");
  tc_render_options o{};
  if (options) o = *options;
  if (o.guide_record || o.keep_moments)
    return fail(ctx, TC_ERR_INVALID, "animation frames do not record training samples or keep moments");
  TC_CUDA(ctx, cudaSetDevice(ctx->device));
  auto* a = new tc_animation();
  a->ctx = ctx;
  a->params = *params;
  a->params.accumulated_samples = 0;
  a->options = o;
  a->exposure = exposure_stops;
  a->update_lights = (flags & TC_ANIM_UPDATE_LIGHTS) != 0;
  a->rebuild = (flags & TC_ANIM_REBUILD) != 0;
  a->npix = size_t(params->width) * params->height;
  cudaError_t e = cudaSuccess;
  auto host = [&](void** p, size_t bytes) {
    if (e == cudaSuccess && bytes) e = cudaHostAlloc(p, bytes, cudaHostAllocDefault);
  };
  host(reinterpret_cast<void**>(&a->h_spheres), sizeof(tc_gpu_sphere) * ctx->sphere_count);
  host(reinterpret_cast<void**>(&a->h_triangles), sizeof(tc_gpu_triangle) * ctx->triangle_count);
  host(reinterpret_cast<void**>(&a->h_lights), sizeof(tcb::DevLight) * ctx->light_count);
  if (ctx->any_attr) host(reinterpret_cast<void**>(&a->h_attrs), sizeof(tc_gpu_triangle_attributes) * ctx->triangle_count);
  if (a->rebuild) {
    host(reinterpret_cast<void**>(&a->h_status), sizeof(uint32_t));
    if (ctx->any_attr) host(reinterpret_cast<void**>(&a->h_attr_flags), sizeof(uint32_t) * ctx->triangle_count);
    if (e == cudaSuccess) e = ctx->builder.plan(ctx->sphere_count, ctx->triangle_count);
    if (e == cudaSuccess)
      e = ctx->pairs.reserve(sizeof(tcb::PairNode) * std::max<size_t>(ctx->builder.pair_count(), 1));
    if (e == cudaSuccess) e = ctx->build_status.reserve(sizeof(uint32_t));
    if (e == cudaSuccess && a->h_attr_flags) e = ctx->attr_flags.reserve(sizeof(uint32_t) * ctx->triangle_count);
  }
  host(reinterpret_cast<void**>(&a->h_frame), 20 * sizeof(float));
  host(reinterpret_cast<void**>(&a->h_rgba), 4 * a->npix);
  host(reinterpret_cast<void**>(&a->h_counters), 4 * sizeof(unsigned long long));
  if (e == cudaSuccess) e = a->d_frame.reserve(20 * sizeof(float));
  if (e == cudaSuccess) e = a->d_rgba.reserve(4 * a->npix);
  if (e == cudaSuccess && ctx->sphere_count) e = ctx->raw_spheres.reserve(sizeof(tc_gpu_sphere) * ctx->sphere_count);
  if (e == cudaSuccess && ctx->triangle_count)
    e = ctx->raw_triangles.reserve(sizeof(tc_gpu_triangle) * ctx->triangle_count);
  if (e != cudaSuccess) {
    animation_free(a);
    return cuda_fail(ctx, e, "animation buffers");
  }
  cudaStream_t st = ctx->stream;
  // One direct run sizes every buffer the frame needs; the capture then records the same work.
  int rc = animation_stage(a, first_frame, params->frame_index);
  if (rc == TC_OK) rc = animation_enqueue(a, st);
  if (rc == TC_OK && (e = cudaStreamSynchronize(st)) != cudaSuccess) rc = cuda_fail(ctx, e, "animation warm-up");
  if (rc == TC_OK) {
    ctx->raw_spheres_valid = ctx->raw_triangles_valid = true;
    if ((e = cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed)) != cudaSuccess) {
      rc = cuda_fail(ctx, e, "cudaStreamBeginCapture");
    } else {
      rc = animation_enqueue(a, st);
      cudaGraph_t g = nullptr;
      const cudaError_t e2 = cudaStreamEndCapture(st, &g);
      a->graph = g;
      if (rc == TC_OK && e2 != cudaSuccess) rc = cuda_fail(ctx, e2, "cudaStreamEndCapture");
      if (rc == TC_OK && (e = cudaGraphInstantiate(&a->exec, a->graph, 0)) != cudaSuccess)
        rc = cuda_fail(ctx, e, "cudaGraphInstantiate");
    }
  }
  if (rc != TC_OK) {
    animation_free(a);
    return rc;
  }
  *out = a;
  return TC_OK;
}

int tc_animation_frame(tc_animation* a, const tc_scene_data* frame, uint32_t frame_index, uint8_t* rgba,
                       size_t n_bytes) {
  if (!a) return fail(nullptr, TC_ERR_INVALID, "animation is null");
  tc_context* ctx = a->ctx;
  if (!frame) return fail(ctx, TC_ERR_INVALID, "frame is null");
  if (rgba && n_bytes < 4 * a->npix) return fail(ctx, TC_ERR_INVALID, "output buffer holds fewer than 4*width*height bytes");
  if (int rc = animation_stage(a, frame, frame_index)) return rc;
  TC_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  TC_CUDA(ctx, cudaEventRecord(ctx->ev_begin, st));
  TC_CUDA(ctx, cudaGraphLaunch(a->exec, st));
  TC_CUDA(ctx, cudaEventRecord(ctx->ev_end, st));
  TC_CUDA(ctx, cudaStreamSynchronize(st));
  ctx->width = a->params.width;
  ctx->height = a->params.height;
  ctx->accumulated = a->params.samples;
  if (a->rebuild && *a->h_status)
    return fail(ctx, TC_ERR_DEVICE_STATUS,
                "the frame's centroids coincide in a node of more than four primitives (a degenerate leaf); "
                "animate this scene with refits or upload its frames");
  cudaEventElapsedTime(&ctx->stats.total_ms, ctx->ev_begin, ctx->ev_end);
  clear_phase_stats(ctx->stats);
  ctx->stats.kernel_ms = ctx->stats.total_ms;
  if (int rc = finish_render_stats(ctx, a->h_counters, uint64_t(a->npix) * a->params.samples, false)) return rc;
  if (rgba) std::memcpy(rgba, a->h_rgba, 4 * a->npix);
  return TC_OK;
}

int tc_animation_destroy(tc_animation* a) {
  if (!a) return TC_OK;
  if (a->ctx) {
    cudaSetDevice(a->ctx->device);
    cudaStreamSynchronize(a->ctx->stream);
  }
  animation_free(a);
  return TC_OK;
}

int tc_render_no_alloc(tc_context* ctx, const tc_gpu_render_params* p, double* sums, size_t n_doubles, void* stream) {
  if (!ctx) return fail(nullptr, TC_ERR_INVALID, "context is null");
  if (!p || !sums) return fail(ctx, TC_ERR_INVALID, "render params or sums buffer is null");
  if (!ctx->has_scene) return fail(ctx, TC_ERR_STATE, "tc_render_no_alloc before tc_upload_scene");
  if (ctx->scene.tri_verts) return fail(ctx, TC_ERR_INVALID, "tc_render_no_alloc uses the Moller-Trumbore triangle test");
  if (p->width == 0 || p->height == 0) return fail(ctx, TC_ERR_INVALID, "render dimensions must be nonzero");
  if (p->samples == 0) return fail(ctx, TC_ERR_INVALID, "sample batch must be greater than zero");
  const uint64_t npix = uint64_t(p->width) * p->height;
  if (npix > (1ull << 31)) return fail(ctx, TC_ERR_INVALID, "image is too large: at most 2^31 pixels");
  if (n_doubles < 3 * npix)
    return fail(ctx, TC_ERR_INVALID, "sums buffer holds " + std::to_string(n_doubles) + " doubles; " +
                                         std::to_string(3 * npix) + " (3 per pixel) are needed");
  TC_CUDA(ctx, cudaSetDevice(ctx->device));
  if (!ctx->static_scratch) TC_CUDA(ctx, tcb::render_static_scratch(ctx->device, &ctx->static_scratch));
  unsigned long long* scratch = ctx->static_scratch;
  static_assert(tcb::kStaticScratchWords >= 4, "the render scratch needs 4 words");
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
  if (p->accumulated_samples == 0) TC_CUDA(ctx, cudaMemsetAsync(sums, 0, sizeof(double) * 3 * npix, st));
  TC_CUDA(ctx, cudaMemsetAsync(scratch, 0, 4 * sizeof(unsigned long long), st));
  tcb::RenderLaunch L{};
  L.f.scene = ctx->scene;
  L.f.width = p->width;
  L.f.height = p->height;
  L.f.samples = p->samples;
  L.f.max_bounces = p->max_bounces;
  L.f.frame_index = p->frame_index;
  L.f.sample_base = p->accumulated_samples;
  L.f.samples_per_item = 1u;
  L.f.items_per_pixel = (p->samples + L.f.samples_per_item - 1) / L.f.samples_per_item;
  L.total_items = npix * L.f.items_per_pixel;
  L.f.accum = sums;
  L.f.accum_sq = nullptr;
  L.work_counter = scratch;
  L.counters = scratch + 1;
  L.min_active = kDefaultRefillLanes;
  const int block = 128;
  const int per_sm = tcb::render_max_blocks_per_sm(block, false);
  if (per_sm <= 0) return fail(ctx, TC_ERR_CUDA, "render kernel cannot be resident with this block size");
  // Like tc_render: a frame with fewer work items than the resident grid needs fewer blocks.
  const uint64_t grid = std::max<uint64_t>(
      1, std::min<uint64_t>(uint64_t(per_sm) * ctx->sm_count, (L.total_items + block - 1) / block));
  TC_CUDA(ctx, tcb::launch_render(L, block, int(grid), false, st));
  return TC_OK;
}

int tc_readback(tc_context* ctx, float* rgba, size_t n_floats) {
  if (!ctx) return fail(nullptr, TC_ERR_INVALID, "context is null");
  if (!rgba) return fail(ctx, TC_ERR_INVALID, "output buffer is null");
  if (ctx->accumulated == 0) return fail(ctx, TC_ERR_STATE, "tc_readback before tc_render");
  const size_t npix = size_t(ctx->width) * ctx->height;
  if (n_floats < 4 * npix) return fail(ctx, TC_ERR_INVALID, "output buffer holds fewer than 4*width*height floats");
  TC_CUDA(ctx, cudaSetDevice(ctx->device));
  TC_CUDA(ctx, tcb::launch_resolve(ctx->accum.as<double>(), uint32_t(npix), 1.0 / double(ctx->accumulated),
                                   ctx->image.as<float4>(), ctx->stream));
  TC_CUDA(ctx, cudaMemcpyAsync(rgba, ctx->image.ptr, sizeof(float4) * npix, cudaMemcpyDeviceToHost, ctx->stream));
  TC_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return TC_OK;
}

int tc_display_rgba8_async(tc_context* ctx, float exposure_stops, void* d_rgba, size_t n_bytes, void* stream) {
  if (!ctx) return fail(nullptr, TC_ERR_INVALID, "context is null");
  if (!d_rgba) return fail(ctx, TC_ERR_INVALID, "output buffer is null");
  if (ctx->accumulated == 0) return fail(ctx, TC_ERR_STATE, "display conversion before tc_render");
  if (!std::isfinite(exposure_stops)) return fail(ctx, TC_ERR_INVALID, "exposure must be finite");
  const size_t npix = size_t(ctx->width) * ctx->height;
  if (n_bytes < 4 * npix) return fail(ctx, TC_ERR_INVALID, "output buffer holds fewer than 4*width*height bytes");
  TC_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
  TC_CUDA(ctx, tcb::launch_display_from_sums(ctx->accum.as<double>(), uint32_t(npix), 1.0 / double(ctx->accumulated),
                                             exposure_stops, static_cast<uint32_t*>(d_rgba), st));
  return TC_OK;
}

int tc_readback_rgba8(tc_context* ctx, float exposure_stops, uint8_t* rgba, size_t n_bytes) {
  if (!ctx) return fail(nullptr, TC_ERR_INVALID, "context is null");
  if (!rgba) return fail(ctx, TC_ERR_INVALID, "output buffer is null");
  if (ctx->accumulated == 0) return fail(ctx, TC_ERR_STATE, "tc_readback_rgba8 before tc_render");
  const size_t npix = size_t(ctx->width) * ctx->height;
  if (n_bytes < 4 * npix) return fail(ctx, TC_ERR_INVALID, "output buffer holds fewer than 4*width*height bytes");
  TC_CUDA(ctx, cudaSetDevice(ctx->device));
  TC_CUDA(ctx, ctx->display.reserve(4 * npix));
  if (int rc = tc_display_rgba8_async(ctx, exposure_stops, ctx->display.ptr, 4 * npix, nullptr)) return rc;
  TC_CUDA(ctx, cudaMemcpyAsync(rgba, ctx->display.ptr, 4 * npix, cudaMemcpyDeviceToHost, ctx->stream));
  TC_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return TC_OK;
}

int tc_encode_jpeg(tc_context* ctx, uint32_t quality, float exposure_stops, uint8_t* out, size_t capacity,
                   size_t* length) {
  if (!ctx) return fail(nullptr, TC_ERR_INVALID, "context is null");
  if (!length) return fail(ctx, TC_ERR_INVALID, "length pointer is null");
  if (quality < 1 || quality > 100) return fail(ctx, TC_ERR_INVALID, "JPEG quality must be between 1 and 100");
  if (ctx->accumulated == 0) return fail(ctx, TC_ERR_STATE, "tc_encode_jpeg before tc_render");
  if (!std::isfinite(exposure_stops)) return fail(ctx, TC_ERR_INVALID, "exposure must be finite");
  TC_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  auto jpeg_fail = [&](nvjpegStatus_t status, const char* what) {
    return fail(ctx, TC_ERR_CUDA, std::string(what) + " failed with nvJPEG status " + std::to_string(int(status)));
  };
  nvjpegStatus_t js;
  if (!ctx->jpeg) {
    if ((js = nvjpegCreateSimple(&ctx->jpeg)) != NVJPEG_STATUS_SUCCESS) {
      ctx->jpeg = nullptr;
      return jpeg_fail(js, "nvjpegCreateSimple");
    }
    if ((js = nvjpegEncoderStateCreate(ctx->jpeg, &ctx->jpeg_state, st)) != NVJPEG_STATUS_SUCCESS)
      return jpeg_fail(js, "nvjpegEncoderStateCreate");
    if ((js = nvjpegEncoderParamsCreate(ctx->jpeg, &ctx->jpeg_params, st)) != NVJPEG_STATUS_SUCCESS)
      return jpeg_fail(js, "nvjpegEncoderParamsCreate");
  }
  if ((js = nvjpegEncoderParamsSetQuality(ctx->jpeg_params, int(quality), st)) != NVJPEG_STATUS_SUCCESS)
    return jpeg_fail(js, "nvjpegEncoderParamsSetQuality");
  if ((js = nvjpegEncoderParamsSetSamplingFactors(ctx->jpeg_params, NVJPEG_CSS_420, st)) != NVJPEG_STATUS_SUCCESS)
    return jpeg_fail(js, "nvjpegEncoderParamsSetSamplingFactors");
  const size_t npix = size_t(ctx->width) * ctx->height;
  TC_CUDA(ctx, ctx->jpeg_rgb.reserve(3 * npix));
  TC_CUDA(ctx, tcb::launch_display_rgb8_from_sums(ctx->accum.as<double>(), uint32_t(npix), 1.0 / double(ctx->accumulated),
                                                  exposure_stops, ctx->jpeg_rgb.as<uint8_t>(), st));
  nvjpegImage_t img{};
  img.channel[0] = ctx->jpeg_rgb.as<unsigned char>();
  img.pitch[0] = 3 * size_t(ctx->width);
  if ((js = nvjpegEncodeImage(ctx->jpeg, ctx->jpeg_state, ctx->jpeg_params, &img, NVJPEG_INPUT_RGBI, int(ctx->width),
                              int(ctx->height), st)) != NVJPEG_STATUS_SUCCESS)
    return jpeg_fail(js, "nvjpegEncodeImage");
  TC_CUDA(ctx, cudaStreamSynchronize(st));
  size_t len = 0;
  if ((js = nvjpegEncodeRetrieveBitstream(ctx->jpeg, ctx->jpeg_state, nullptr, &len, st)) != NVJPEG_STATUS_SUCCESS)
    return jpeg_fail(js, "nvjpegEncodeRetrieveBitstream");
  *length = len;
  if (!out) return TC_OK;
  if (capacity < len)
    return fail(ctx, TC_ERR_INVALID, "output buffer holds " + std::to_string(capacity) + " bytes; the frame needs " +
                                         std::to_string(len));
  if ((js = nvjpegEncodeRetrieveBitstream(ctx->jpeg, ctx->jpeg_state, out, &len, st)) != NVJPEG_STATUS_SUCCESS)
    return jpeg_fail(js, "nvjpegEncodeRetrieveBitstream");
  TC_CUDA(ctx, cudaStreamSynchronize(st));
  *length = len;
  return TC_OK;
}

int tc_readback_sums(tc_context* ctx, double* sum, double* sum_sq, size_t n_doubles, uint32_t* samples) {
  if (!ctx) return fail(nullptr, TC_ERR_INVALID, "context is null");
  if (ctx->accumulated == 0) return fail(ctx, TC_ERR_STATE, "tc_readback_sums before tc_render");
  const size_t n = size_t(3) * ctx->width * ctx->height;
  if ((sum || sum_sq) && n_doubles < n) return fail(ctx, TC_ERR_INVALID, "buffer holds fewer than 3*width*height doubles");
  if (sum_sq && !ctx->has_moments) return fail(ctx, TC_ERR_STATE, "moments were not kept for this accumulation");
  TC_CUDA(ctx, cudaSetDevice(ctx->device));
  if (sum) TC_CUDA(ctx, cudaMemcpyAsync(sum, ctx->accum.ptr, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
  if (sum_sq)
    TC_CUDA(ctx, cudaMemcpyAsync(sum_sq, ctx->accum_sq.ptr, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
  TC_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (samples) *samples = ctx->accumulated;
  return TC_OK;
}

int tc_trace_closest_device_async(tc_context* ctx, const float* d_rays, size_t n, float tmin, uint32_t* d_prim,
                                  float* d_t, void* stream) {
  if (!ctx) return fail(nullptr, TC_ERR_INVALID, "context is null");
  if (!ctx->has_scene) return fail(ctx, TC_ERR_STATE, "trace before tc_upload_scene");
  if (n && (!d_rays || !d_prim || !d_t)) return fail(ctx, TC_ERR_INVALID, "ray or output pointer is null");
  TC_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
  TC_CUDA(ctx, tcb::launch_trace_closest(ctx->scene, d_rays, n, tmin, d_prim, d_t, st));
  return TC_OK;
}

int tc_trace_closest(tc_context* ctx, const float* rays, size_t n, float tmin, uint32_t* prim, float* t) {
  if (!ctx) return fail(nullptr, TC_ERR_INVALID, "context is null");
  if (!ctx->has_scene) return fail(ctx, TC_ERR_STATE, "trace before tc_upload_scene");
  if (n == 0) return TC_OK;
  if (!rays || !prim || !t) return fail(ctx, TC_ERR_INVALID, "ray or output pointer is null");
  TC_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  TC_CUDA(ctx, ctx->ray_buf.reserve(sizeof(float) * 6 * n));
  TC_CUDA(ctx, ctx->prim_buf.reserve(sizeof(uint32_t) * n));
  TC_CUDA(ctx, ctx->t_buf.reserve(sizeof(float) * n));
  TC_CUDA(ctx, cudaEventRecord(ctx->ev_begin, st));
  TC_CUDA(ctx, cudaMemcpyAsync(ctx->ray_buf.ptr, rays, sizeof(float) * 6 * n, cudaMemcpyHostToDevice, st));
  TC_CUDA(ctx, cudaEventRecord(ctx->ev_kernel0, st));
  TC_CUDA(ctx, tcb::launch_trace_closest(ctx->scene, ctx->ray_buf.as<float>(), n, tmin, ctx->prim_buf.as<uint32_t>(),
                                         ctx->t_buf.as<float>(), st));
  TC_CUDA(ctx, cudaEventRecord(ctx->ev_kernel1, st));
  TC_CUDA(ctx, cudaMemcpyAsync(prim, ctx->prim_buf.ptr, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, st));
  TC_CUDA(ctx, cudaMemcpyAsync(t, ctx->t_buf.ptr, sizeof(float) * n, cudaMemcpyDeviceToHost, st));
  TC_CUDA(ctx, cudaEventRecord(ctx->ev_end, st));
  TC_CUDA(ctx, cudaStreamSynchronize(st));
  clear_phase_stats(ctx->stats);
  cudaEventElapsedTime(&ctx->stats.kernel_ms, ctx->ev_kernel0, ctx->ev_kernel1);
  cudaEventElapsedTime(&ctx->stats.total_ms, ctx->ev_begin, ctx->ev_end);
  ctx->stats.rays = n;
  ctx->stats.extension_rays = n;
  ctx->stats.shadow_rays = 0;
  ctx->stats.paths = 0;
  return TC_OK;
}

namespace {

int guide_alloc(tc_context* ctx) {
  if (ctx->has_guide) return TC_OK;
  TC_CUDA(ctx, ctx->g_params.reserve(sizeof(float) * tcb::kGuideParams));
  TC_CUDA(ctx, ctx->g_m.reserve(sizeof(float) * tcb::kGuideParams));
  TC_CUDA(ctx, ctx->g_v.reserve(sizeof(float) * tcb::kGuideParams));
  TC_CUDA(ctx, ctx->g_grad.reserve(sizeof(float) * (tcb::kGuideParams + 1)));
  TC_CUDA(ctx, ctx->g_images.reserve(tcb::kImgBytes));
  TC_CUDA(ctx, ctx->g_biases.reserve(sizeof(float) * 224));
  TC_CUDA(ctx, ctx->g_status.reserve(sizeof(int)));
  ctx->guide.params = ctx->g_params.as<float>();
  ctx->guide.adam_m = ctx->g_m.as<float>();
  ctx->guide.adam_v = ctx->g_v.as<float>();
  ctx->guide.grad = ctx->g_grad.as<float>();
  ctx->guide.images = ctx->g_images.as<uint8_t>();
  ctx->guide.biases = ctx->g_biases.as<float>();
  ctx->guide.status = ctx->g_status.as<int>();
  ctx->has_guide = true;
  return TC_OK;
}

int guide_check_status(tc_context* ctx) {
  int status = 0;
  TC_CUDA(ctx, cudaMemcpyAsync(&status, ctx->guide.status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  TC_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (status) {
    cudaMemsetAsync(ctx->guide.status, 0, sizeof(int), ctx->stream);
    return fail(ctx, TC_ERR_DEVICE_STATUS, "a guiding kernel gave up waiting for its tensor-core work");
  }
  return TC_OK;
}

// Samples as 3 float4 per sample (position + weight, normal, direction).
void pack_samples(const float* s, size_t n, std::vector<float>& out) {
  out.assign(n * 12, 0.0f);
  for (size_t i = 0; i < n; ++i) {
    const float* r = s + 10 * i;
    float* o = out.data() + 12 * i;
    o[0] = r[0]; o[1] = r[1]; o[2] = r[2]; o[3] = r[9];
    o[4] = r[3]; o[5] = r[4]; o[6] = r[5];
    o[8] = r[6]; o[9] = r[7]; o[10] = r[8];
  }
}

}  // namespace

int tc_guide_set_params(tc_context* ctx, const float* params, const float* bounds) {
  if (!ctx) return fail(nullptr, TC_ERR_INVALID, "context is null");
  if (!params || !bounds) return fail(ctx, TC_ERR_INVALID, "params or bounds is null");
  if (!(bounds[3] > 0.0f) || !std::isfinite(bounds[3])) return fail(ctx, TC_ERR_INVALID, "bounds scale must be positive");
  TC_CUDA(ctx, cudaSetDevice(ctx->device));
  int rc = guide_alloc(ctx);
  if (rc != TC_OK) return rc;
  cudaStream_t st = ctx->stream;
  TC_CUDA(ctx, cudaMemcpyAsync(ctx->guide.params, params, sizeof(float) * tcb::kGuideParams, cudaMemcpyHostToDevice, st));
  TC_CUDA(ctx, cudaMemsetAsync(ctx->guide.adam_m, 0, sizeof(float) * tcb::kGuideParams, st));
  TC_CUDA(ctx, cudaMemsetAsync(ctx->guide.adam_v, 0, sizeof(float) * tcb::kGuideParams, st));
  TC_CUDA(ctx, cudaMemsetAsync(ctx->guide.grad, 0, sizeof(float) * (tcb::kGuideParams + 1), st));
  TC_CUDA(ctx, cudaMemsetAsync(ctx->guide.status, 0, sizeof(int), st));
  ctx->guide.bounds = tcb::GuideBounds{bounds[0], bounds[1], bounds[2], bounds[3]};
  ctx->guide.adam_step = 0;
  TC_CUDA(ctx, tcb::guide_refresh_images(ctx->guide, st));
  TC_CUDA(ctx, cudaStreamSynchronize(st));
  return TC_OK;
}

int tc_guide_get_params(tc_context* ctx, float* params) {
  if (!ctx || !params) return fail(ctx, TC_ERR_INVALID, "context or output is null");
  if (!ctx->has_guide) return fail(ctx, TC_ERR_STATE, "guiding parameters were never set");
  TC_CUDA(ctx, cudaSetDevice(ctx->device));
  TC_CUDA(ctx, cudaMemcpyAsync(params, ctx->guide.params, sizeof(float) * tcb::kGuideParams, cudaMemcpyDeviceToHost,
                               ctx->stream));
  TC_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return TC_OK;
}

int tc_guide_infer(tc_context* ctx, const float* queries, size_t n, float* out) {
  if (!ctx) return fail(nullptr, TC_ERR_INVALID, "context is null");
  if (!ctx->has_guide) return fail(ctx, TC_ERR_STATE, "guiding parameters were never set");
  if (n == 0) return TC_OK;
  if (!queries || !out) return fail(ctx, TC_ERR_INVALID, "query or output pointer is null");
  TC_CUDA(ctx, cudaSetDevice(ctx->device));
  std::vector<float> q(n * 8, 0.0f);
  for (size_t i = 0; i < n; ++i)
    for (int c = 0; c < 3; ++c) {
      q[8 * i + c] = queries[6 * i + c];
      q[8 * i + 4 + c] = queries[6 * i + 3 + c];
    }
  cudaStream_t st = ctx->stream;
  TC_CUDA(ctx, ctx->g_in.reserve(sizeof(float) * q.size()));
  TC_CUDA(ctx, ctx->g_out.reserve(sizeof(float4) * tcb::kGuideDecodedF4 * n));
  TC_CUDA(ctx, cudaMemcpyAsync(ctx->g_in.ptr, q.data(), sizeof(float) * q.size(), cudaMemcpyHostToDevice, st));
  TC_CUDA(ctx, cudaEventRecord(ctx->ev_kernel0, st));
  TC_CUDA(ctx, tcb::guide_launch_infer(ctx->guide, ctx->g_in.as<float4>(), uint32_t(n), ctx->g_out.as<float4>(),
                                       ctx->sm_count, st));
  TC_CUDA(ctx, cudaEventRecord(ctx->ev_kernel1, st));
  TC_CUDA(ctx, cudaMemcpyAsync(out, ctx->g_out.ptr, sizeof(float4) * tcb::kGuideDecodedF4 * n, cudaMemcpyDeviceToHost, st));
  int rc = guide_check_status(ctx);
  clear_phase_stats(ctx->stats);
  cudaEventElapsedTime(&ctx->stats.kernel_ms, ctx->ev_kernel0, ctx->ev_kernel1);
  return rc;
}

int tc_guide_loss_grad(tc_context* ctx, const float* samples, size_t n, float* grad, float* loss) {
  if (!ctx) return fail(nullptr, TC_ERR_INVALID, "context is null");
  if (!ctx->has_guide) return fail(ctx, TC_ERR_STATE, "guiding parameters were never set");
  if (n == 0 || !samples) return fail(ctx, TC_ERR_INVALID, "no samples");
  TC_CUDA(ctx, cudaSetDevice(ctx->device));
  std::vector<float> packed;
  pack_samples(samples, n, packed);
  cudaStream_t st = ctx->stream;
  TC_CUDA(ctx, ctx->g_in.reserve(sizeof(float) * packed.size()));
  TC_CUDA(ctx, cudaMemcpyAsync(ctx->g_in.ptr, packed.data(), sizeof(float) * packed.size(), cudaMemcpyHostToDevice, st));
  TC_CUDA(ctx, cudaMemsetAsync(ctx->guide.grad, 0, sizeof(float) * (tcb::kGuideParams + 1), st));
  TC_CUDA(ctx, cudaEventRecord(ctx->ev_kernel0, st));
  TC_CUDA(ctx, tcb::guide_launch_loss_grad(ctx->guide, ctx->g_in.as<float4>(), uint32_t(n), 1.0f / float(n),
                                           ctx->sm_count, st));
  TC_CUDA(ctx, cudaEventRecord(ctx->ev_kernel1, st));
  std::vector<float> g(tcb::kGuideParams + 1);
  TC_CUDA(ctx, cudaMemcpyAsync(g.data(), ctx->guide.grad, sizeof(float) * g.size(), cudaMemcpyDeviceToHost, st));
  int rc = guide_check_status(ctx);
  clear_phase_stats(ctx->stats);
  cudaEventElapsedTime(&ctx->stats.kernel_ms, ctx->ev_kernel0, ctx->ev_kernel1);
  if (rc != TC_OK) return rc;
  if (grad) std::memcpy(grad, g.data(), sizeof(float) * tcb::kGuideParams);
  if (loss) *loss = g[tcb::kGuideParams];
  return TC_OK;
}

int tc_guide_adam_step(tc_context* ctx, float lr) {
  if (!ctx) return fail(nullptr, TC_ERR_INVALID, "context is null");
  if (!ctx->has_guide) return fail(ctx, TC_ERR_STATE, "guiding parameters were never set");
  TC_CUDA(ctx, cudaSetDevice(ctx->device));
  TC_CUDA(ctx, tcb::guide_launch_adam(ctx->guide, lr, ctx->stream));
  TC_CUDA(ctx, cudaMemsetAsync(ctx->guide.grad + tcb::kGuideParams, 0, sizeof(float), ctx->stream));
  TC_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return TC_OK;
}

int tc_guide_train(tc_context* ctx, const float* samples, size_t n, uint32_t steps, uint32_t batch, float lr,
                   uint64_t seed, float* losses) {
  if (!ctx) return fail(nullptr, TC_ERR_INVALID, "context is null");
  if (!ctx->has_guide) return fail(ctx, TC_ERR_STATE, "guiding parameters were never set");
  if (n == 0 || !samples || batch == 0) return fail(ctx, TC_ERR_INVALID, "no samples or zero batch");
  TC_CUDA(ctx, cudaSetDevice(ctx->device));
  // Seeded shuffle (SplitMix64-driven Fisher-Yates), then consecutive batches.
  std::vector<uint32_t> order(n);
  for (size_t i = 0; i < n; ++i) order[i] = uint32_t(i);
  uint64_t x = seed;
  auto next = [&x]() {
    uint64_t z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  };
  for (size_t i = n - 1; i > 0; --i) std::swap(order[i], order[size_t(next() % (i + 1))]);
  std::vector<float> shuffled(n * 10);
  for (size_t i = 0; i < n; ++i) std::memcpy(&shuffled[10 * i], samples + 10 * size_t(order[i]), 40);
  std::vector<float> packed;
  pack_samples(shuffled.data(), n, packed);
  cudaStream_t st = ctx->stream;
  TC_CUDA(ctx, ctx->g_in.reserve(sizeof(float) * packed.size()));
  TC_CUDA(ctx, cudaMemcpyAsync(ctx->g_in.ptr, packed.data(), sizeof(float) * packed.size(), cudaMemcpyHostToDevice, st));
  const uint32_t b = uint32_t(std::min<size_t>(batch, n));
  std::vector<float> step_loss(steps, 0.0f);
  TC_CUDA(ctx, ctx->g_out.reserve(sizeof(float) * std::max<uint32_t>(steps, 1)));
  TC_CUDA(ctx, cudaEventRecord(ctx->ev_kernel0, st));
  size_t cursor = 0;
  for (uint32_t s = 0; s < steps; ++s) {
    if (cursor + b > n) cursor = 0;
    TC_CUDA(ctx, tcb::guide_launch_loss_grad(ctx->guide, ctx->g_in.as<float4>() + 3 * cursor, b, 1.0f / float(b),
                                             ctx->sm_count, st));
    TC_CUDA(ctx, cudaMemcpyAsync(ctx->g_out.as<float>() + s, ctx->guide.grad + tcb::kGuideParams, sizeof(float),
                                 cudaMemcpyDeviceToDevice, st));
    TC_CUDA(ctx, cudaMemsetAsync(ctx->guide.grad + tcb::kGuideParams, 0, sizeof(float), st));
    TC_CUDA(ctx, tcb::guide_launch_adam(ctx->guide, lr, st));
    cursor += b;
  }
  TC_CUDA(ctx, cudaEventRecord(ctx->ev_kernel1, st));
  if (steps) TC_CUDA(ctx, cudaMemcpyAsync(step_loss.data(), ctx->g_out.ptr, sizeof(float) * steps, cudaMemcpyDeviceToHost, st));
  int rc = guide_check_status(ctx);
  clear_phase_stats(ctx->stats);
  cudaEventElapsedTime(&ctx->stats.kernel_ms, ctx->ev_kernel0, ctx->ev_kernel1);
  if (rc != TC_OK) return rc;
  if (losses) std::memcpy(losses, step_loss.data(), sizeof(float) * steps);
  return TC_OK;
}

// Positive-weight training samples of the last recorded batch into rec_samples; their number and
// weight sum come back to the host.
// Appends the positive-weight training samples of the batch just recorded to the sample pool
// (`fresh`: empties the pool first). Enqueued on `st` after the batch; no host synchronisation.
static int append_training_samples(tc_context* ctx, bool fresh, cudaStream_t st) {
  TC_CUDA(ctx, ctx->rec_samples.reserve(sizeof(float4) * 3 * size_t(kGuidePoolSamples)));
  TC_CUDA(ctx, ctx->rec_wsum.reserve(2 * sizeof(uint32_t)));
  if (fresh || !ctx->has_records) TC_CUDA(ctx, cudaMemsetAsync(ctx->rec_wsum.ptr, 0, 2 * sizeof(uint32_t), st));
  float* d_wsum = ctx->rec_wsum.as<float>();
  uint32_t* d_count = reinterpret_cast<uint32_t*>(d_wsum + 1);
  TC_CUDA(ctx, tcb::launch_guide_samples(ctx->rec_records.as<float4>(), ctx->rec_count.as<uint32_t>(), ctx->rec_capacity,
                                         ctx->rec_path_rad.as<float4>(), ctx->rec_samples.as<float4>(),
                                         kGuidePoolSamples, d_count, d_wsum, st));
  return TC_OK;
}

// Number of samples in the pool and the sum of their weights (waits for the stream).
static int pool_counts(tc_context* ctx, uint32_t* count, float* wsum) {
  cudaStream_t st = ctx->stream;
  uint32_t host[2] = {0, 0};
  TC_CUDA(ctx, cudaMemcpyAsync(host, ctx->rec_wsum.ptr, sizeof(host), cudaMemcpyDeviceToHost, st));
  TC_CUDA(ctx, cudaStreamSynchronize(st));
  std::memcpy(wsum, &host[0], sizeof(float));
  *count = std::min(host[1], kGuidePoolSamples);
  return TC_OK;
}

int tc_guide_train_recorded(tc_context* ctx, uint32_t steps, uint32_t batch, float lr, uint64_t seed, float* losses,
                            uint32_t* n_samples) {
  if (!ctx) return fail(nullptr, TC_ERR_INVALID, "context is null");
  if (!ctx->has_guide) return fail(ctx, TC_ERR_STATE, "guiding parameters were never set");
  if (!ctx->has_records) return fail(ctx, TC_ERR_STATE, "no batch was rendered with guide_record = 1");
  if (batch == 0) return fail(ctx, TC_ERR_INVALID, "batch must be positive");
  TC_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  TC_CUDA(ctx, cudaEventRecord(ctx->ev_kernel0, st));
  uint32_t count = 0;
  float wsum = 0.0f;
  if (int rc = pool_counts(ctx, &count, &wsum)) return rc;
  if (n_samples) *n_samples = count;
  if (count == 0 || !(wsum > 0.0f)) return fail(ctx, TC_ERR_STATE, "the recorded batch carries no radiance to learn from");
  const float mean = wsum / float(count);
  const uint32_t b = std::min(batch, count);
  TC_CUDA(ctx, ctx->g_out.reserve(sizeof(float) * std::max<uint32_t>(steps, 1)));
  uint64_t x = seed;
  for (uint32_t s = 0; s < steps; ++s) {
    x += 0x9E3779B97F4A7C15ull;
    uint64_t z = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    const uint32_t gather = uint32_t(z ^ (z >> 31)) | 1u;
    TC_CUDA(ctx, tcb::guide_launch_loss_grad(ctx->guide, ctx->rec_samples.as<float4>(), b, 1.0f / float(b),
                                             ctx->sm_count, st, 1.0f / mean, 50.0f, gather, count));
    TC_CUDA(ctx, cudaMemcpyAsync(ctx->g_out.as<float>() + s, ctx->guide.grad + tcb::kGuideParams, sizeof(float),
                                 cudaMemcpyDeviceToDevice, st));
    TC_CUDA(ctx, cudaMemsetAsync(ctx->guide.grad + tcb::kGuideParams, 0, sizeof(float), st));
    TC_CUDA(ctx, tcb::guide_launch_adam(ctx->guide, lr, st));
  }
  TC_CUDA(ctx, cudaEventRecord(ctx->ev_kernel1, st));
  std::vector<float> step_loss(steps);
  if (steps) TC_CUDA(ctx, cudaMemcpyAsync(step_loss.data(), ctx->g_out.ptr, sizeof(float) * steps, cudaMemcpyDeviceToHost, st));
  int rc = guide_check_status(ctx);
  clear_phase_stats(ctx->stats);
  cudaEventElapsedTime(&ctx->stats.kernel_ms, ctx->ev_kernel0, ctx->ev_kernel1);
  if (rc != TC_OK) return rc;
  if (losses && steps) std::memcpy(losses, step_loss.data(), sizeof(float) * steps);
  return TC_OK;
}

int tc_guide_recorded_samples(tc_context* ctx, float* out, size_t n_floats, uint32_t* count) {
  if (!ctx) return fail(nullptr, TC_ERR_INVALID, "context is null");
  if (!ctx->has_records) return fail(ctx, TC_ERR_STATE, "no batch was rendered with guide_record = 1");
  TC_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  uint32_t n = 0;
  float wsum = 0.0f;
  if (int rc = pool_counts(ctx, &n, &wsum)) return rc;
  if (count) *count = n;
  if (out) {
    const size_t m = std::min<size_t>(n_floats / 12, n);
    TC_CUDA(ctx, cudaMemcpyAsync(out, ctx->rec_samples.ptr, sizeof(float4) * 3 * m, cudaMemcpyDeviceToHost, st));
    TC_CUDA(ctx, cudaStreamSynchronize(st));
  }
  return TC_OK;
}

int tc_get_stats(const tc_context* ctx, tc_stats* out) {
  if (!ctx || !out) return fail(nullptr, TC_ERR_INVALID, "context or output is null");
  *out = ctx->stats;
  return TC_OK;
}

long tc_build_bvh_host(const tc_gpu_sphere* spheres, size_t n_spheres, const tc_gpu_triangle* triangles,
                       size_t n_triangles, tc_gpu_bvh_node* nodes, size_t node_capacity, tc_gpu_primitive_ref* prims,
                       size_t prim_capacity) {
  if ((n_spheres && !spheres) || (n_triangles && !triangles))
    return fail(nullptr, TC_ERR_INVALID, "geometry pointer is null for a nonzero count");
  std::vector<tcb::SphereIn> sph(n_spheres);
  for (size_t i = 0; i < n_spheres; ++i)
    sph[i] = tcb::SphereIn{{spheres[i].center_radius[0], spheres[i].center_radius[1], spheres[i].center_radius[2]},
                           spheres[i].center_radius[3]};
  std::vector<tcb::TriangleIn> tri(n_triangles);
  for (size_t i = 0; i < n_triangles; ++i)
    for (int c = 0; c < 3; ++c) {
      tri[i].v[0][c] = triangles[i].v0[c];
      tri[i].v[1][c] = triangles[i].v1[c];
      tri[i].v[2][c] = triangles[i].v2[c];
    }
  tcb::FlatHierarchy flat = tcb::build_median_split(sph.data(), sph.size(), tri.data(), tri.size());
  if (flat.nodes.size() > node_capacity || flat.prims.size() > prim_capacity)
    return fail(nullptr, TC_ERR_INVALID, "output capacity is too small for the hierarchy");
  if ((!nodes && !flat.nodes.empty()) || (!prims && !flat.prims.empty()))
    return fail(nullptr, TC_ERR_INVALID, "output pointer is null");
  for (size_t i = 0; i < flat.nodes.size(); ++i) {
    tc_gpu_bvh_node& o = nodes[i];
    std::memset(&o, 0, sizeof(o));
    for (int c = 0; c < 3; ++c) {
      o.min[c] = flat.nodes[i].min[c];
      o.max[c] = flat.nodes[i].max[c];
    }
    o.first_or_right = flat.nodes[i].first_or_right;
    o.primitive_count = flat.nodes[i].count;
  }
  for (size_t i = 0; i < flat.prims.size(); ++i) prims[i] = tc_gpu_primitive_ref{flat.prims[i].kind, flat.prims[i].index};
  return long(flat.nodes.size());
}

}  // extern "C"
