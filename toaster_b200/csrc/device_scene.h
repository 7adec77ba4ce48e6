// Kernel-facing view of one uploaded scene and the launch interface between the host runtime
// (api.cu) and the kernels (kernels.cu).
#ifndef TOASTER_B200_DEVICE_SCENE_H
#define TOASTER_B200_DEVICE_SCENE_H

#include <cuda_runtime.h>
#include <stdint.h>

#include "layout.h"

namespace tcb {

struct DevScene {
  const PairNode* pairs;
  const PrimRecord* prims;
  const ChildRec* root;  // device memory: the root's bounds and link
  const DevMaterial* materials;
  uint32_t material_count;
  uint32_t light_count;
  const DevLight* lights;
  const float4* attributes;  // GpuTriangleAttributes as 5 float4 per triangle, or null
  const uint32_t* texels;    // packed RGBA8 texture atlas, or null
  // Environment (lat-long): RGB texels, marginal row CDF (H), conditional row CDFs (W*H) and the
  // per-texel solid-angle density numerator p(x,y)*W*H/(2*pi^2) (W*H), all FP32 built from FP64
  // prefix sums.
  const float4* env_rgb;
  const uint2* env_alias_marg;   // alias table over rows (env_height entries)
  const uint2* env_alias_cond;   // per row, alias table over its columns (env_width entries each)
  const float* env_pdf;
  uint32_t env_width, env_height;
  float env_intensity;
  float env_rotation_turns;  // rotation_degrees / 360
  uint32_t env_sampleable;   // 1 when the importance distribution has positive mass
  uint32_t background;       // 0 sky, 1 black, 2 environment
  float cam_origin[3], cam_lower_left[3], cam_horizontal[3], cam_vertical[3];
  // Watertight triangle test (tc_set_triangle_test): the vertices of every leaf-order primitive
  // record (3 float4, triangles only), or null for the reference's Moller-Trumbore test.
  const float4* tri_verts;
};

// Training-data recording and guided wavefront rounds (render modes kRecord / kGuided).
struct GuideLaunch {
  // Recording: one 4-float4 record per diffuse scatter (position + path id, normal + T'.x,
  // direction + T'.y, radiance so far + T'.z) and the final radiance of every path.
  float4* records;
  uint32_t* record_count;
  uint32_t record_capacity;
  float4* path_radiance;
  // Guided rounds: paths suspended at a diffuse vertex (6 float4 each) with their decoded
  // mixtures (10 float4 each); this round's suspensions go to out_state / out_query.
  const float4* in_state;
  const uint32_t* in_count;
  const float4* in_mix;
  float4* out_state;
  float4* out_query;
  uint32_t* out_count;
  uint32_t capacity;
  uint32_t resume;         // 0: start the wave's camera paths, 1: resume in_state
  uint32_t wave_first_sample;
  uint32_t wave_spp;
  float guide_fraction;    // probability of sampling the guide's mixture at a diffuse vertex
  // Batched guided rounds: suspended paths per frame (n counters) and, when resuming, the
  // exclusive prefix of the previous round's per-frame counts (n + 1 entries, the total last).
  uint32_t* job_out_count;
  const uint32_t* in_job_prefix;
};

// Path kernel modes.
enum RenderMode : int { kModePlain = 0, kModeRecord = 1, kModeGuided = 2 };

// One independent frame: its scene, image and sample range. A single-frame launch carries it
// inline (RenderLaunch::f); a batched launch reads one per job from device memory.
struct FrameJob {
  DevScene scene;
  double* accum;               // 3 doubles per pixel (running sums)
  double* accum_sq;            // 3 doubles per pixel or null
  uint64_t item_begin;         // batched launches: first global work item of this frame
  uint32_t width, height, samples, max_bounces;
  uint32_t frame_index;
  uint32_t sample_base;        // samples already accumulated (decorrelates progressive batches)
  uint32_t samples_per_item;   // samples a lane traces for one pixel before fetching new work
  uint32_t items_per_pixel;
  // Replayed frames (CUDA graphs): when set, the frame index and the camera (origin, lower-left
  // corner, horizontal, vertical; 4 floats each) are read from device memory at run time instead
  // of the values above, so one captured launch serves every frame.
  const uint32_t* frame_index_dev;
  const float* camera_dev;
  // Batched guided launches: first pixel of this frame in the concatenation of all frames' pixels,
  // and the frame's region (offset, capacity) in the wave's suspended-path buffers.
  uint32_t pix_begin;
  uint32_t wave_offset, wave_capacity;
};

struct RenderLaunch {
  FrameJob f;                  // the frame of a single-frame launch
  const FrameJob* jobs;        // batched launch: job_count frames in device memory (else null)
  uint32_t job_count;
  uint64_t total_items;
  unsigned long long* work_counter;
  unsigned long long* counters;  // [0] paths, [1] extension rays, [2] shadow rays
  int short_stack;               // traversal stack entries per thread kept in shared memory
  int min_active;                // a warp pauses traversal for refills below this many busy lanes
  GuideLaunch g;
};

// Wavefront schedule of plain renders: every path in flight owns a slot of per-path state in
// device memory, and each iteration runs three launches over it:
//   logic   per slot: adds the shadow-ray results of the last vertex, consumes the last
//           extension hit (miss -> environment, emissive -> emission, else the slot joins the
//           queue of its material), finishes paths into the FP64 image sums and starts new
//           camera paths in free slots (their rays join the extension queue);
//   shade   per material queue (diffuse, then metal, then dielectric, so a warp shades one
//           material): next-event shadow rays and the scattered extension ray;
//   trace   extension rays (closest hit) then shadow rays (first hit), 32 rays of one kind per
//           warp; a shadow ray that hits something zeroes its contribution.
// State word per slot: bits 0-23 remaining depth, then the flags below.
constexpr uint32_t kWfDepthMask = 0x00FFFFFFu;
constexpr uint32_t kWfAlive = 1u << 24;          // the slot holds a path
constexpr uint32_t kWfExtPending = 1u << 25;     // its extension ray is queued / traced
constexpr uint32_t kWfNeePending = 1u << 26;     // its two shadow-ray contributions are to be added
constexpr uint32_t kWfTerminate = 1u << 27;      // the path ends once its contributions are added
constexpr uint32_t kWfEmission = 1u << 28;       // emission seen by the extension ray counts
// Material word of an extension hit (hit.w): material index in the low bits, kind on top.
constexpr uint32_t kWfKindShift = 28;
constexpr uint32_t kWfMaterialMask = (1u << kWfKindShift) - 1u;
// Queue counters (uint32 each), cleared before every iteration.
enum WfCounter : int {
  kWfExtCount = 0, kWfShadowCount = 1, kWfMatCount = 2,  // [2..4]: diffuse, metal, dielectric
  kWfLive = 5, kWfTraceCursor = 6, kWfCounters = 8
};

struct WavefrontLaunch {
  RenderLaunch r;        // frame (r.f), work counter and launch counters; r.g: guiding (in_mix,
                         // guide_fraction) and recording (records != null)
  uint32_t capacity;     // path slots
  uint32_t* state;       // state word
  float4* ray_o;         // (ray origin.xyz, solid-angle pdf of the last diffuse bounce or -1)
  float4* ray_d;         // (ray direction.xyz, -)
  float4* thr;           // (throughput.xyz, pixel)
  float4* rad;           // (radiance.xyz, the path's work item)
  uint4* rng;            // PCG32 state and increment
  uint4* hit;            // (t bits, primitive record or kNoNode, tag, material word) of the extension ray
  float4* nee;           // 2 per slot: light and environment shadow-ray contributions
  float4* shadow_q;      // 2 per entry: (origin.xyz, tmax), (direction.xyz, target nee index)
  uint32_t* ext_q;       // slots whose extension ray is to be traced
  uint32_t* mat_q;       // 3 x capacity: slots to shade, per material kind
  uint32_t* q;           // kWfCounters counters
  int refill_lanes;      // > 1: trace lanes refill once fewer than this many of a warp still traverse
  // Guided renders: the inference queries of the diffuse queue (2 float4 per entry); their decoded
  // mixtures go to r.g.in_mix (kGuideDecodedF4 float4 per entry) with r.g.guide_fraction.
  float4* query;
  // Ray sorting (sort_keys != null): every queued ray's key (kind, direction octant, bucket of its
  // origin's primitive in leaf order), per-block bin counts and the sorted order of the entries.
  uint32_t* ext_key;     // capacity entries
  uint32_t* shadow_key;  // 2 x capacity entries
  uint32_t* sort_counts; // kWfSortBins x kWfSortBlocks
  uint32_t* sorted;      // 3 x capacity entries: queue entry at each sorted position
  uint32_t prim_count;   // primitive records (bucket scale)
  // Recording: per slot, the scatter record and the environment-NEE record of the diffuse vertex
  // shaded last (kNoNode when none); the next logic launch completes or drops them.
  uint2* rec_ref;
  // 1 once every work item has been handed out (the host learns it from an earlier iteration's
  // counter): a logic block with no live slot then has nothing to do.
  uint32_t work_done;
};
// Ray sorting: 2 kinds x 8 direction octants x 64 origin buckets, counted by kWfSortBlocks blocks.
constexpr int kWfSortBuckets = 64;
constexpr int kWfSortBins = 2 * 8 * kWfSortBuckets;
constexpr int kWfSortBlocks = 148;

// Vertices of every triangle record in leaf order (verts[3k..3k+2]) gathered from the scene-order
// triangles (tc_gpu_triangle records) through the records' tags.
cudaError_t launch_triangle_vertices(const PrimRecord* prims, uint32_t n, const void* triangles, float4* verts,
                                     cudaStream_t stream);

// Launchers implemented in kernels.cu. All enqueue on `stream` and return the launch error.
cudaError_t launch_trace_closest(const DevScene& s, const float* rays, uint64_t n, float tmin, uint32_t* prim,
                                 float* t, cudaStream_t stream);
cudaError_t launch_render(const RenderLaunch& r, int block_size, int grid_size, bool moments, cudaStream_t stream,
                          int mode = kModePlain);
int render_max_blocks_per_sm(int block_size, bool moments, int mode = kModePlain, int short_stack = 0,
                             int min_active = 1);
// One wavefront iteration (logic, [guide inference,] shade, trace) on `stream`; the caller
// clears w.q first. `guide` (guided renders) is the network that infers the diffuse queue.
// `marks`, when set, are kWfMarks timing events recorded before the logic launch and after the
// logic, inference (guided only), shading and trace groups.
struct GuideDevice;
constexpr int kWfMarks = 5;
cudaError_t launch_wavefront_iteration(const WavefrontLaunch& w, bool moments, int sm_count, cudaStream_t stream,
                                       const GuideDevice* guide = nullptr, const cudaEvent_t* marks = nullptr);
// Batched launch over r.jobs (r.job_count frames, items concatenated in job order): plain, or one
// round of the guided wavefront (r.g, with per-frame regions of the wave buffers).
cudaError_t launch_render_batch(const RenderLaunch& r, int block_size, int grid_size, cudaStream_t stream,
                                bool guided = false);
int render_batch_max_blocks_per_sm(int block_size, bool guided = false);
// prefix[0..n) = exclusive prefix of min(counts[i], jobs[i].wave_capacity); prefix[n] = total.
cudaError_t launch_job_prefix(const uint32_t* counts, const FrameJob* jobs, uint32_t n, uint32_t* prefix,
                              cudaStream_t stream);
// Training samples (3 float4 each: position + weight, normal, direction) from recorded diffuse
// scatters and environment shadow rays: weight = luminance of the radiance that arrived along
// the recorded direction, over the direction's sampling pdf. Only positive-weight samples are
// appended (compacted, order unspecified) to `samples`, which holds `sample_capacity` of them:
// *sample_count counts every positive-weight sample offered (so it may pass the capacity) and
// *weight_sum adds the weights of those stored. The caller zeroes both to start a new pool.
cudaError_t launch_guide_samples(const float4* records, const uint32_t* record_count, uint32_t capacity,
                                 const float4* path_radiance, float4* samples, uint32_t sample_capacity,
                                 uint32_t* sample_count, float* weight_sum, cudaStream_t stream);
// Device address of the library's static render scratch (kStaticScratchWords 64-bit words) in
// the CUDA context current on `device`, which must be the current device. The caller keeps it
// with the other resources of that context.
constexpr int kStaticScratchWords = 32;
cudaError_t render_static_scratch(int device, unsigned long long** out);
cudaError_t launch_resolve(const double* accum, uint32_t pixels, double inv_samples, float4* out,
                           cudaStream_t stream);
// Environment importance tables from RGB texels; `row_sums` is FP64 scratch of H entries.
// Whether launch_env_tables builds each alias table in shared memory (max(w, h) x 16 bytes); otherwise
// it needs alias_q ((h + 1) x max(w, h) doubles) and alias_idx (2 x as many indices).
inline bool env_alias_in_shared(uint32_t w, uint32_t h) {
  return size_t(w > h ? w : h) * (sizeof(double) + 2 * sizeof(uint32_t)) <= 200u * 1024u;
}
cudaError_t launch_env_tables(const float4* rgb, uint32_t w, uint32_t h, float intensity, float* marginal,
                              float* conditional, float* pdf, double* row_sums, double* total_out,
                              double* alias_q, uint32_t* alias_idx, uint2* cond_alias, uint2* marg_alias,
                              cudaStream_t stream);

}  // namespace tcb

#endif
