/*
 * toaster_cuda.h — C ABI of the B200 (sm_100a) path-tracing backend for toaster.
 *
 * This library replaces the `toaster-gpu` compute path (wgpu + shaders/pathtrace_spheres.wgsl).
 * It consumes the same packed scene records that `toaster_gpu::scene_upload::scene_to_gpu`
 * produces (crates/toaster-gpu/src/gpu_types.rs, byte-identical #[repr(C)] layouts) and returns
 * the same linear-HDR float4 image, row-major with y down and alpha = 1.
 *
 * Conventions
 *   - Every tc_* function returns TC_OK (0) or a negative TC_ERR_* code; tc_last_error() gives
 *     the message. The same checks that toaster-gpu performs with anyhow::ensure! are made here
 *     and reported as TC_ERR_INVALID.
 *   - Host pointers are copied; the library owns every device buffer and one CUDA stream per
 *     context. Calls are synchronous unless their name ends in _async, and except
 *     tc_render_no_alloc, which only enqueues its work. One context per thread.
 *   - There is no CPU fallback: without a usable sm_100 GPU, tc_create fails.
 */
#ifndef TOASTER_CUDA_H
#define TOASTER_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TC_ABI_VERSION 1

enum tc_status {
  TC_OK = 0,
  TC_ERR_INVALID = -1,    /* bad argument or scene contents */
  TC_ERR_CUDA = -2,       /* CUDA runtime or launch failure */
  TC_ERR_NO_DEVICE = -3,  /* no sm_100 device at the requested ordinal */
  TC_ERR_STATE = -4,      /* call out of order (e.g. render before upload) */
  TC_ERR_DEVICE_STATUS = -5 /* a kernel reported a bounded-wait or capacity failure */
};

/* ---------------------------------------------------------------- scene records
 * Byte-compatible with crates/toaster-gpu/src/gpu_types.rs (sizes pinned by its test
 * gpu_types_match_wgsl_layout_sizes, gpu_types.rs:200-211). */

/* GpuRenderParams (gpu_types.rs:8-56), 96 bytes. */
typedef struct tc_gpu_render_params {
  uint32_t width, height, samples, max_bounces;
  uint32_t sphere_count, triangle_count, material_count, frame_index;
  uint32_t background_kind; /* 0 sky, 1 black, 2 environment */
  uint32_t light_count;
  float total_light_weight;
  uint32_t _pad0;
  uint32_t environment_width, environment_height;
  float environment_intensity, environment_rotation_degrees;
  uint32_t accumulated_samples;
  uint32_t _pad1[3];
  uint32_t bvh_node_count, bvh_primitive_count;
  uint32_t _pad2[2];
} tc_gpu_render_params;

/* GpuCamera (gpu_types.rs:61-70), 64 bytes: origin, lower-left corner, horizontal, vertical. */
typedef struct tc_gpu_camera {
  float origin[4], lower_left_corner[4], horizontal[4], vertical[4];
} tc_gpu_camera;

/* GpuSphere (gpu_types.rs:75-83), 32 bytes. */
typedef struct tc_gpu_sphere {
  float center_radius[4];
  uint32_t material_index, _pad0[3];
} tc_gpu_sphere;

/* GpuTriangle (gpu_types.rs:88-100), 64 bytes. */
typedef struct tc_gpu_triangle {
  float v0[4], v1[4], v2[4];
  uint32_t material_index, _pad0[3];
} tc_gpu_triangle;

/* GpuTriangleAttributes (gpu_types.rs:105-123), 80 bytes; flags bit0 normals, bit1 uvs. */
typedef struct tc_gpu_triangle_attributes {
  float n0[4], n1[4], n2[4];
  float uv0[2], uv1[2], uv2[2];
  uint32_t flags, _pad0;
} tc_gpu_triangle_attributes;

/* GpuMaterial (gpu_types.rs:128-143), 48 bytes; kind 0 diffuse, 1 metal, 2 dielectric,
 * 3 emissive; params = (roughness, ior, emission strength, unused). */
typedef struct tc_gpu_material {
  uint32_t kind, texture_offset, texture_width, texture_height;
  float albedo[4];
  float params[4];
} tc_gpu_material;

/* GpuLight (gpu_types.rs:148-167), 96 bytes; kind 0 triangle, 1 sphere;
 * area_weight_cumulative = (area, weight, cumulative weight, unused). */
typedef struct tc_gpu_light {
  uint32_t kind, material_index, _pad0[2];
  float v0[4], v1[4], v2[4], center_radius[4];
  float area_weight_cumulative[4];
} tc_gpu_light;

/* GpuBvhNode (gpu_types.rs:172-184), 48 bytes; primitive_count > 0 marks a leaf. */
typedef struct tc_gpu_bvh_node {
  float min[4], max[4];
  uint32_t first_or_right, primitive_count, _pad[2];
} tc_gpu_bvh_node;

/* GpuPrimitiveRef (gpu_types.rs:189-194), 8 bytes; kind 0 sphere, 1 triangle. */
typedef struct tc_gpu_primitive_ref {
  uint32_t kind, index;
} tc_gpu_primitive_ref;

/* SceneGpuData (crates/toaster-gpu/src/scene_upload.rs:17-40) as pointers and counts.
 * bvh_nodes / bvh_primitives may be NULL: the library then builds the same median-split
 * hierarchy itself (crates/toaster-bvh/src/bvh.rs:92-154). environment_pixels holds
 * float4 texels (linear RGB, lane w ignored: the library builds its own 2-D CDF). */
typedef struct tc_scene_data {
  tc_gpu_render_params params;
  tc_gpu_camera camera;
  const tc_gpu_sphere* spheres;
  size_t sphere_count;
  const tc_gpu_triangle* triangles;
  size_t triangle_count;
  const tc_gpu_triangle_attributes* triangle_attributes;
  size_t triangle_attribute_count;
  const tc_gpu_material* materials;
  size_t material_count;
  const tc_gpu_light* lights;
  size_t light_count;
  const tc_gpu_bvh_node* bvh_nodes;
  size_t bvh_node_count;
  const tc_gpu_primitive_ref* bvh_primitives;
  size_t bvh_primitive_count;
  const uint32_t* texture_pixels;
  size_t texture_pixel_count;
  const float* environment_pixels;
  size_t environment_pixel_count;
} tc_scene_data;

/* Per-dispatch options beyond GpuRenderParams. Zero-initialised means defaults. */
typedef struct tc_render_options {
  uint32_t block_size;       /* threads per block for the path kernel; 0 = tuned default */
  uint32_t samples_per_item; /* samples one lane traces for a pixel before taking new work; 0 = default */
  uint32_t keep_moments;     /* 1: also accumulate per-pixel sums of squared samples (FP64) */
  uint32_t guiding;          /* 1: learned path guiding at diffuse vertices (needs tc_guide_set_params) */
  uint32_t guide_record;     /* record (position, normal, direction, incident radiance) training
                                samples at every diffuse scatter of this batch and at every
                                environment shadow ray that reaches the sky, into the context's
                                sample pool (16,777,216 samples; later ones are dropped):
                                1 = empty the pool first, 2 = add to it. Plain renders, and
                                guided renders on the wavefront schedule (their samples weighted
                                by the mixture pdf they were drawn with) */
  uint32_t wave_paths;       /* paths in flight: guided wavefront (0 = 2^23) or plain wavefront
                                schedule (0 = 2^23) */
  uint32_t short_stack;      /* traversal stack entries per thread held in shared memory (0..16;
                                deeper entries live in local memory); 0 = none */
  uint32_t refill_lanes;     /* a warp pauses traversal to refill finished lanes once fewer than
                                this many of its 32 lanes are still traversing (1..32; 1 = only
                                when all have finished); 0 = default. refill_lanes > 1 or
                                short_stack > 0 select the resumable traversal, for plain renders
                                without moments; other launches ignore both */
  float guide_fraction;      /* guided renders: probability of sampling the network's mixture at a
                                diffuse vertex (one-sample MIS with cosine sampling, the mixture pdf
                                (1 - f) cos/pi + f q); in [0, 1), 0 = default 0.5 */
  uint32_t schedule;         /* plain and guided renders: TC_SCHEDULE_AUTO (0) = the wavefront for
                                tc_render and tc_autotune calls of at least 2^20 paths and 1 or more
                                bounces, the megakernel otherwise; TC_SCHEDULE_MEGAKERNEL (1) = one
                                persistent path kernel (guided: in rounds with inference between);
                                TC_SCHEDULE_WAVEFRONT (2) = per-path state in device memory and
                                three launches per bounce (logic, material-sorted shading, tracing
                                with one ray kind per warp; guided: the diffuse queue inferred
                                between logic and shading), wave_paths slots (0 = 2^23). Batched
                                launches and captured animation frames use the megakernel. */
  uint32_t ray_sort;         /* wavefront schedule: sort each iteration's queued rays by kind, direction
                                octant and the leaf-order bucket of their origin's primitive before
                                tracing (three small launches), so a warp's rays start near each other
                                and head the same way. 0 = library default (off), 1 = off, 2 = on */
  uint32_t phase_timing;     /* wavefront schedule: 1 = record CUDA events between each iteration's
                                launch groups on the render's stream and report their summed device
                                time in tc_stats (trace_ms, logic_ms, shade_ms, guide_ms); 0 = off */
} tc_render_options;
#define TC_SCHEDULE_AUTO 0u
#define TC_SCHEDULE_MEGAKERNEL 1u
#define TC_SCHEDULE_WAVEFRONT 2u

/* Counters of the most recent tc_render / tc_trace_* call. */
typedef struct tc_stats {
  uint64_t paths;            /* camera paths traced */
  uint64_t rays;             /* extension + shadow rays */
  uint64_t extension_rays;
  uint64_t shadow_rays;
  float kernel_ms;           /* device time of the main kernel (CUDA events) */
  float total_ms;            /* device time of the whole call including copies */
  uint32_t bvh_depth;        /* deepest leaf of the uploaded hierarchy */
  uint32_t status_flags;     /* device status word (0 = clean) */
  uint32_t kernel_launches;  /* this library's kernel launches of the last render call (path kernels,
                                guide inference; not memsets or copies) */
  float trace_ms;            /* wavefront render with phase_timing: device time of the trace launches
                                (ray sorting included); 0 otherwise */
  float logic_ms;            /* ... of the logic launches */
  float shade_ms;            /* ... of the shading launches */
  float guide_ms;            /* ... of the guide inference launches (guided wavefront) */
  uint32_t wf_iterations;    /* wavefront iterations of the last render; 0 for the megakernel */
} tc_stats;

typedef struct tc_context tc_context;

/* Library and device --------------------------------------------------------------------- */
int tc_abi_version(void);
/* Message of the last failure on this thread when ctx is NULL (e.g. after tc_create). */
const char* tc_last_error(const tc_context* ctx);

/* Replaces toaster-gpu create_gpu_context (crates/toaster-gpu/src/device.rs:49-100). */
int tc_create(int device_ordinal, tc_context** out_ctx);
int tc_destroy(tc_context* ctx);

/* Makes the context enqueue its work on `stream` (a cudaStream_t of the context's device owned
 * by the caller), or on its own stream again when NULL. Lets a host time calls with its own
 * CUDA events. No reference counterpart (wgpu owns its queue). */
int tc_set_stream(tc_context* ctx, void* stream);

/* Replaces create_scene_gpu_buffers + the queue.write_buffer uploads
 * (crates/toaster-gpu/src/buffers.rs:117-271, path_tracer.rs:676-721). */
int tc_upload_scene(tc_context* ctx, const tc_scene_data* scene);

/* Triangle test of the scenes uploaded after this call (no reference counterpart: the reference
 * uses Moller-Trumbore only, crates/toaster-cpu/src/intersect.rs:87-120):
 *   TC_TRIANGLE_MOLLER_TRUMBORE (0, default)  the reference's test, operation for operation: the
 *                                             parity mode, bit-exact closest hits;
 *   TC_TRIANGLE_WATERTIGHT (1)                the FP32 watertight test of Woop, Benthin and Wald
 *                                             (JCGT 2013): no ray slips between triangles that share
 *                                             an edge; hit distances round differently, so ties and
 *                                             near-ties may pick another primitive than the reference.
 * The watertight test keeps a second copy of the triangle vertices in leaf order (48 B per
 * primitive) and is traced by tc_trace_closest and by plain renders on the wavefront schedule;
 * other render calls on such a scene fail with TC_ERR_INVALID. */
#define TC_TRIANGLE_MOLLER_TRUMBORE 0
#define TC_TRIANGLE_WATERTIGHT 1
int tc_set_triangle_test(tc_context* ctx, int test);

/* Where tc_upload_scene builds the median-split hierarchy when the scene brings none: 0 = on the
 * device for scenes of at least 4,096 primitives, on the host below (default); 1 = always on the
 * host; 2 = always on the device. Both builds produce the reference's tree (same topology,
 * primitive order and bounds). The device build runs level by level with a segmented stable
 * sort; a node whose centroids all coincide (a degenerate leaf of the reference) makes it fall
 * back to the host build. Replaces the host-side FlatBvh::build of scene_upload.rs:296-340. */
int tc_set_hierarchy_build(tc_context* ctx, int mode);

/* Replaces the camera write_buffer (path_tracer.rs:680-684). */
int tc_set_camera(tc_context* ctx, const tc_gpu_camera* camera);

/* What one scene evaluation changed; mirrors toaster_scene::SceneChanges
 * (crates/toaster-scene/src/evaluation.rs:9-18). Nonzero = changed. */
typedef struct tc_scene_changes {
  uint32_t camera;             /* camera basis or position */
  uint32_t spheres;            /* at least one sphere moved or resized */
  uint32_t triangles;          /* at least one triangle or its attributes changed */
  uint32_t emissive_geometry;  /* a moved primitive is emissive: the light records change */
} tc_scene_changes;

/* Per-frame update of an uploaded scene (the evaluated frame of path_tracer.rs:611-721). Instead
 * of the reference's host rebuild + full re-upload, the changed geometry is copied to the device
 * and the hierarchy is refit there: primitive records are rewritten and every box is recomputed
 * bottom-up with the topology of the last tc_upload_scene. Intersections stay exact; only the
 * tree's quality drifts under large motion (call tc_upload_scene to rebuild). `scene` holds the
 * whole evaluated frame in the reference records; its counts must equal the uploaded scene's
 * (path_tracer.rs:639-653). Materials are not re-read. Lights are re-packed when
 * emissive_geometry is set, the camera when camera is set. Synchronous. */
int tc_update_geometry(tc_context* ctx, const tc_scene_data* scene, const tc_scene_changes* changes);

/* Replaces dispatch_compute_2d (crates/toaster-gpu/src/dispatch.rs:28-60): traces
 * params->samples paths per pixel. params->accumulated_samples == 0 starts a new image;
 * otherwise it must equal the samples already accumulated (progressive mode,
 * path_tracer.rs:900-923). options may be NULL. */
int tc_render(tc_context* ctx, const tc_gpu_render_params* params, const tc_render_options* options);

/* n independent frames of possibly different scenes and sizes: contexts[i] holds scene i (from
 * tc_upload_scene) and renders params[i] under the same progressive contract as tc_render. Frames
 * too small to fill the GPU share one persistent launch: their work items share one queue, so
 * they fill the GPU together instead of one launch (and one tail) each. With options->schedule
 * TC_SCHEDULE_AUTO, a frame of at least 2^20 paths (which fills the GPU by itself) is rendered by
 * its own wavefront call instead, after the shared launch; TC_SCHEDULE_MEGAKERNEL puts every frame
 * in the shared launch, TC_SCHEDULE_WAVEFRONT every frame with at least one bounce in a call of its own.
 * No reference counterpart: the reference renders scenes one dispatch at a time
 * (dispatch.rs:28-60). All contexts must be on one device and distinct; the work runs on
 * contexts[0]'s stream after the others' pending work, and tc_get_stats(contexts[0]) reports the
 * whole batch. Options may set block_size and samples_per_item; moments and recording are
 * rejected. With options->guiding every context needs guide parameters (tc_guide_set_params); the
 * frames of the shared launch need one sample count and run the guided wavefront over all of them
 * at once, in waves of whole samples per pixel (wave_paths, 0 = 2^23 paths), each frame's
 * suspended paths in a region of their own that the frame's own network infers. Synchronous. */
int tc_render_batch(tc_context* const* contexts, const tc_gpu_render_params* params, size_t n,
                    const tc_render_options* options);

/* Autotuner: a coordinate search over the launch shape on the uploaded scene at params' size,
 * one knob at a time, each stage keeping the fastest value: first the schedule {megakernel,
 * wavefront}; then for the megakernel block size {64, 128, 256}, refill lanes {1, 12, 20, 28},
 * shared-memory short-stack entries {0, 8, 16} and samples per work item {1, 2, 4} (guided: its
 * wave width {2^21, 2^22, 2^23} paths instead); for the wavefront the trace launch's refill lanes
 * {1, 12, 20, 28} and its path slots {2^21, 2^22, 2^23}. Each shape
 * runs once untimed and once timed (CUDA events) with probe_samples spp (0 = min(params->samples,
 * 4)). Other fields of `base` are kept. The context's accumulated image is replaced by the last
 * probe. No reference counterpart. */
typedef struct tc_tune_result {
  tc_render_options best;
  float best_kernel_ms;       /* device time of the fastest probe */
  float best_mpaths_per_s;    /* its throughput */
  uint32_t candidates;        /* shapes timed */
  uint32_t probe_samples;
} tc_tune_result;
int tc_autotune(tc_context* ctx, const tc_gpu_render_params* params, const tc_render_options* base,
                uint32_t probe_samples, tc_tune_result* out);

/* Animated frames through one captured CUDA graph (the frame loop of
 * render_gpu_with_sink, path_tracer.rs:591-840, with its per-frame host rebuild replaced by a
 * device refit). tc_animation_create renders `first_frame` once to size every buffer, then
 * captures a frame's whole device work: the copy of the frame's geometry, camera and frame index
 * from pinned staging, the hierarchy update, the render of `params` (plain, or guided when
 * options->guiding is set and the context holds trained guide weights), display conversion
 * (exposure_stops) and the RGBA8 readback. tc_animation_frame copies one evaluated frame (same
 * counts as the uploaded scene) into the staging, replays the graph and writes 4*width*height
 * bytes to rgba (may be NULL). Each frame is independent (accumulated_samples = 0) and seeded by
 * frame_index. The context must not be used by other calls while an animation replays on it.
 * flags:
 *   TC_ANIM_UPDATE_LIGHTS  re-pack the light records every frame (moving emitters);
 *   TC_ANIM_REBUILD        build the frame's median-split hierarchy on the device inside the graph
 *                          (the reference's per-frame tree, so hits stay bit-exact) instead of
 *                          refitting the first frame's tree. A refit is cheaper, but its boxes
 *                          loosen as primitives move apart; a rebuild keeps traversal cost flat.
 *                          A frame whose tree would need a degenerate leaf fails with
 *                          TC_ERR_DEVICE_STATUS. */
#define TC_ANIM_UPDATE_LIGHTS 1u
#define TC_ANIM_REBUILD 2u
typedef struct tc_animation tc_animation;
int tc_animation_create(tc_context* ctx, const tc_scene_data* first_frame, const tc_gpu_render_params* params,
                        const tc_render_options* options, float exposure_stops, uint32_t flags,
                        tc_animation** out);
int tc_animation_frame(tc_animation* anim, const tc_scene_data* frame, uint32_t frame_index, uint8_t* rgba,
                       size_t n_bytes);
int tc_animation_destroy(tc_animation* anim);

/* Replaces readback_pixels (crates/toaster-gpu/src/readback.rs:8-25): writes width*height
 * float4 linear-HDR averages into rgba (n_floats >= 4*width*height). */
int tc_readback(tc_context* ctx, float* rgba, size_t n_floats);

/* Display conversion on the device, then readback of 4 bytes per pixel: exposure (2^stops),
 * ACES fitted tone map, clamp, sRGB transfer and rounding to RGBA8 (alpha 255), row-major,
 * y down. Replaces readback_pixels + pixels_to_rgba_image (crates/toaster-gpu/src/
 * image_output.rs:57-88 over crates/toaster-core/src/color.rs:24-74), which convert on the
 * host after copying 16 bytes per pixel. n_bytes >= 4*width*height. */
int tc_readback_rgba8(tc_context* ctx, float exposure_stops, uint8_t* rgba, size_t n_bytes);

/* JPEG frame of the accumulated image at `quality` 1..100: display conversion (as
 * tc_readback_rgba8, alpha dropped) and baseline JPEG encoding (4:2:0) on the device with nvJPEG;
 * only the compressed bytes cross to the host. Replaces encode_pixels_to_jpeg
 * (crates/toaster-gpu/src/image_output.rs:27-56), which the MJPEG preview stream of
 * toaster-server sends frame by frame (routes.rs:84-106). *length receives the frame's size; with
 * out = NULL nothing is copied (a size query), and a capacity below the size fails. The
 * encoder's bytes differ from the image crate's; both decode to the same picture within JPEG
 * error. */
int tc_encode_jpeg(tc_context* ctx, uint32_t quality, float exposure_stops, uint8_t* out, size_t capacity,
                   size_t* length);

/* The same conversion into caller-owned device memory (d_rgba, n_bytes >= 4*width*height),
 * enqueued on `stream` (NULL = the context's stream) without synchronising, for sinks that
 * consume frames on the device. No reference counterpart. */
int tc_display_rgba8_async(tc_context* ctx, float exposure_stops, void* d_rgba, size_t n_bytes, void* stream);

/* Same traversal and estimator as tc_render, for callers that must not have the library allocate
 * device memory at render time: hosts whose device memory all belongs to their own pool or
 * framework allocator (a cudaMalloc beside the pool is invisible to its accounting and fails once
 * the pool has reserved the rest of HBM), and embedders that run under a fixed device-memory
 * budget which has to be known before the first frame. No reference counterpart (toaster-gpu
 * allocates all its buffers through wgpu).
 * It calls no cudaMalloc, cudaFree or other allocating routine. The scene comes from an earlier
 * tc_upload_scene; the caller supplies the FP64 per-pixel sums: `sums` is device memory of at
 * least 3*width*height doubles (n_doubles). accumulated_samples == 0 clears it first, otherwise
 * the batch is added to it. The image is sums / (total samples), which the caller tracks.
 * Scratch: the path kernel's work counter and ray counters live in one 256-byte static device
 * array of the library (at most 32 64-bit words; this call uses 4 at any image size), which
 * every GPU that loads the library holds until the process exits. All calls share it and it
 * keeps the last call's values: each call clears the words it uses before its kernel, and calls
 * whose work overlaps on the GPU race on it, so serialise them (one stream, or wait between
 * calls). Set-up: the first call on each context looks up the array's device address in that
 * context's CUDA context (cudaGetSymbolAddress, with the context's device current) and keeps it
 * with the context; make that first call before any stream capture. A context does not survive
 * a cudaDeviceReset (none of its buffers do); create a new one afterwards.
 * Ordering: the work is enqueued on `stream` (NULL = the context's stream) and not
 * synchronised, and it reads the context's scene buffers. Synchronise `stream` before the next
 * call that changes the context (tc_upload_scene, tc_update_geometry, tc_set_camera,
 * tc_destroy and the like) or reads `sums` on the host.
 * Rejects frames above 2^31 pixels and sums buffers smaller than 3*width*height doubles. */
int tc_render_no_alloc(tc_context* ctx, const tc_gpu_render_params* params, double* sums, size_t n_doubles,
                       void* stream);

/* Per-pixel FP64 running sums (3 per pixel) and, when keep_moments was set, sums of squared
 * sample values (3 per pixel). Either pointer may be NULL. *samples receives the count. */
int tc_readback_sums(tc_context* ctx, double* sum, double* sum_sq, size_t n_doubles, uint32_t* samples);

/* Closest hit for n host rays (origin.xyz, direction.xyz; 6 floats each) with minimum
 * distance tmin: prim[i] = kind << 31 | scene index, with the GpuPrimitiveRef kind codes
 * (0 sphere, 1 triangle), or TC_MISS; t[i] = hit distance or +inf. Traversal and
 * intersection follow crates/toaster-cpu/src/intersect.rs:172-263 bit for bit. */
#define TC_MISS 0xFFFFFFFFu
#define TC_PRIM_TRIANGLE_BIT 0x80000000u
int tc_trace_closest(tc_context* ctx, const float* rays, size_t n, float tmin, uint32_t* prim, float* t);

/* Same as tc_trace_closest on device-resident buffers, enqueued on `stream` (a cudaStream_t,
 * NULL = the context stream); nothing is synchronised. */
int tc_trace_closest_device_async(tc_context* ctx, const float* d_rays, size_t n, float tmin, uint32_t* d_prim,
                                  float* d_t, void* stream);

int tc_get_stats(const tc_context* ctx, tc_stats* out);

/* Learned path guiding (no reference counterpart: toaster has no guiding) ----------------------
 * An MLP maps an 80-wide encoding of a surface point (12-frequency Fourier features of
 * (p - centre) * scale, plus the normal) through three 64-wide ReLU layers to an 8-lobe von
 * Mises-Fisher mixture over directions. BF16 weights and activations, FP32 accumulation on the
 * tcgen05 tensor cores, FP32 master weights and Adam. Parameters are packed as W1[64][80], b1[64],
 * W2[64][64], b2[64], W3[64][64], b3[64], W4[32][64], b4[32] (15,584 floats); W1 columns 75..79
 * are padding and stay zero. */
#define TC_GUIDE_PARAMS 15584
/* Sets the weights (resets the Adam state) and the encoding frame bounds = (cx, cy, cz, scale). */
int tc_guide_set_params(tc_context* ctx, const float* params, const float* bounds);
int tc_guide_get_params(tc_context* ctx, float* params);
/* queries: n x 6 floats (position, normal); out: n x 40 floats = 8 x (mu.xyz, kappa) + 8 weights. */
int tc_guide_infer(tc_context* ctx, const float* queries, size_t n, float* out);
/* samples: n x 10 floats (position, normal, direction, weight). Writes the gradient of the mean
 * weighted negative log-likelihood (TC_GUIDE_PARAMS floats) and the loss. */
int tc_guide_loss_grad(tc_context* ctx, const float* samples, size_t n, float* grad, float* loss);
/* One Adam step (beta 0.9/0.999, eps 1e-8) with the gradient of the last tc_guide_loss_grad. */
int tc_guide_adam_step(tc_context* ctx, float lr);
/* steps x (loss + gradient on `batch` samples + Adam) over the given samples, visited in a
 * seeded random order. losses (optional) receives one value per step. */
int tc_guide_train(tc_context* ctx, const float* samples, size_t n, uint32_t steps, uint32_t batch, float lr,
                   uint64_t seed, float* losses);

/* Runs `steps` Adam steps on batches of `batch` samples drawn at random from the sample pool:
 * the samples of every tc_render with guide_record since the last one with guide_record = 1
 * (weight = luminance of the radiance that arrived along the scattered direction times
 * cos / (pi p) for a direction drawn with pdf p, or, for an environment shadow ray that reached
 * the sky, its radiance times the BSDF side's MIS share over the light pdf; normalised by the
 * pool's mean weight and clamped at 50x the mean; directions that carried no radiance are
 * dropped, as they add nothing to the weighted likelihood). losses (optional) receives one value
 * per step and n_samples (optional) the number of samples in the pool. */
int tc_guide_train_recorded(tc_context* ctx, uint32_t steps, uint32_t batch, float lr, uint64_t seed, float* losses,
                            uint32_t* n_samples);

/* The sample pool, as tc_guide_train_recorded sees it: 12 floats each (position + weight, normal + 0, direction + 0), weight = luminance of
 * the radiance that arrived along the recorded direction. Only directions that carried radiance
 * are kept (in an unspecified order). Writes min(count, n_floats / 12) samples; *count receives
 * their number. out may be NULL to query the count. No reference counterpart (inspection of the
 * guiding data). */
int tc_guide_recorded_samples(tc_context* ctx, float* out, size_t n_floats, uint32_t* count);

/* Tensor-core self-test (no reference counterpart): one 128 x n tile D = A * B^T with bf16 A
 * (128 x k, row-major) and B (n x k, row-major) staged in shared memory as K-major
 * (mn_major = 0) or MN-major (1) operands, FP32 accumulation in tensor memory. d receives
 * 128 x n floats. 16 <= n <= 128 and 16 <= k <= 80, both multiples of 16. */
int tc_umma_selftest(const uint16_t* a, const uint16_t* b, float* d, int n, int k, int a_mn_major, int b_mn_major);

/* Cache read-bandwidth probe (no reference counterpart; measurement only): every SM streams a
 * zero-filled device buffer of `bytes` (>= 1 MiB, allocated and freed by the call) `passes` times
 * with 16-byte loads that bypass L1, after one untimed pass. A buffer smaller than L2 (126 MB on
 * B200) gives the L2 read bandwidth, a larger one HBM. *gb_per_s receives the rate (CUDA events).
 * The path kernel's roofline on L2-resident scenes is quoted against this figure. Errors are
 * reported by tc_probe_last_error. */
int tc_probe_cache_read(int device_ordinal, size_t bytes, int passes, double* gb_per_s);
const char* tc_probe_last_error(void);

/* Host-only helpers (no GPU needed) -------------------------------------------------------- */

/* Builds the median-split hierarchy of crates/toaster-bvh for the given spheres and triangles
 * (spheres first, triangles padded by 1e-5, scene_upload.rs:296-346) and writes it in the
 * reference's flat layout. Capacities: nodes >= 2*(n_spheres+n_triangles)-1, prims >= n.
 * Returns the node count (>= 0) or a negative error. */
long tc_build_bvh_host(const tc_gpu_sphere* spheres, size_t n_spheres, const tc_gpu_triangle* triangles,
                       size_t n_triangles, tc_gpu_bvh_node* nodes, size_t node_capacity,
                       tc_gpu_primitive_ref* prims, size_t prim_capacity);

/* Byte sizes of the record types as compiled into the library (layout check). */
int tc_record_sizes(uint32_t* out, size_t n);

/* Scene files (host only) ------------------------------------------------------------------
 * Replaces toaster_gpu::scene_upload::load_scene_gpu (crates/toaster-gpu/src/scene_upload.rs:54-57:
 * toaster_scene::load_scene, crates/toaster-scene/src/loader.rs:534-971, then scene_to_gpu,
 * scene_upload.rs:79-294) for a caller without the Rust loader: reads a scene JSON file with its glTF / GLB meshes
 * (crates/toaster-assets/src/gltf_loader.rs:11-233; 8-bit PNG base-colour textures) and its
 * Radiance .hdr or PNG environment map, validates it with the reference loader's rules and packs
 * the records. The hierarchy is not packed (bvh_nodes NULL): tc_upload_scene builds it.
 * Animation, physics, triggers, spawn points and event reactions are skipped. On failure returns
 * TC_ERR_INVALID with the message in error (NUL-terminated, truncated to error_capacity). */
typedef struct tc_loaded_scene tc_loaded_scene;
int tc_scene_load(const char* path, tc_loaded_scene** out, char* error, size_t error_capacity);
/* The packed records; valid until tc_loaded_scene_free. */
const tc_scene_data* tc_loaded_scene_data(const tc_loaded_scene* scene);
/* The scene's display exposure in stops (its "display" block, 0 when absent). */
int tc_loaded_scene_display(const tc_loaded_scene* scene, float* exposure_stops);
int tc_loaded_scene_free(tc_loaded_scene* scene);

#ifdef __cplusplus
}
#endif

#endif /* TOASTER_CUDA_H */
