//! Declarations of the C ABI in `include/toaster_cuda.h`.
//!
//! The scene records are toaster-gpu's own `#[repr(C)]` types (`toaster_gpu::gpu_types`), whose
//! layouts the library takes byte for byte; only the pointer-and-count wrapper of
//! `SceneGpuData` and the option structs are declared here.

use std::ffi::{c_char, c_int, c_void, CStr};

use anyhow::{bail, Result};
use toaster_gpu::gpu_types::{
    GpuBvhNode, GpuCamera, GpuLight, GpuMaterial, GpuPrimitiveRef, GpuRenderParams, GpuSphere, GpuTriangle,
    GpuTriangleAttributes,
};
use toaster_gpu::scene_upload::SceneGpuData;

/// `tc_scene_data`: `SceneGpuData` as pointers and counts (borrowed for one call).
#[repr(C)]
pub struct TcSceneData {
    /// Render dimensions, sampling controls and resource counts.
    pub params: GpuRenderParams,
    /// Camera basis and image plane.
    pub camera: GpuCamera,
    /// Packed spheres.
    pub spheres: *const GpuSphere,
    /// Sphere count.
    pub sphere_count: usize,
    /// Packed triangles.
    pub triangles: *const GpuTriangle,
    /// Triangle count.
    pub triangle_count: usize,
    /// Per-triangle normals and texture coordinates, or null.
    pub triangle_attributes: *const GpuTriangleAttributes,
    /// Attribute count (0 or the triangle count).
    pub triangle_attribute_count: usize,
    /// Materials.
    pub materials: *const GpuMaterial,
    /// Material count.
    pub material_count: usize,
    /// Emissive primitives for next-event estimation.
    pub lights: *const GpuLight,
    /// Light count.
    pub light_count: usize,
    /// Flattened hierarchy in the reference layout, or null (the library builds the same tree).
    pub bvh_nodes: *const GpuBvhNode,
    /// Node count.
    pub bvh_node_count: usize,
    /// Leaf-ordered primitive references, or null with `bvh_nodes`.
    pub bvh_primitives: *const GpuPrimitiveRef,
    /// Reference count.
    pub bvh_primitive_count: usize,
    /// RGBA8 texture atlas.
    pub texture_pixels: *const u32,
    /// Texel count.
    pub texture_pixel_count: usize,
    /// Linear HDR environment texels (4 floats each).
    pub environment_pixels: *const f32,
    /// Environment texel count.
    pub environment_pixel_count: usize,
}

impl TcSceneData {
    /// Borrows every array of `scene`. With `with_bvh` false the hierarchy is left out and the
    /// library builds it (on the device for large scenes).
    pub fn borrow(scene: &SceneGpuData, with_bvh: bool) -> Self {
        fn ptr<T>(v: &[T]) -> *const T {
            if v.is_empty() {
                std::ptr::null()
            } else {
                v.as_ptr()
            }
        }
        Self {
            params: scene.params,
            camera: scene.camera,
            spheres: ptr(&scene.spheres),
            sphere_count: scene.spheres.len(),
            triangles: ptr(&scene.triangles),
            triangle_count: scene.triangles.len(),
            triangle_attributes: ptr(&scene.triangle_attributes),
            triangle_attribute_count: scene.triangle_attributes.len(),
            materials: ptr(&scene.materials),
            material_count: scene.materials.len(),
            lights: ptr(&scene.lights),
            light_count: scene.lights.len(),
            bvh_nodes: if with_bvh { ptr(&scene.bvh_nodes) } else { std::ptr::null() },
            bvh_node_count: if with_bvh { scene.bvh_nodes.len() } else { 0 },
            bvh_primitives: if with_bvh { ptr(&scene.bvh_primitives) } else { std::ptr::null() },
            bvh_primitive_count: if with_bvh { scene.bvh_primitives.len() } else { 0 },
            texture_pixels: ptr(&scene.texture_pixels),
            texture_pixel_count: scene.texture_pixels.len(),
            environment_pixels: ptr(&scene.environment_pixels).cast(),
            environment_pixel_count: scene.environment_pixels.len(),
        }
    }
}

/// `tc_render_options` (zero = library defaults).
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct TcRenderOptions {
    /// Threads per block of the path kernel.
    pub block_size: u32,
    /// Samples a lane traces for one pixel before taking new work.
    pub samples_per_item: u32,
    /// Also accumulate per-pixel sums of squared samples.
    pub keep_moments: u32,
    /// Learned path guiding.
    pub guiding: u32,
    /// Record guiding training samples.
    pub guide_record: u32,
    /// Paths in flight of the wavefront schedules.
    pub wave_paths: u32,
    /// Shared-memory traversal stack entries.
    pub short_stack: u32,
    /// Dynamic-fetch threshold of the traversal.
    pub refill_lanes: u32,
    /// Guided renders: probability of sampling the network's mixture.
    pub guide_fraction: f32,
    /// Plain and guided renders: 0 automatic, 1 megakernel, 2 wavefront.
    pub schedule: u32,
    /// Wavefront: 0 default, 1 no ray sorting, 2 rays sorted before tracing.
    pub ray_sort: u32,
    /// Wavefront: 1 = device time of each launch group in the statistics.
    pub phase_timing: u32,
}

/// `tc_scene_changes`, the `SceneChanges` of an evaluated frame.
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct TcSceneChanges {
    /// Camera basis or position changed.
    pub camera: u32,
    /// At least one sphere changed.
    pub spheres: u32,
    /// At least one triangle or its attributes changed.
    pub triangles: u32,
    /// A moved primitive is emissive.
    pub emissive_geometry: u32,
}

/// `tc_stats`: counters and device times of the last call.
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct TcStats {
    /// Camera paths traced.
    pub paths: u64,
    /// Extension + shadow rays.
    pub rays: u64,
    /// Extension rays.
    pub extension_rays: u64,
    /// Shadow rays.
    pub shadow_rays: u64,
    /// Device time of the path kernels.
    pub kernel_ms: f32,
    /// Device time of the whole call.
    pub total_ms: f32,
    /// Depth of the uploaded hierarchy.
    pub bvh_depth: u32,
    /// Device status word.
    pub status_flags: u32,
    /// Kernel launches of the last render call.
    pub kernel_launches: u32,
    /// Wavefront with phase timing: device time of the trace launches.
    pub trace_ms: f32,
    /// ... of the logic launches.
    pub logic_ms: f32,
    /// ... of the shading launches.
    pub shade_ms: f32,
    /// ... of the guide inference launches.
    pub guide_ms: f32,
    /// Wavefront iterations of the last render.
    pub wf_iterations: u32,
}

/// Opaque `tc_context`.
pub enum TcContext {}
/// Opaque `tc_animation`.
pub enum TcAnimation {}
/// Opaque `tc_loaded_scene`.
pub enum TcLoadedScene {}

/// `TC_ANIM_UPDATE_LIGHTS`: re-pack light records every animation frame.
pub const TC_ANIM_UPDATE_LIGHTS: u32 = 1;
/// `TC_ANIM_REBUILD`: per-frame device hierarchy build inside the animation graph.
pub const TC_ANIM_REBUILD: u32 = 2;

extern "C" {
    pub fn tc_abi_version() -> c_int;
    pub fn tc_last_error(ctx: *const TcContext) -> *const c_char;
    pub fn tc_create(device: c_int, out: *mut *mut TcContext) -> c_int;
    pub fn tc_destroy(ctx: *mut TcContext) -> c_int;
    pub fn tc_set_stream(ctx: *mut TcContext, stream: *mut c_void) -> c_int;
    pub fn tc_upload_scene(ctx: *mut TcContext, scene: *const TcSceneData) -> c_int;
    pub fn tc_update_geometry(ctx: *mut TcContext, scene: *const TcSceneData, changes: *const TcSceneChanges) -> c_int;
    pub fn tc_set_camera(ctx: *mut TcContext, camera: *const GpuCamera) -> c_int;
    pub fn tc_render(ctx: *mut TcContext, params: *const GpuRenderParams, opts: *const TcRenderOptions) -> c_int;
    pub fn tc_readback(ctx: *mut TcContext, rgba: *mut f32, n_floats: usize) -> c_int;
    pub fn tc_readback_rgba8(ctx: *mut TcContext, exposure_stops: f32, rgba: *mut u8, n_bytes: usize) -> c_int;
    pub fn tc_trace_closest(ctx: *mut TcContext, rays: *const f32, n: usize, tmin: f32, prim: *mut u32,
                            t: *mut f32) -> c_int;
    pub fn tc_get_stats(ctx: *const TcContext, out: *mut TcStats) -> c_int;
    pub fn tc_animation_create(ctx: *mut TcContext, first: *const TcSceneData, params: *const GpuRenderParams,
                               opts: *const TcRenderOptions, exposure_stops: f32, flags: u32,
                               out: *mut *mut TcAnimation) -> c_int;
    pub fn tc_animation_frame(anim: *mut TcAnimation, frame: *const TcSceneData, frame_index: u32, rgba: *mut u8,
                              n_bytes: usize) -> c_int;
    pub fn tc_animation_destroy(anim: *mut TcAnimation) -> c_int;
    pub fn tc_scene_load(path: *const c_char, out: *mut *mut TcLoadedScene, error: *mut c_char,
                         error_capacity: usize) -> c_int;
    pub fn tc_loaded_scene_data(scene: *const TcLoadedScene) -> *const TcSceneData;
    pub fn tc_loaded_scene_display(scene: *const TcLoadedScene, exposure_stops: *mut f32) -> c_int;
    pub fn tc_loaded_scene_free(scene: *mut TcLoadedScene) -> c_int;
}

/// Maps a `tc_*` status to `anyhow`, with the library's message (the reference's error style).
pub fn check(ctx: *const TcContext, code: c_int) -> Result<()> {
    if code == 0 {
        return Ok(());
    }
    // SAFETY: tc_last_error returns a NUL-terminated string owned by the library (per context, or
    // per thread when ctx is null) that stays valid until the next call on it.
    let msg = unsafe { CStr::from_ptr(tc_last_error(ctx)) }.to_string_lossy().into_owned();
    bail!("{msg} (toaster_cuda status {code})")
}
