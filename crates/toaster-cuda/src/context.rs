//! Owned CUDA context of the library: one per device, freed on drop.

use anyhow::{ensure, Result};
use image::RgbaImage;
use toaster_gpu::gpu_types::GpuRenderParams;
use toaster_gpu::scene_upload::SceneGpuData;
use toaster_gpu::GpuAdapterInfo;
use toaster_scene::SceneChanges;

use crate::ffi::{self, TcContext, TcRenderOptions, TcSceneChanges, TcSceneData, TcStats};

/// A `tc_context`: device buffers of one scene, its accumulation and its stream.
pub struct CudaContext {
    raw: *mut TcContext,
    device: i32,
}

impl CudaContext {
    /// Replaces `create_gpu_context` (crates/toaster-gpu/src/device.rs:49-100): fails without an
    /// sm_100 device at `device`.
    pub fn new(device: i32) -> Result<Self> {
        let mut raw = std::ptr::null_mut();
        // SAFETY: `raw` is a valid out pointer; on failure it stays null and the error is per thread.
        ffi::check(std::ptr::null(), unsafe { ffi::tc_create(device, &mut raw) })?;
        Ok(Self { raw, device })
    }

    /// Adapter description in the reference's terms.
    pub fn adapter_info(&self) -> GpuAdapterInfo {
        GpuAdapterInfo {
            name: format!("CUDA device {}", self.device),
            backend: "CUDA".to_string(),
            device_type: "DiscreteGpu".to_string(),
            driver: "toaster_cuda (sm_100a)".to_string(),
            driver_info: format!("C ABI version {}", unsafe { ffi::tc_abi_version() }),
        }
    }

    /// Uploads a whole scene (replaces `create_scene_gpu_buffers` + the first `write_buffer`s).
    /// With `with_bvh` the caller's flattened hierarchy is used, else the library builds the same
    /// median-split tree itself.
    pub fn upload(&mut self, scene: &SceneGpuData, with_bvh: bool) -> Result<()> {
        let sd = TcSceneData::borrow(scene, with_bvh);
        // SAFETY: `sd` borrows `scene`'s arrays for the duration of the call; the library copies them.
        ffi::check(self.raw, unsafe { ffi::tc_upload_scene(self.raw, &sd) })
    }

    /// Applies an evaluated frame's changes (replaces the per-frame `write_buffer`s of
    /// path_tracer.rs:676-721): changed geometry is copied and the hierarchy refit on the device.
    pub fn update(&mut self, scene: &SceneGpuData, changes: SceneChanges) -> Result<()> {
        let sd = TcSceneData::borrow(scene, false);
        let ch = TcSceneChanges {
            camera: changes.camera as u32,
            spheres: changes.spheres as u32,
            triangles: changes.triangles as u32,
            emissive_geometry: changes.emissive_geometry as u32,
        };
        // SAFETY: as in `upload`.
        ffi::check(self.raw, unsafe { ffi::tc_update_geometry(self.raw, &sd, &ch) })
    }

    /// Traces `params.samples` paths per pixel (replaces `dispatch_compute_2d`, dispatch.rs:28-60).
    pub fn render(&mut self, params: &GpuRenderParams, options: &TcRenderOptions) -> Result<()> {
        // SAFETY: both pointers are valid for the call.
        ffi::check(self.raw, unsafe { ffi::tc_render(self.raw, params, options) })
    }

    /// Linear HDR float4 pixels of the accumulation (replaces `readback_pixels`, readback.rs:8-25).
    pub fn readback(&mut self, width: u32, height: u32) -> Result<Vec<[f32; 4]>> {
        let n = width as usize * height as usize;
        let mut pixels = vec![[0.0f32; 4]; n];
        // SAFETY: the buffer holds 4 * n floats.
        ffi::check(self.raw, unsafe { ffi::tc_readback(self.raw, pixels.as_mut_ptr().cast(), 4 * n) })?;
        Ok(pixels)
    }

    /// Display image converted on the device (exposure, ACES fitted, sRGB), the bytes
    /// `pixels_to_rgba_image` (image_output.rs:59) produces on the host.
    pub fn readback_rgba8(&mut self, width: u32, height: u32, exposure_stops: f32) -> Result<RgbaImage> {
        let n = width as usize * height as usize * 4;
        let mut bytes = vec![0u8; n];
        // SAFETY: the buffer holds n bytes.
        ffi::check(self.raw, unsafe { ffi::tc_readback_rgba8(self.raw, exposure_stops, bytes.as_mut_ptr(), n) })?;
        let image = RgbaImage::from_raw(width, height, bytes);
        ensure!(image.is_some(), "RGBA8 readback does not match {width}x{height}");
        Ok(image.unwrap())
    }

    /// Counters and device times of the last call.
    pub fn stats(&self) -> Result<TcStats> {
        let mut s = TcStats::default();
        // SAFETY: `s` is a valid out pointer.
        ffi::check(self.raw, unsafe { ffi::tc_get_stats(self.raw, &mut s) })?;
        Ok(s)
    }

    /// The raw handle, for calls this wrapper does not cover.
    pub fn raw(&self) -> *mut TcContext {
        self.raw
    }
}

impl Drop for CudaContext {
    fn drop(&mut self) {
        // SAFETY: `raw` came from tc_create and is destroyed once.
        unsafe {
            ffi::tc_destroy(self.raw);
        }
    }
}
