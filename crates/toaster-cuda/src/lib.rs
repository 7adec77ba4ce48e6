//! B200 (sm_100a) CUDA backend for toaster's GPU path tracing.
//!
//! The public functions have the signatures of `toaster_gpu`'s (crates/toaster-gpu/src/lib.rs:28-37)
//! so `toaster-cli` can switch backends with one flag; they take the same scene records
//! (`toaster_gpu::scene_upload::scene_to_gpu`), sinks and schedules. The device work is done by the
//! static library built from `toaster_b200/csrc` (`include/toaster_cuda.h`): hand-written CUDA
//! kernels for the traversal, the estimator, the FP64 accumulation and the display conversion.
//! There is no CPU fallback: without an sm_100 device the first call fails.

/// Raw declarations of the C ABI.
pub mod ffi;
/// Owned library context.
pub mod context;
/// Frame loop and the `toaster_gpu`-compatible entry points.
pub mod path_tracer;

pub use context::CudaContext;
pub use path_tracer::{
    benchmark_gpu_evaluator, benchmark_gpu_scene, render_evaluated_gpu_animation,
    render_evaluated_gpu_animation_with_sink, render_evaluated_gpu_video, render_gpu_animation_with_sink,
    render_gpu_progressive_with_sink, render_scene_gpu, render_scene_gpu_animation,
    render_scene_gpu_animation_with_sink, render_scene_gpu_video,
};
pub use toaster_gpu::{
    frame_output_path, AnimationConfig, CompletedFrame, FramePacing, FrameSink, GpuBenchmarkConfig,
    GpuBenchmarkResult, GpuFrameTimings, ProgressiveRenderConfig,
};
