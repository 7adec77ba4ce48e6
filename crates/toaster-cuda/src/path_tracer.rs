//! The frame loop of `toaster_gpu` (crates/toaster-gpu/src/path_tracer.rs:518-849) with its device
//! work done by the CUDA library: same schedules, evaluators, sinks, progressive contract, seeds
//! and timing fields; the wgpu buffers, bind groups, pipeline, dispatch, map-and-copy readback
//! and host display conversion are replaced by `tc_upload_scene` / `tc_render` /
//! `tc_readback_rgba8`.

use std::path::Path;
use std::process::{Child, ChildStdin, Command, Stdio};
use std::time::{Duration, Instant};

use anyhow::{anyhow, ensure, Context, Result};
use image::RgbaImage;
use std::io::Write;
use toaster_gpu::image_output::save_rgba_image_to_png;
use toaster_gpu::scene_upload::scene_to_gpu;
use toaster_gpu::{
    frame_output_path, AnimationConfig, CompletedFrame, FramePacing, FrameSink, GpuBenchmarkConfig,
    GpuBenchmarkResult, GpuFrameTimings, ProgressiveRenderConfig,
};
use toaster_scene::{AnimationEvaluator, EvaluationRequest, SceneChanges, SceneEvaluationTimings, SceneEvaluator};

use crate::context::CudaContext;
use crate::ffi::TcRenderOptions;

/// Device ordinal used by the entry points (`TOASTER_CUDA_DEVICE`, default 0).
fn device_ordinal() -> i32 {
    std::env::var("TOASTER_CUDA_DEVICE").ok().and_then(|v| v.parse().ok()).unwrap_or(0)
}

#[derive(Clone, Copy, PartialEq, Eq)]
enum FrameMode {
    Animated,
    StaticIndependent,
}

/// Renders a scene's time-zero frame to a PNG.
pub async fn render_scene_gpu(scene_path: &Path, out_path: &Path) -> Result<()> {
    render_scene_gpu_animation(scene_path, out_path, AnimationConfig::single_frame()).await
}

/// Renders a finite animation schedule to numbered PNG files.
pub async fn render_scene_gpu_animation(scene_path: &Path, out_path: &Path, animation: AnimationConfig) -> Result<()> {
    let source_scene = toaster_scene::load_scene(scene_path)?;
    ensure!(
        !source_scene.physics.is_some_and(|physics| physics.enabled),
        "path-based GPU helpers do not evaluate enabled physics; use an evaluator-driven entrypoint"
    );
    let mut evaluator = AnimationEvaluator::new(source_scene);
    render_evaluated_gpu_animation(&mut evaluator, out_path, animation).await
}

/// Renders a finite evaluator-driven schedule to numbered PNG files.
pub async fn render_evaluated_gpu_animation(
    evaluator: &mut dyn SceneEvaluator,
    out_path: &Path,
    animation: AnimationConfig,
) -> Result<()> {
    let frame_count = animation.frame_limit().context("PNG animation rendering requires a finite frame count")?;
    let mut sink = PngFrameSink { out_path, frame_count };
    render_evaluated_gpu_animation_with_sink(evaluator, animation, FramePacing::Unpaced, &mut sink).await
}

/// Renders a finite animation and streams its RGBA frames into an MP4 encoder.
pub async fn render_scene_gpu_video(scene_path: &Path, video_path: &Path, animation: AnimationConfig) -> Result<()> {
    let source_scene = toaster_scene::load_scene(scene_path)?;
    ensure!(
        !source_scene.physics.is_some_and(|physics| physics.enabled),
        "path-based GPU helpers do not evaluate enabled physics; use an evaluator-driven entrypoint"
    );
    let mut evaluator = AnimationEvaluator::new(source_scene);
    render_evaluated_gpu_video(&mut evaluator, video_path, animation).await
}

/// Renders a finite evaluator-driven schedule into an MP4 encoder (FFmpeg on the PATH).
pub async fn render_evaluated_gpu_video(
    evaluator: &mut dyn SceneEvaluator,
    video_path: &Path,
    animation: AnimationConfig,
) -> Result<()> {
    let fps = animation.fps().context("video export requires an animated render with --fps")?;
    ensure!(animation.frame_limit().is_some(), "video export requires a finite --duration or --frames");
    let width = evaluator.source_scene().render.width;
    let height = evaluator.source_scene().render.height;
    let mut sink = VideoFrameSink { writer: Some(FfmpegWriter::start(video_path, width, height, fps)?) };
    let render_result = render_evaluated_gpu_animation_with_sink(evaluator, animation, FramePacing::Unpaced, &mut sink).await;
    let finish_result = sink.finish();
    match (render_result, finish_result) {
        (Ok(()), Ok(())) => Ok(()),
        (Err(e), Ok(())) | (Ok(()), Err(e)) => Err(e),
        (Err(render_error), Err(finish_error)) => {
            Err(anyhow!("{render_error:#}; video finalization also failed: {finish_error:#}"))
        }
    }
}

/// Loads a scene and renders its animation through a caller-provided sink.
pub async fn render_scene_gpu_animation_with_sink(
    scene_path: &Path,
    animation: AnimationConfig,
    pacing: FramePacing,
    sink: &mut dyn FrameSink,
) -> Result<()> {
    validate_pacing(animation, pacing)?;
    let source_scene = toaster_scene::load_scene(scene_path)?;
    ensure!(
        !source_scene.physics.is_some_and(|physics| physics.enabled),
        "path-based GPU helpers do not evaluate enabled physics; use an evaluator-driven entrypoint"
    );
    render_gpu_animation_with_sink(&source_scene, animation, pacing, sink).await
}

/// Renders an already loaded scene as independent animation frames.
pub async fn render_gpu_animation_with_sink(
    source_scene: &toaster_scene::Scene,
    animation: AnimationConfig,
    pacing: FramePacing,
    sink: &mut dyn FrameSink,
) -> Result<()> {
    ensure!(
        !source_scene.physics.is_some_and(|physics| physics.enabled),
        "scene-only GPU helpers do not evaluate enabled physics; use an evaluator-driven entrypoint"
    );
    let mut evaluator = AnimationEvaluator::new(source_scene.clone());
    render_evaluated_gpu_animation_with_sink(&mut evaluator, animation, pacing, sink).await
}

/// Renders frames supplied by a renderer-neutral scene evaluator.
pub async fn render_evaluated_gpu_animation_with_sink(
    evaluator: &mut dyn SceneEvaluator,
    animation: AnimationConfig,
    pacing: FramePacing,
    sink: &mut dyn FrameSink,
) -> Result<()> {
    render_cuda_with_sink(evaluator, animation, pacing, None, FrameMode::Animated, sink).map(|_| ())
}

/// Accumulates a static scene in linear HDR batches and delivers each update.
pub async fn render_gpu_progressive_with_sink(
    source_scene: &toaster_scene::Scene,
    schedule: AnimationConfig,
    pacing: FramePacing,
    config: ProgressiveRenderConfig,
    sink: &mut dyn FrameSink,
) -> Result<()> {
    ensure!(schedule.loop_duration().is_none(), "progressive preview does not support an animation loop duration");
    ensure!(
        !source_scene.physics.is_some_and(|physics| physics.enabled),
        "progressive preview does not support physics-enabled scenes"
    );
    ensure!(source_scene.animation.tracks.is_empty(), "progressive preview requires a scene without animation tracks");
    let mut evaluator = AnimationEvaluator::new(source_scene.clone());
    render_cuda_with_sink(&mut evaluator, schedule, pacing, Some(config), FrameMode::Animated, sink).map(|_| ())
}

/// Benchmarks static independent frames using one device setup.
pub async fn benchmark_gpu_scene(source_scene: &toaster_scene::Scene, config: GpuBenchmarkConfig) -> Result<GpuBenchmarkResult> {
    ensure!(
        !source_scene.physics.is_some_and(|physics| physics.enabled),
        "scene-only GPU benchmarks do not evaluate enabled physics; use an evaluator-driven benchmark"
    );
    let mut evaluator = AnimationEvaluator::new(source_scene.clone());
    benchmark_gpu_evaluator(&mut evaluator, config).await
}

/// Benchmarks evaluator-produced time-zero frames using one device setup.
pub async fn benchmark_gpu_evaluator(
    evaluator: &mut dyn SceneEvaluator,
    config: GpuBenchmarkConfig,
) -> Result<GpuBenchmarkResult> {
    let total_frames =
        config.warmup_frames().checked_add(config.measured_frames()).context("benchmark frame count overflowed")?;
    let schedule = AnimationConfig::from_frame_count(1, total_frames)?;
    let measured = usize::try_from(config.measured_frames()).context("benchmark measured frame count is too large")?;
    let mut sink = BenchmarkFrameSink { warmup_frames: config.warmup_frames(), timings: Vec::with_capacity(measured), final_image: None };
    let summary = render_cuda_with_sink(evaluator, schedule, FramePacing::Unpaced, None, FrameMode::StaticIndependent, &mut sink)?;
    ensure!(sink.timings.len() == measured, "GPU benchmark completed without all requested measurements");
    let final_image = sink.final_image.context("GPU benchmark did not produce a measured image")?;
    Ok(GpuBenchmarkResult { adapter: summary.adapter, setup_time: summary.setup_time, frames: sink.timings, final_image })
}

struct RenderSummary {
    adapter: toaster_gpu::GpuAdapterInfo,
    setup_time: Duration,
}

/// The shared single-setup loop of every sink-driven mode.
fn render_cuda_with_sink(
    evaluator: &mut dyn SceneEvaluator,
    animation: AnimationConfig,
    pacing: FramePacing,
    progressive: Option<ProgressiveRenderConfig>,
    frame_mode: FrameMode,
    sink: &mut dyn FrameSink,
) -> Result<RenderSummary> {
    validate_pacing(animation, pacing)?;
    let initial = evaluator.evaluate(animation.evaluation_request(0))?;
    let initial_counters = initial.counters.clone();
    let initial_scene = initial.scene;
    let display = initial_scene.display;
    let mut scene = scene_to_gpu(&initial_scene)?;
    let counts = |s: &toaster_gpu::scene_upload::SceneGpuData| {
        (s.spheres.len(), s.triangles.len(), s.triangle_attributes.len(), s.materials.len(), s.lights.len(),
         s.bvh_primitives.len())
    };
    let initial_counts = counts(&scene);

    let setup_start = Instant::now();
    let mut ctx = CudaContext::new(device_ordinal())?;
    // The reference's own flattened hierarchy goes to the device, so hits follow its traversal.
    ctx.upload(&scene, true)?;
    let setup_time = setup_start.elapsed();
    let options = TcRenderOptions::default();

    let pacing_started_at = Instant::now();
    let mut frame = 0_u32;
    let mut accumulated_samples = 0_u32;
    while animation.frame_limit().is_none_or(|limit| frame < limit) {
        if !sink.should_continue() {
            break;
        }
        let frame_start = Instant::now();
        let request = if progressive.is_some() || frame_mode == FrameMode::StaticIndependent {
            EvaluationRequest { time_seconds: 0.0, loop_cycle: 0 }
        } else {
            animation.evaluation_request(frame)
        };
        let time_seconds = request.time_seconds;
        let (changes, evaluation_timings, counters, bvh_rebuild) = if progressive.is_some() || frame == 0 {
            (SceneChanges::default(), SceneEvaluationTimings::default(), initial_counters.clone(), Duration::ZERO)
        } else {
            let evaluated = evaluator.evaluate(request)?;
            let pack_start = Instant::now();
            let next = scene_to_gpu(&evaluated.scene)?;
            let packed = pack_start.elapsed();
            ensure!(
                counts(&next) == initial_counts,
                "evaluated scenes must preserve GPU geometry, material, light, and BVH primitive counts"
            );
            scene = next;
            (evaluated.changes, evaluated.timings, evaluated.counters, packed)
        };
        let requested = sink.samples_for_frame().unwrap_or(scene.params.samples);
        ensure!(requested > 0, "frame sink sample count must be greater than zero");
        scene.params.samples = match progressive {
            Some(config) => progressive_batch(requested, accumulated_samples, config.target_samples())?
                .context("progressive render is already complete")?,
            None => requested,
        };
        scene.params.frame_index = match frame_mode {
            FrameMode::Animated => frame,
            FrameMode::StaticIndependent => 0,
        };
        scene.params.accumulated_samples = if progressive.is_some() { accumulated_samples } else { 0 };

        let upload_start = Instant::now();
        if changes.spheres || changes.triangles || changes.emissive_geometry {
            ctx.upload(&scene, true)?;
        } else if changes.camera {
            ctx.update(&scene, changes)?;
        }
        let gpu_upload = upload_start.elapsed();
        let scene_update_upload = frame_start.elapsed();

        let dispatch_start = Instant::now();
        ctx.render(&scene.params, &options)?;
        let dispatch_wait = dispatch_start.elapsed();
        let readback_start = Instant::now();
        let image = ctx.readback_rgba8(scene.params.width, scene.params.height, display.exposure_stops)?;
        let readback = readback_start.elapsed();
        let render_time = frame_start.elapsed();
        let mut timings = GpuFrameTimings {
            animation_evaluation: evaluation_timings.animation_evaluation,
            physics_evaluation: evaluation_timings.physics_evaluation,
            geometry_update: evaluation_timings.geometry_update,
            light_rebuild: Duration::ZERO,
            bvh_rebuild,
            gpu_upload,
            scene_update_upload,
            dispatch_wait,
            readback,
            conversion: Duration::ZERO, // converted on the device inside `readback`
            output: Duration::ZERO,
            total: render_time,
        };
        let completed_samples = if progressive.is_some() {
            accumulated_samples.checked_add(scene.params.samples).context("progressive accumulated sample count overflowed")?
        } else {
            scene.params.samples
        };
        let output_start = Instant::now();
        sink.deliver(CompletedFrame {
            index: frame,
            time_seconds,
            width: scene.params.width,
            height: scene.params.height,
            samples: scene.params.samples,
            accumulated_samples: completed_samples,
            max_bounces: scene.params.max_bounces,
            timings,
            render_time,
            image: &image,
            counters: &counters,
        })?;
        timings.output = output_start.elapsed();
        timings.total = frame_start.elapsed();
        sink.record_timings(frame, timings);

        accumulated_samples = completed_samples;
        if progressive.is_some_and(|config| accumulated_samples >= config.target_samples()) {
            break;
        }
        let next_frame = frame.checked_add(1).context("render frame index exceeded the supported range")?;
        if !animation.frame_limit().is_none_or(|limit| next_frame < limit) || !sink.should_continue() {
            break;
        }
        if pacing == FramePacing::RealTime {
            let fps = animation.fps().context("real-time frame pacing requires an FPS")?;
            let deadline = pacing_started_at + Duration::from_secs_f64(next_frame as f64 / fps as f64);
            if let Some(delay) = deadline.checked_duration_since(Instant::now()) {
                std::thread::sleep(delay);
            }
        }
        frame = next_frame;
    }
    Ok(RenderSummary { adapter: ctx.adapter_info(), setup_time })
}

/// The progressive contract of path_tracer.rs:900-923: the next batch, clamped to the target.
fn progressive_batch(requested: u32, accumulated: u32, target: u32) -> Result<Option<u32>> {
    ensure!(requested > 0, "sample batch must be greater than zero");
    ensure!(target > 0, "sample target must be greater than zero");
    ensure!(accumulated <= target, "accumulated samples exceed the progressive target");
    if accumulated == target {
        return Ok(None);
    }
    Ok(Some(requested.min(target - accumulated)))
}

fn validate_pacing(animation: AnimationConfig, pacing: FramePacing) -> Result<()> {
    if pacing == FramePacing::RealTime {
        ensure!(animation.fps().is_some(), "real-time frame pacing requires an FPS");
    }
    Ok(())
}

/// Numbered PNG output (the reference's PNG sink).
struct PngFrameSink<'a> {
    out_path: &'a Path,
    frame_count: u32,
}

impl FrameSink for PngFrameSink<'_> {
    fn deliver(&mut self, frame: CompletedFrame<'_>) -> Result<()> {
        save_rgba_image_to_png(frame.image, &frame_output_path(self.out_path, frame.index, self.frame_count))
    }
}

/// Benchmark sink: keeps measured timings and the last measured image.
struct BenchmarkFrameSink {
    warmup_frames: u32,
    timings: Vec<GpuFrameTimings>,
    final_image: Option<RgbaImage>,
}

impl FrameSink for BenchmarkFrameSink {
    fn deliver(&mut self, frame: CompletedFrame<'_>) -> Result<()> {
        if frame.index >= self.warmup_frames {
            self.final_image = Some(frame.image.clone());
        }
        Ok(())
    }

    fn record_timings(&mut self, frame_index: u32, timings: GpuFrameTimings) {
        if frame_index >= self.warmup_frames {
            self.timings.push(timings);
        }
    }
}

/// RGBA frames piped into an FFmpeg H.264 encoder.
struct FfmpegWriter {
    child: Child,
    stdin: Option<ChildStdin>,
}

impl FfmpegWriter {
    fn start(path: &Path, width: u32, height: u32, fps: u32) -> Result<Self> {
        let mut child = Command::new("ffmpeg")
            .args(["-y", "-loglevel", "error", "-f", "rawvideo", "-pix_fmt", "rgba", "-s"])
            .arg(format!("{width}x{height}"))
            .args(["-r", &fps.to_string(), "-i", "-", "-c:v", "libx264", "-pix_fmt", "yuv420p"])
            .arg(path)
            .stdin(Stdio::piped())
            .spawn()
            .context("failed to start ffmpeg for video export")?;
        let stdin = child.stdin.take();
        Ok(Self { child, stdin })
    }

    fn write(&mut self, image: &RgbaImage) -> Result<()> {
        let stdin = self.stdin.as_mut().context("video encoder input is closed")?;
        stdin.write_all(image.as_raw()).context("failed to write a frame to ffmpeg")
    }

    fn finish(mut self) -> Result<()> {
        drop(self.stdin.take());
        let status = self.child.wait().context("failed to wait for ffmpeg")?;
        ensure!(status.success(), "ffmpeg exited with {status}");
        Ok(())
    }
}

struct VideoFrameSink {
    writer: Option<FfmpegWriter>,
}

impl VideoFrameSink {
    fn finish(&mut self) -> Result<()> {
        match self.writer.take() {
            Some(w) => w.finish(),
            None => Ok(()),
        }
    }
}

impl FrameSink for VideoFrameSink {
    fn deliver(&mut self, frame: CompletedFrame<'_>) -> Result<()> {
        self.writer.as_mut().context("video encoder is closed")?.write(frame.image)
    }
}
