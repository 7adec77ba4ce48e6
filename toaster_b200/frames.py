"""The frame loop of toaster-gpu over the CUDA library: schedules, frame sinks and evaluators.

Mirrors the public surface of ``toaster_gpu`` (crates/toaster-gpu/src/lib.rs:28-37) so a host that
drives the reference through it can switch backends:

- ``AnimationConfig`` and ``frame_output_path`` (crates/toaster-gpu/src/animation.rs:8-153);
- ``FrameSink`` / ``CompletedFrame`` / ``GpuFrameTimings`` (path_tracer.rs:30-180), the PNG and
  benchmark sinks (:183-255) and an MJPEG sink like the preview server's stream
  (crates/toaster-server/src/routes.rs:82-110) fed by the device JPEG encoder;
- ``render_evaluated_gpu_animation``, ``render_evaluated_gpu_video`` (Motion-JPEG AVI),
  ``render_evaluated_gpu_animation_with_sink``, ``render_gpu_progressive_with_sink`` and
  ``benchmark_gpu_evaluator`` (:268-515), all running the
  loop of ``render_gpu_with_sink`` (:517-840): evaluate, pack, update the device scene, render,
  convert for display, deliver, record timings;
- the path-based helpers ``render_scene_gpu``, ``render_scene_gpu_animation``,
  ``render_scene_gpu_video``, ``render_scene_gpu_animation_with_sink``,
  ``render_gpu_animation_with_sink`` and ``benchmark_gpu_scene``, over the native scene loader.

Differences by design: the display conversion runs on the device inside ``readback`` (the
``conversion`` timing is zero); a frame whose geometry changed is re-uploaded, which rebuilds
the hierarchy (on the device from 4,096 primitives), or, with ``hierarchy="refit"``, refit on
the device; device kernel time is reported beside the host stage timings. A scene evaluator is
any object with ``evaluate(time_seconds, loop_cycle) -> EvaluatedScene``: the reference's
animation tracks and physics are not part of this package.
"""

from __future__ import annotations

import dataclasses
import math
import time
from pathlib import Path
from typing import Callable, Optional, Union

import numpy as np

from .renderer import GpuRenderer, progressive_batch, render_frame_seed
from .scene import Scene, SceneGpuData, scene_to_gpu
from .stream import AviMjpegWriter, encode_png, mjpeg_part


class FramePacing:
    """Frame pacing of the loop (path_tracer.rs): as fast as possible, or one frame per 1/fps."""

    UNPACED = "unpaced"
    REAL_TIME = "realtime"


# ------------------------------------------------------------------------------------ schedules
@dataclasses.dataclass(frozen=True)
class AnimationConfig:
    """Frame schedule (animation.rs:8-133): optional FPS, optional frame limit, optional loop."""

    fps: Optional[int] = None
    frame_limit: Optional[int] = 1
    loop_duration_seconds: Optional[float] = None

    @staticmethod
    def single_frame() -> "AnimationConfig":
        return AnimationConfig(None, 1, None)

    @staticmethod
    def from_duration(fps: int, duration_seconds: float) -> "AnimationConfig":
        _validate_fps(fps)
        d = float(np.float32(duration_seconds))
        if not math.isfinite(d) or d <= 0.0:
            raise ValueError("duration must be finite and greater than zero")
        count = math.ceil(float(fps) * d)
        if count > 0xFFFFFFFF:
            raise ValueError("animation frame count is too large")
        return AnimationConfig(fps, count, None)

    @staticmethod
    def from_frame_count(fps: int, frame_count: int) -> "AnimationConfig":
        _validate_fps(fps)
        if frame_count <= 0:
            raise ValueError("frames must be greater than zero")
        return AnimationConfig(fps, frame_count, None)

    @staticmethod
    def indefinite(fps: int) -> "AnimationConfig":
        _validate_fps(fps)
        return AnimationConfig(fps, None, None)

    def with_loop_duration(self, duration_seconds: float) -> "AnimationConfig":
        d = float(np.float32(duration_seconds))
        if not math.isfinite(d) or d <= 0.0:
            raise ValueError("loop duration must be finite and greater than zero")
        return dataclasses.replace(self, loop_duration_seconds=d)

    def evaluation_request(self, frame: int) -> tuple:
        """(time in seconds as f32, loop cycle) of a frame: frame / fps in f64, wrapped by the loop."""
        absolute = 0.0 if self.fps is None else frame / float(self.fps)
        if self.loop_duration_seconds is None:
            return float(np.float32(absolute)), 0
        d = float(self.loop_duration_seconds)
        cycle = math.floor(absolute / d)
        return float(np.float32(absolute - cycle * d)), int(cycle)

    def time_for_frame(self, frame: int) -> float:
        return self.evaluation_request(frame)[0]


def _validate_fps(fps: int) -> None:
    if fps <= 0:
        raise ValueError("fps must be greater than zero")


def frame_output_path(out_path, frame: int, frame_count: int) -> Path:
    """``out.png`` for a single frame, else ``out_0007.png`` (animation.rs:135-153)."""
    out_path = Path(out_path)
    if frame_count == 1:
        return out_path
    stem = out_path.stem or "frame"
    ext = out_path.suffix[1:] if out_path.suffix else "png"
    return out_path.parent / f"{stem}_{frame:04d}.{ext}"


@dataclasses.dataclass(frozen=True)
class ProgressiveRenderConfig:
    """Exact accumulated-sample target of a static progressive render (path_tracer.rs:110-129)."""

    target_samples: int

    def __post_init__(self):
        if self.target_samples <= 0:
            raise ValueError("progressive target samples must be greater than zero")


@dataclasses.dataclass(frozen=True)
class GpuBenchmarkConfig:
    """Warm-up and measured frame counts of a benchmark (path_tracer.rs:57-92)."""

    warmup_frames: int
    measured_frames: int

    def __post_init__(self):
        if self.measured_frames <= 0:
            raise ValueError("benchmark measured frame count must be greater than zero")
        if self.warmup_frames < 0:
            raise ValueError("benchmark warm-up frame count must not be negative")


# ---------------------------------------------------------------------------- frames and sinks
@dataclasses.dataclass
class GpuFrameTimings:
    """Stage timings of one frame in seconds (path_tracer.rs:30-56), plus the device kernel time."""

    animation_evaluation: float = 0.0
    physics_evaluation: float = 0.0
    geometry_update: float = 0.0
    light_rebuild: float = 0.0
    bvh_rebuild: float = 0.0
    gpu_upload: float = 0.0
    scene_update_upload: float = 0.0
    dispatch_wait: float = 0.0
    readback: float = 0.0
    conversion: float = 0.0
    output: float = 0.0
    total: float = 0.0
    kernel_ms: float = 0.0


@dataclasses.dataclass
class CompletedFrame:
    """One converted frame handed to a sink (path_tracer.rs:132-160)."""

    index: int
    time_seconds: float
    width: int
    height: int
    samples: int
    accumulated_samples: int
    max_bounces: int
    timings: GpuFrameTimings
    render_time: float
    image: Optional[np.ndarray]  # (height, width, 4) uint8, valid only during deliver(); None for JPEG sinks
    counters: dict
    jpeg: Optional[bytes] = None  # the frame as JPEG bytes, for sinks that ask for them


class FrameSink:
    """Consumer of completed frames (path_tracer.rs:162-180); delivery applies backpressure.

    A sink whose ``jpeg_quality`` is set receives the frame JPEG-encoded on the device
    (``CompletedFrame.jpeg``) instead of RGBA8 pixels, as a preview stream wants it."""

    jpeg_quality: Optional[int] = None

    def deliver(self, frame: CompletedFrame) -> None:
        raise NotImplementedError

    def should_continue(self) -> bool:
        return True

    def samples_for_frame(self) -> Optional[int]:
        return None

    def record_timings(self, frame_index: int, timings: GpuFrameTimings) -> None:
        pass


class PngFrameSink(FrameSink):
    """Writes each frame as a PNG named by ``frame_output_path`` (path_tracer.rs:183-204)."""

    def __init__(self, out_path, frame_count: int):
        self.out_path, self.frame_count = Path(out_path), frame_count
        self.written = []

    def deliver(self, frame: CompletedFrame) -> None:
        path = frame_output_path(self.out_path, frame.index, self.frame_count)
        path.write_bytes(encode_png(frame.image))
        self.written.append(path)


class MjpegFrameSink(FrameSink):
    """Writes every frame as one ``multipart/x-mixed-replace`` part to a binary stream, the way the
    reference's preview server publishes frames (crates/toaster-server/src/routes.rs:82-110); the
    JPEG is made on the device. ``max_frames`` ends the stream after that many frames."""

    def __init__(self, stream, quality: int = 85, max_frames: Optional[int] = None):
        self.stream, self.jpeg_quality, self.max_frames = stream, quality, max_frames
        self.frames = 0

    def deliver(self, frame: CompletedFrame) -> None:
        self.stream.write(mjpeg_part(frame.jpeg))
        self.frames += 1

    def should_continue(self) -> bool:
        return self.max_frames is None or self.frames < self.max_frames


class VideoFrameSink(FrameSink):
    """Motion-JPEG AVI video of every frame (path_tracer.rs:206-234 writes through ffmpeg; here the
    frames are JPEG-encoded on the device and muxed by AviMjpegWriter). ``finish`` closes it."""

    def __init__(self, path, width: int, height: int, fps: int, quality: int = 90):
        self.writer = AviMjpegWriter(path, width, height, fps)
        self.jpeg_quality = quality

    def deliver(self, frame: CompletedFrame) -> None:
        self.writer.write_frame(frame.jpeg)

    def finish(self) -> None:
        self.writer.close()


class BenchmarkFrameSink(FrameSink):
    """Keeps measured timings and the last measured image (path_tracer.rs:236-255)."""

    def __init__(self, warmup_frames: int):
        self.warmup_frames = warmup_frames
        self.timings = []
        self.final_image = None

    def deliver(self, frame: CompletedFrame) -> None:
        if frame.index >= self.warmup_frames:
            self.final_image = frame.image.copy()

    def record_timings(self, frame_index: int, timings: GpuFrameTimings) -> None:
        if frame_index >= self.warmup_frames:
            self.timings.append(timings)


# ---------------------------------------------------------------------------------- evaluators
@dataclasses.dataclass
class SceneChanges:
    """What an evaluated frame changed (crates/toaster-scene/src/evaluation.rs:9-18)."""

    camera: bool = False
    spheres: bool = False
    triangles: bool = False
    emissive_geometry: bool = False

    def geometry(self) -> bool:
        return self.spheres or self.triangles


@dataclasses.dataclass
class EvaluatedScene:
    scene: Union[Scene, SceneGpuData]
    changes: SceneChanges = dataclasses.field(default_factory=SceneChanges)
    counters: dict = dataclasses.field(default_factory=dict)
    evaluation_seconds: float = 0.0
    exposure_stops: Optional[float] = None


class StaticSceneEvaluator:
    """A scene without animation: every request returns it unchanged."""

    def __init__(self, scene: Union[Scene, SceneGpuData], exposure_stops: Optional[float] = None):
        self.scene, self.exposure_stops = scene, exposure_stops

    def evaluate(self, time_seconds: float, loop_cycle: int = 0) -> EvaluatedScene:
        return EvaluatedScene(self.scene, SceneChanges(), exposure_stops=self.exposure_stops)


class FunctionSceneEvaluator:
    """Frames from a function of time; every frame after the first counts as moved geometry
    (and moved emitters when ``moving_lights``)."""

    def __init__(self, fn: Callable[[float], Union[Scene, SceneGpuData]], moving_lights: bool = True,
                 moving_camera: bool = False):
        self.fn, self.moving_lights, self.moving_camera = fn, moving_lights, moving_camera

    def evaluate(self, time_seconds: float, loop_cycle: int = 0) -> EvaluatedScene:
        t0 = time.perf_counter()
        scene = self.fn(time_seconds)
        ch = SceneChanges(self.moving_camera, True, True, self.moving_lights)
        return EvaluatedScene(scene, ch, evaluation_seconds=time.perf_counter() - t0)


def _counts(d: SceneGpuData) -> tuple:
    return (len(d.spheres), len(d.triangles), len(d.triangle_attributes), len(d.materials), len(d.lights))


def _pack(evaluated: EvaluatedScene) -> tuple:
    s = evaluated.scene
    t0 = time.perf_counter()
    if isinstance(s, SceneGpuData):
        return s, 0.0, (evaluated.exposure_stops or 0.0)
    data = scene_to_gpu(s)
    exposure = evaluated.exposure_stops if evaluated.exposure_stops is not None else getattr(s, "exposure_stops", 0.0)
    return data, time.perf_counter() - t0, exposure


# ----------------------------------------------------------------------------------- the loop
@dataclasses.dataclass
class GpuRenderSummary:
    setup_time: float
    frames: int


def render_gpu_with_sink(evaluator, animation: AnimationConfig, sink: FrameSink,
                         progressive: Optional[ProgressiveRenderConfig] = None, static_independent: bool = False,
                         pacing: str = "unpaced", hierarchy: str = "rebuild", device: int = 0,
                         renderer: Optional[GpuRenderer] = None) -> GpuRenderSummary:
    """The frame loop of path_tracer.rs:517-840 on the CUDA library."""
    if pacing not in ("unpaced", "realtime"):
        raise ValueError("pacing must be 'unpaced' or 'realtime'")
    if pacing == "realtime" and animation.fps is None:
        raise ValueError("real-time frame pacing requires an FPS")
    if hierarchy not in ("rebuild", "refit"):
        raise ValueError("hierarchy must be 'rebuild' or 'refit'")
    initial = evaluator.evaluate(*animation.evaluation_request(0))
    data, _, exposure = _pack(initial)
    counts = _counts(data)
    setup0 = time.perf_counter()
    own = renderer is None
    r = renderer if renderer is not None else GpuRenderer(device)
    try:
        r.upload(data)
        setup = time.perf_counter() - setup0
        started = time.perf_counter()
        frame, accumulated = 0, 0
        while animation.frame_limit is None or frame < animation.frame_limit:
            if not sink.should_continue():
                break
            f0 = time.perf_counter()
            timings = GpuFrameTimings()
            if progressive is not None or static_independent:
                t_sec, cycle = 0.0, 0
            else:
                t_sec, cycle = animation.evaluation_request(frame)
            if frame == 0 or progressive is not None:
                evaluated, changes = initial, SceneChanges()
            else:
                evaluated = evaluator.evaluate(t_sec, cycle)
                changes = evaluated.changes
                timings.animation_evaluation = evaluated.evaluation_seconds
            u0 = time.perf_counter()
            if frame > 0 and progressive is None:
                data, timings.geometry_update, exposure = _pack(evaluated)
                if _counts(data) != counts:
                    raise ValueError("evaluated scenes must preserve GPU geometry, material, light, and BVH "
                                     "primitive counts")
                g0 = time.perf_counter()
                if changes.geometry() or changes.emissive_geometry:
                    if hierarchy == "rebuild":
                        r.upload(data)
                    else:
                        r.update_geometry(data, camera=changes.camera, spheres=changes.spheres,
                                          triangles=changes.triangles, emissive_geometry=changes.emissive_geometry)
                elif changes.camera:
                    r.set_camera(data.camera)
                timings.gpu_upload = time.perf_counter() - g0
            timings.scene_update_upload = time.perf_counter() - u0
            requested = sink.samples_for_frame() or int(data.params["samples"][0])
            if requested <= 0:
                raise ValueError("frame sink sample count must be greater than zero")
            if progressive is not None:
                samples = progressive_batch(requested, accumulated, progressive.target_samples)
                if samples is None:
                    raise ValueError("progressive render is already complete")
            else:
                samples = requested
            d0 = time.perf_counter()
            r.render(samples=samples, frame_index=render_frame_seed(frame, static_independent),
                     accumulate=progressive is not None and accumulated > 0)
            timings.dispatch_wait = time.perf_counter() - d0
            timings.kernel_ms = float(r.stats()["kernel_ms"])
            b0 = time.perf_counter()
            image, jpeg = None, None
            if sink.jpeg_quality is not None:
                jpeg = r.encode_jpeg(int(sink.jpeg_quality), exposure)
            else:
                image = r.readback_rgba8(exposure)
            timings.readback = time.perf_counter() - b0
            render_time = time.perf_counter() - f0
            timings.total = render_time
            completed = accumulated + samples if progressive is not None else samples
            o0 = time.perf_counter()
            sink.deliver(CompletedFrame(frame, t_sec, r.width, r.height, samples, completed,
                                        int(data.params["max_bounces"][0]), timings, render_time, image,
                                        dict(evaluated.counters), jpeg))
            timings.output = time.perf_counter() - o0
            timings.total = time.perf_counter() - f0
            sink.record_timings(frame, timings)
            accumulated = completed
            if progressive is not None and accumulated >= progressive.target_samples:
                break
            nxt = frame + 1
            if (animation.frame_limit is not None and nxt >= animation.frame_limit) or not sink.should_continue():
                break
            if pacing == "realtime":
                delay = started + nxt / animation.fps - time.perf_counter()
                if delay > 0:
                    time.sleep(delay)
            frame = nxt
        return GpuRenderSummary(setup, frame + 1)
    finally:
        if own:
            r.close()


def render_evaluated_gpu_animation_with_sink(evaluator, animation: AnimationConfig, sink: FrameSink,
                                             pacing: str = "unpaced", **kw) -> None:
    render_gpu_with_sink(evaluator, animation, sink, pacing=pacing, **kw)


def render_evaluated_gpu_animation(evaluator, out_path, animation: AnimationConfig, **kw) -> list:
    """Every frame as a numbered PNG (path_tracer.rs:287-300); returns the written paths."""
    if animation.frame_limit is None:
        raise ValueError("PNG animation rendering requires a finite frame count")
    sink = PngFrameSink(out_path, animation.frame_limit)
    render_gpu_with_sink(evaluator, animation, sink, **kw)
    return sink.written


def render_evaluated_gpu_video(evaluator, video_path, animation: AnimationConfig, quality: int = 90, **kw) -> int:
    """Every frame into one Motion-JPEG AVI file (path_tracer.rs:316-356: finite frames and an
    FPS are required); returns the frame count. The file is finalised even if rendering fails."""
    if animation.fps is None:
        raise ValueError("video export requires an animated render with an FPS")
    if animation.frame_limit is None:
        raise ValueError("video export requires a finite frame count")
    first = evaluator.evaluate(*animation.evaluation_request(0)).scene
    params = first.params[0] if isinstance(first, SceneGpuData) else None
    width = int(params["width"]) if params is not None else first.width
    height = int(params["height"]) if params is not None else first.height
    sink = VideoFrameSink(video_path, width, height, animation.fps, quality)
    try:
        render_gpu_with_sink(evaluator, animation, sink, **kw)
    finally:
        sink.finish()
    return sink.writer.frames


def render_gpu_progressive_with_sink(scene: Union[Scene, SceneGpuData], schedule: AnimationConfig,
                                     config: ProgressiveRenderConfig, sink: FrameSink, pacing: str = "unpaced",
                                     **kw) -> None:
    """Static progressive accumulation to exactly the target (path_tracer.rs:391-430)."""
    if schedule.loop_duration_seconds is not None:
        raise ValueError("progressive preview does not support an animation loop duration")
    render_gpu_with_sink(StaticSceneEvaluator(scene), schedule, sink, progressive=config, pacing=pacing, **kw)


@dataclasses.dataclass
class GpuBenchmarkResult:
    """Setup time, per-frame timings of the measured frames and the last measured image
    (path_tracer.rs:94-108)."""

    setup_time: float
    frames: list
    final_image: np.ndarray


def benchmark_gpu_evaluator(evaluator, config: GpuBenchmarkConfig, **kw) -> GpuBenchmarkResult:
    """Static independent frames at time 0 with seed 0 (path_tracer.rs:474-515)."""
    schedule = AnimationConfig.from_frame_count(1, config.warmup_frames + config.measured_frames)
    sink = BenchmarkFrameSink(config.warmup_frames)
    summary = render_gpu_with_sink(evaluator, schedule, sink, static_independent=True, **kw)
    if len(sink.timings) != config.measured_frames:
        raise RuntimeError("GPU benchmark completed without all requested measurements")
    if sink.final_image is None:
        raise RuntimeError("GPU benchmark did not produce a measured image")
    return GpuBenchmarkResult(summary.setup_time, sink.timings, sink.final_image)


# ------------------------------------------------------------------------ path-based helpers
def _static_file_evaluator(scene_path) -> StaticSceneEvaluator:
    """A scene file's frames for the path-based helpers: loaded and packed by the native loader.
    Animation tracks would need toaster-scene's evaluator, which this package does not include."""
    import json

    from .scene import load_scene_gpu

    doc = json.loads(Path(scene_path).read_text(encoding="utf-8"))
    if isinstance(doc, dict) and ((doc.get("animation") or {}).get("tracks") or []):
        raise ValueError("the scene has animation tracks: evaluate them with an evaluator and call "
                         "render_evaluated_gpu_animation")
    data, exposure = load_scene_gpu(scene_path)
    return StaticSceneEvaluator(data, exposure)


def render_scene_gpu(scene_path, out_path, **kw) -> list:
    """One frame of a scene file as PNG (path_tracer.rs:266-268)."""
    return render_scene_gpu_animation(scene_path, out_path, AnimationConfig.single_frame(), **kw)


def render_scene_gpu_animation(scene_path, out_path, animation: AnimationConfig, **kw) -> list:
    """Numbered PNG frames of a scene file (path_tracer.rs:270-283)."""
    return render_evaluated_gpu_animation(_static_file_evaluator(scene_path), out_path, animation, **kw)


def render_scene_gpu_video(scene_path, video_path, animation: AnimationConfig, **kw) -> int:
    """A scene file as Motion-JPEG AVI video (path_tracer.rs:302-314)."""
    return render_evaluated_gpu_video(_static_file_evaluator(scene_path), video_path, animation, **kw)


def render_scene_gpu_animation_with_sink(scene_path, animation: AnimationConfig, pacing: str, sink: FrameSink,
                                         **kw) -> None:
    """A scene file's frames into a sink (path_tracer.rs:358-372)."""
    render_gpu_with_sink(_static_file_evaluator(scene_path), animation, sink, pacing=pacing, **kw)


def render_gpu_animation_with_sink(scene: Union[Scene, SceneGpuData], animation: AnimationConfig, pacing: str,
                                   sink: FrameSink, **kw) -> None:
    """A loaded scene's frames into a sink (path_tracer.rs:374-389)."""
    render_gpu_with_sink(StaticSceneEvaluator(scene), animation, sink, pacing=pacing, **kw)


def benchmark_gpu_scene(scene, config: GpuBenchmarkConfig, **kw) -> GpuBenchmarkResult:
    """Benchmark frames of a scene file or a loaded scene (path_tracer.rs:460-472)."""
    ev = _static_file_evaluator(scene) if isinstance(scene, (str, Path)) else StaticSceneEvaluator(scene)
    return benchmark_gpu_evaluator(ev, config, **kw)
