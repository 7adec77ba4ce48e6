"""The host frame loop (toaster_b200.frames): schedules, sinks and the loop's contract (CPU).

Schedules restate the reference's own tests (crates/toaster-gpu/src/animation.rs:155-226). The
loop runs against a recording stand-in for GpuRenderer, which checks the calls the loop makes
(upload, refit, camera, render parameters, readback) and the reference loop's rules
(path_tracer.rs:517-840): progressive batches that land exactly on the target, seeds per frame,
sample overrides from the sink, cancellation, count preservation, PNG naming.
"""

import math

import numpy as np
import pytest

from toaster_b200 import configs
from toaster_b200.frames import (AnimationConfig, BenchmarkFrameSink, FrameSink, FunctionSceneEvaluator,
                                 GpuBenchmarkConfig, MjpegFrameSink, ProgressiveRenderConfig, StaticSceneEvaluator,
                                 benchmark_gpu_evaluator, frame_output_path, render_evaluated_gpu_animation,
                                 render_gpu_progressive_with_sink, render_gpu_with_sink)
from toaster_b200.scene import load_scene, scene_to_gpu


# ------------------------------------------------------------------- animation.rs:155-226
def test_duration_uses_ceiling_and_explicit_fps():
    a = AnimationConfig.from_duration(24, 1.01)
    assert a.frame_limit == 25 and a.time_for_frame(12) == 0.5
    assert AnimationConfig.from_duration(24, 1.1).frame_limit == 27


def test_frame_count_is_exact():
    a = AnimationConfig.from_frame_count(30, 17)
    assert a.frame_limit == 17 and a.fps == 30


def test_single_frame_has_no_inferred_fps():
    a = AnimationConfig.single_frame()
    assert a.fps is None and a.frame_limit == 1 and a.time_for_frame(0) == 0.0


def test_indefinite_animation_has_no_frame_limit():
    a = AnimationConfig.indefinite(12)
    assert a.fps == 12 and a.frame_limit is None and a.time_for_frame(24) == 2.0


def test_loop_duration_wraps_animation_time_without_wrapping_frame_count():
    a = AnimationConfig.indefinite(4).with_loop_duration(2.0)
    assert a.time_for_frame(7) == 1.75 and a.time_for_frame(8) == 0.0
    assert a.evaluation_request(8)[1] == 1 and a.time_for_frame(10) == 0.5
    assert a.frame_limit is None and a.loop_duration_seconds == 2.0


def test_rejects_invalid_timing():
    for bad in (lambda: AnimationConfig.from_duration(0, 1.0), lambda: AnimationConfig.from_duration(24, math.nan),
                lambda: AnimationConfig.from_duration(24, 0.0), lambda: AnimationConfig.from_frame_count(24, 0),
                lambda: AnimationConfig.indefinite(0), lambda: AnimationConfig.indefinite(24).with_loop_duration(math.nan),
                lambda: AnimationConfig.indefinite(24).with_loop_duration(0.0),
                lambda: ProgressiveRenderConfig(0), lambda: GpuBenchmarkConfig(1, 0)):
        with pytest.raises(ValueError):
            bad()


def test_frame_output_paths(tmp_path):
    assert frame_output_path(tmp_path / "out.png", 3, 1) == tmp_path / "out.png"
    assert frame_output_path(tmp_path / "out.png", 7, 240) == tmp_path / "out_0007.png"
    assert frame_output_path(tmp_path / "clip", 12, 30) == tmp_path / "clip_0012.png"


# ------------------------------------------------------------------------- the loop, recorded
class RecordingRenderer:
    """Stands in for GpuRenderer: records calls, returns an image that encodes the call count."""

    def __init__(self):
        self.calls = []
        self.width = self.height = 0
        self.accumulated = 0

    def upload(self, data):
        self.calls.append(("upload", len(data.spheres), len(data.triangles)))
        self.width, self.height = int(data.params["width"][0]), int(data.params["height"][0])
        self.accumulated = 0

    def update_geometry(self, data, camera=False, spheres=True, triangles=True, emissive_geometry=False):
        self.calls.append(("refit", camera, spheres, triangles, emissive_geometry))

    def set_camera(self, camera):
        self.calls.append(("camera",))

    def render(self, samples=None, frame_index=0, accumulate=False, **kw):
        if accumulate and self.accumulated == 0:
            raise AssertionError("accumulate without a previous batch")
        self.accumulated = (self.accumulated if accumulate else 0) + samples
        self.calls.append(("render", samples, frame_index, accumulate))

    def stats(self):
        return {"kernel_ms": 1.0}

    def encode_jpeg(self, quality=90, exposure_stops=0.0):
        self.calls.append(("jpeg", quality, exposure_stops))
        return b"\xff\xd8" + bytes([len(self.calls) % 256]) + b"\xff\xd9"

    def readback_rgba8(self, exposure_stops=0.0):
        self.calls.append(("readback", exposure_stops))
        return np.full((self.height, self.width, 4), len(self.calls) % 256, np.uint8)

    def close(self):
        raise AssertionError("the loop must not close a renderer it was given")


class ListSink(FrameSink):
    def __init__(self, stop_after=None, samples=None):
        self.frames, self.timings, self.stop_after, self.samples = [], [], stop_after, samples

    def deliver(self, frame):
        self.frames.append((frame.index, frame.time_seconds, frame.samples, frame.accumulated_samples,
                            frame.image.shape))

    def should_continue(self):
        return self.stop_after is None or len(self.frames) < self.stop_after

    def samples_for_frame(self):
        return self.samples

    def record_timings(self, index, timings):
        self.timings.append((index, timings.total >= timings.dispatch_wait >= 0))


def small_scene():
    s = configs.plain_small()
    s.width, s.height, s.samples = 16, 8, 5
    return s


def test_progressive_batches_land_exactly_on_the_target():
    r, sink = RecordingRenderer(), ListSink()
    render_gpu_progressive_with_sink(small_scene(), AnimationConfig.indefinite(30), ProgressiveRenderConfig(12), sink,
                                     renderer=r)
    renders = [c for c in r.calls if c[0] == "render"]
    assert [c[1] for c in renders] == [5, 5, 2]
    assert [c[2] for c in renders] == [0, 1, 2]  # animated seeds: the frame index
    assert [c[3] for c in renders] == [False, True, True]
    assert [f[3] for f in sink.frames] == [5, 10, 12] and r.accumulated == 12
    assert sum(1 for c in r.calls if c[0] == "upload") == 1  # static: one upload, no refit
    assert all(ok for _, ok in sink.timings)


def test_sink_overrides_samples_and_cancels():
    r, sink = RecordingRenderer(), ListSink(stop_after=2, samples=3)
    render_gpu_with_sink(StaticSceneEvaluator(small_scene()), AnimationConfig.from_frame_count(24, 10), sink,
                         renderer=r)
    assert [f[2] for f in sink.frames] == [3, 3] and len(sink.frames) == 2


def test_animated_frames_rebuild_or_refit_and_keep_counts():
    anim = configs.BallisticAnimation(width=32, height=18, samples=2, frames=4)
    ev = FunctionSceneEvaluator(lambda t: anim.scene(int(round(t * 24))))
    for hierarchy, kind in (("rebuild", "upload"), ("refit", "refit")):
        r, sink = RecordingRenderer(), ListSink()
        render_gpu_with_sink(ev, AnimationConfig.from_frame_count(24, 4), sink, hierarchy=hierarchy, renderer=r)
        assert [c[0] for c in r.calls if c[0] in ("upload", "refit")] == ["upload"] + [kind] * 3
        assert [f[1] for f in sink.frames] == [np.float32(k / 24) for k in range(4)]
        assert [c[2] for c in r.calls if c[0] == "render"] == [0, 1, 2, 3]
    grows = FunctionSceneEvaluator(lambda t: configs.plain_small() if t == 0 else configs.mixed())
    with pytest.raises(ValueError, match="preserve"):
        render_gpu_with_sink(grows, AnimationConfig.from_frame_count(24, 2), ListSink(), renderer=RecordingRenderer())


def test_benchmark_uses_seed_zero_and_measures_after_warmup():
    r = RecordingRenderer()
    res = benchmark_gpu_evaluator(StaticSceneEvaluator(small_scene()), GpuBenchmarkConfig(2, 3), renderer=r)
    assert len(res.frames) == 3 and res.final_image.shape == (8, 16, 4)
    assert [c[2] for c in r.calls if c[0] == "render"] == [0] * 5


def test_png_animation_names_every_frame(tmp_path):
    r = RecordingRenderer()
    written = render_evaluated_gpu_animation(StaticSceneEvaluator(small_scene(), exposure_stops=1.5),
                                             tmp_path / "clip.png", AnimationConfig.from_frame_count(24, 3),
                                             renderer=r)
    assert [p.name for p in written] == ["clip_0000.png", "clip_0001.png", "clip_0002.png"]
    assert all(p.read_bytes()[:8] == b"\x89PNG\r\n\x1a\n" for p in written)
    assert {c[1] for c in r.calls if c[0] == "readback"} == {1.5}
    with pytest.raises(ValueError, match="finite frame count"):
        render_evaluated_gpu_animation(StaticSceneEvaluator(small_scene()), tmp_path / "x.png",
                                       AnimationConfig.indefinite(24), renderer=r)


def test_loaded_scene_exposure_reaches_the_display(tmp_path):
    doc = ('{"camera": {"position": [0, 0, 3], "look_at": [0, 0, 0], "fov_degrees": 40},'
           ' "render": {"width": 8, "height": 4, "samples": 2, "max_bounces": 2},'
           ' "display": {"exposure_stops": -1.25},'
           ' "materials": [{"name": "m", "type": "diffuse", "albedo": [0.5, 0.5, 0.5]}],'
           ' "objects": [{"type": "sphere", "center": [0, 0, 0], "radius": 1, "material": "m"}]}')
    p = tmp_path / "s.json"
    p.write_text(doc)
    r = RecordingRenderer()
    render_gpu_with_sink(StaticSceneEvaluator(load_scene(p)), AnimationConfig.single_frame(), ListSink(), renderer=r)
    assert [c[1] for c in r.calls if c[0] == "readback"] == [-1.25]


def test_mjpeg_sink_streams_device_jpegs():
    import io

    from toaster_b200.stream import split_mjpeg

    buf = io.BytesIO()
    r = RecordingRenderer()
    sink = MjpegFrameSink(buf, quality=70, max_frames=3)
    render_gpu_with_sink(StaticSceneEvaluator(small_scene()), AnimationConfig.indefinite(30), sink, renderer=r)
    jpegs = split_mjpeg(buf.getvalue())
    assert len(jpegs) == 3 and all(j[:2] == b"\xff\xd8" for j in jpegs)
    assert [c for c in r.calls if c[0] == "readback"] == []
    assert {c[1] for c in r.calls if c[0] == "jpeg"} == {70}


def test_video_export_writes_an_mjpeg_avi(tmp_path):
    from toaster_b200.frames import render_evaluated_gpu_video
    from toaster_b200.stream import read_avi_mjpeg

    r = RecordingRenderer()
    n = render_evaluated_gpu_video(StaticSceneEvaluator(small_scene()), tmp_path / "clip.avi",
                                   AnimationConfig.from_frame_count(12, 4), quality=75, renderer=r)
    w, h, fps, frames = read_avi_mjpeg(tmp_path / "clip.avi")
    assert (n, w, h, fps, len(frames)) == (4, 16, 8, 12, 4)
    assert all(f[:2] == b"\xff\xd8" for f in frames)
    assert {c[1] for c in r.calls if c[0] == "jpeg"} == {75}
    with pytest.raises(ValueError, match="FPS"):
        render_evaluated_gpu_video(StaticSceneEvaluator(small_scene()), tmp_path / "x.avi",
                                   AnimationConfig.single_frame(), renderer=r)


def test_path_based_helpers(tmp_path):
    import json

    from toaster_b200.frames import (FramePacing, benchmark_gpu_scene, render_scene_gpu, render_scene_gpu_animation,
                                     render_scene_gpu_animation_with_sink, render_scene_gpu_video)
    from toaster_b200.stream import read_avi_mjpeg

    doc = {"camera": {"position": [0, 0, 3], "look_at": [0, 0, 0], "fov_degrees": 40},
           "render": {"width": 8, "height": 4, "samples": 2, "max_bounces": 2},
           "display": {"exposure_stops": 0.5},
           "materials": [{"name": "m", "type": "diffuse", "albedo": [0.5, 0.5, 0.5]}],
           "objects": [{"type": "sphere", "center": [0, 0, 0], "radius": 1, "material": "m"}]}
    p = tmp_path / "s.json"
    p.write_text(json.dumps(doc))
    r = RecordingRenderer()
    assert [q.name for q in render_scene_gpu(p, tmp_path / "one.png", renderer=r)] == ["one.png"]
    assert len(render_scene_gpu_animation(p, tmp_path / "f.png", AnimationConfig.from_frame_count(24, 2),
                                          renderer=r)) == 2
    assert render_scene_gpu_video(p, tmp_path / "v.avi", AnimationConfig.from_frame_count(24, 2), renderer=r) == 2
    assert read_avi_mjpeg(tmp_path / "v.avi")[:3] == (8, 4, 24)
    sink = ListSink()
    render_scene_gpu_animation_with_sink(p, AnimationConfig.from_frame_count(24, 3), FramePacing.UNPACED, sink,
                                         renderer=r)
    assert len(sink.frames) == 3
    assert len(benchmark_gpu_scene(p, GpuBenchmarkConfig(1, 2), renderer=r).frames) == 2
    assert {c[1] for c in r.calls if c[0] == "readback"} == {0.5}
    doc["animation"] = {"tracks": [{"type": "translation"}]}
    p.write_text(json.dumps(doc))
    with pytest.raises(ValueError, match="animation tracks"):
        render_scene_gpu(p, tmp_path / "x.png", renderer=r)
