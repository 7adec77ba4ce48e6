"""The host frame loop on the GPU (needs a B200): PNG animation frames equal direct renders of the
same evaluated scenes, a progressive render reaches its exact sample target, and the MJPEG sink
streams device-encoded frames."""

import numpy as np
import pytest

from toaster_b200 import configs
from toaster_b200.frames import (AnimationConfig, FrameSink, FunctionSceneEvaluator, GpuBenchmarkConfig,
                                 MjpegFrameSink, ProgressiveRenderConfig, StaticSceneEvaluator, benchmark_gpu_evaluator,
                                 render_evaluated_gpu_animation, render_gpu_progressive_with_sink,
                                 render_gpu_with_sink)
from toaster_b200.renderer import GpuRenderer
from toaster_b200.scene import _decode_png, scene_to_gpu

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("hierarchy", ["rebuild", "refit"])
def test_png_frames_equal_direct_renders(native_lib, tmp_path, hierarchy):
    anim = configs.BallisticAnimation(width=96, height=54, samples=8, max_bounces=6, frames=3)
    ev = FunctionSceneEvaluator(lambda t: anim.scene(int(round(t * 24))))
    written = render_evaluated_gpu_animation(ev, tmp_path / "f.png", AnimationConfig.from_frame_count(24, 3),
                                             hierarchy=hierarchy)
    assert len(written) == 3
    with GpuRenderer(0) as r:
        for k, path in enumerate(written):
            r.upload(scene_to_gpu(anim.scene(k)))
            r.render(frame_index=k)
            direct = r.readback_rgba8(0.0)
            _, _, _, img = _decode_png(path.read_bytes())
            diff = np.abs(img.astype(int) - direct.astype(int))
            assert diff.max() <= 1 and np.mean(diff == 0) >= 0.999, (hierarchy, k)


def test_progressive_reaches_target_and_benchmark_measures(native_lib):
    scene = configs.mixed(width=64, height=36, samples=5, max_bounces=6)

    class Last(FrameSink):
        def __init__(self):
            self.acc = []

        def deliver(self, frame):
            self.acc.append(frame.accumulated_samples)

    sink = Last()
    render_gpu_progressive_with_sink(scene, AnimationConfig.indefinite(30), ProgressiveRenderConfig(12), sink)
    assert sink.acc == [5, 10, 12]
    res = benchmark_gpu_evaluator(StaticSceneEvaluator(scene), GpuBenchmarkConfig(1, 2))
    assert len(res.frames) == 2 and res.final_image.shape == (36, 64, 4)
    assert all(t.kernel_ms > 0 for t in res.frames)


def test_mjpeg_sink_streams_device_encoded_frames(native_lib):
    import io

    from toaster_b200.stream import split_mjpeg

    anim = configs.BallisticAnimation(width=96, height=54, samples=4, max_bounces=4, frames=4)
    ev = FunctionSceneEvaluator(lambda t: anim.scene(int(round(t * 24)) % 4))
    buf = io.BytesIO()
    render_gpu_with_sink(ev, AnimationConfig.indefinite(24), MjpegFrameSink(buf, quality=80, max_frames=3))
    jpegs = split_mjpeg(buf.getvalue())
    assert len(jpegs) == 3
    assert all(j[:2] == b"\xff\xd8" and j[-2:] == b"\xff\xd9" and len(j) > 500 for j in jpegs)


def test_video_export_holds_the_device_jpegs(native_lib, tmp_path):
    from toaster_b200.frames import render_evaluated_gpu_video
    from toaster_b200.stream import read_avi_mjpeg

    anim = configs.BallisticAnimation(width=96, height=54, samples=4, max_bounces=4, frames=3)
    ev = FunctionSceneEvaluator(lambda t: anim.scene(int(round(t * 24))))
    assert render_evaluated_gpu_video(ev, tmp_path / "clip.avi", AnimationConfig.from_frame_count(24, 3)) == 3
    w, h, fps, frames = read_avi_mjpeg(tmp_path / "clip.avi")
    assert (w, h, fps, len(frames)) == (96, 54, 24, 3)
    assert all(f[:2] == b"\xff\xd8" and f[-2:] == b"\xff\xd9" for f in frames)
