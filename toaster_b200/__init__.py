"""toaster_b200 — a B200-native (sm_100a) CUDA backend for toaster's GPU path-tracing path.

Scene in (toaster's JSON format or packed ``gpu_types`` records), linear-HDR float4 image out,
through the C ABI in include/toaster_cuda.h. ``renderer`` holds the per-call host API, ``frames``
the frame loop (schedules, sinks, animation / video / progressive / benchmark entry points).
"""

from . import gpu_types
from .scene import (EnvironmentMap, Material, Scene, SceneGpuData, load_scene, load_scene_gpu, make_camera,
                    scene_to_gpu)

__all__ = [
    "gpu_types",
    "EnvironmentMap",
    "Material",
    "Scene",
    "SceneGpuData",
    "load_scene",
    "load_scene_gpu",
    "make_camera",
    "scene_to_gpu",
]


def __getattr__(name):
    # The renderer needs the built CUDA library; import it on first use only.
    if name in {"GpuRenderer", "render_hdr", "render_batch", "progressive_batch"}:
        from . import renderer

        return getattr(renderer, name)
    if name in {"AnimationConfig", "FrameSink", "CompletedFrame", "render_evaluated_gpu_animation",
                "render_evaluated_gpu_video", "render_gpu_progressive_with_sink", "benchmark_gpu_evaluator",
                "render_scene_gpu", "benchmark_gpu_scene"}:
        from . import frames

        return getattr(frames, name)
    raise AttributeError(name)
