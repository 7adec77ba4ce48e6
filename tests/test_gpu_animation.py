"""Animated frames through the captured CUDA graph (tc_animation_*) against the direct calls
(tc_update_geometry + tc_render + tc_readback_rgba8) on the same frames (needs a B200).

Both refit the hierarchy built for frame 0 and seed every path by (frame index, pixel, sample), so
they trace identical paths: the FP64 sums differ only in the order of atomic additions and the
display bytes agree except where a channel sits on a rounding boundary.
"""

import numpy as np
import pytest

from toaster_b200 import configs, guiding_eval
from toaster_b200.native import TcError
from toaster_b200.renderer import Animation, GpuRenderer
from toaster_b200.scene import scene_to_gpu

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def anim():
    return configs.BallisticAnimation(width=320, height=180, samples=8, max_bounces=4, frames=48)


def direct_frame(r, anim, k, exposure):
    r.update_geometry(scene_to_gpu(anim.scene(k)), camera=True, spheres=True, triangles=True, emissive_geometry=True)
    r.render(frame_index=k)
    return r.readback_rgba8(exposure)


def test_graph_frames_match_direct_calls(native_lib, anim):
    first = scene_to_gpu(anim.scene(0))
    with GpuRenderer(0) as ra, GpuRenderer(0) as rd:
        ra.upload(first)
        rd.upload(first)
        with Animation(ra, first, exposure_stops=0.5, update_lights=True) as a:
            for k in (1, 7, 30, 47):
                g = a.frame(scene_to_gpu(anim.scene(k)), k)
                d = direct_frame(rd, anim, k, 0.5)
                diff = np.abs(g.astype(np.int16) - d.astype(np.int16))
                assert diff.max() <= 1
                assert np.mean(diff == 0) > 0.999
                assert ra.stats()["paths"] == 320 * 180 * 8


def test_graph_frames_with_rebuild_match_fresh_uploads(native_lib, anim):
    # Rebuild mode builds each frame's own median-split hierarchy, the one a fresh upload builds
    # (and the reference builds), so the two trace identical paths.
    first = scene_to_gpu(anim.scene(0))
    with GpuRenderer(0) as ra, GpuRenderer(0) as rd:
        ra.upload(first)
        with Animation(ra, first, exposure_stops=0.5, update_lights=True, rebuild=True) as a:
            for k in (3, 25, 47):
                data = scene_to_gpu(anim.scene(k))
                g = a.frame(data, k)
                rd.upload(data)
                rd.render(frame_index=k)
                d = rd.readback_rgba8(0.5)
                diff = np.abs(g.astype(np.int16) - d.astype(np.int16))
                assert diff.max() <= 1
                assert np.mean(diff == 0) > 0.999


def test_graph_frames_follow_the_motion(native_lib, anim):
    first = scene_to_gpu(anim.scene(0))
    with GpuRenderer(0) as r:
        r.upload(first)
        with Animation(r, first) as a:
            f0 = a.frame(first, 0).astype(np.float64)
            f0b = a.frame(first, 0).astype(np.float64)
            f20 = a.frame(scene_to_gpu(anim.scene(20)), 0).astype(np.float64)
    assert np.abs(f0b - f0).max() <= 1 and np.mean(f0b == f0) > 0.999  # replays trace the same paths
    assert np.abs(f20 - f0).mean() > 1.0                                # moved geometry changes the picture


def test_guided_graph_frames(native_lib, anim):
    first = scene_to_gpu(anim.scene(0))
    with GpuRenderer(0) as r:
        r.upload(first)
        r.guide_set_params(guiding_eval.initial_params(0), configs.scene_bounds(anim.scene(0)))
        r.render(samples=16, frame_index=0, guide_record=True)
        r.guide_train_recorded(100, 4096, 1e-2, 3)
        with Animation(r, first, guiding=True, update_lights=True) as a:
            img = a.frame(scene_to_gpu(anim.scene(12)), 12)
            assert r.stats()["paths"] == 320 * 180 * 8
    assert img[..., 3].min() == 255 and img[..., :3].mean() > 1.0


def test_animation_rejects_count_change(native_lib, anim):
    first = scene_to_gpu(anim.scene(0))
    other = scene_to_gpu(configs.plain_small())
    with GpuRenderer(0) as r:
        r.upload(first)
        with Animation(r, first) as a:
            with pytest.raises(TcError, match="preserve GPU geometry"):
                a.frame(other, 1)
