"""Batched multi-scene launch (tc_render_batch) against per-scene tc_render (needs a B200).

Every path is seeded by (frame index, pixel, sample) alone, so a frame traced inside a batch takes
exactly the same paths as when it is rendered on its own: the FP64 sums agree up to the order of
the atomic additions.
"""

import numpy as np
import pytest

from toaster_b200 import configs
from toaster_b200.native import TcError
from toaster_b200.renderer import GpuRenderer, render_batch
from toaster_b200.scene import scene_to_gpu

pytestmark = pytest.mark.gpu


def scenes():
    return [configs.plain_small(), configs.mixed(width=160, height=90, samples=8, max_bounces=6),
            configs.room_with_window(width=96, height=54, samples=4, clutter=1024)]


def close(a, b):
    rel = np.abs(a - b) / np.maximum(np.abs(b), 1e-6)
    return np.mean(rel < 1e-9)


def test_batch_matches_individual_renders(native_lib):
    sc = scenes()
    rs = [GpuRenderer(0) for _ in sc]
    try:
        for r, s in zip(rs, sc):
            r.upload(scene_to_gpu(s))
        st = render_batch(rs, frame_index=11)
        assert st["paths"] == sum(s.width * s.height * s.samples for s in sc)
        batched = [r.readback_sums()[0] for r in rs]
        for r, s, b in zip(rs, sc, batched):
            r.render(frame_index=11)
            single = r.readback_sums()[0]
            assert close(b, single) > 0.999
        # Progressive: a second batched pass adds to each image.
        render_batch(rs, frame_index=12, accumulate=True)
        assert all(r.accumulated == 2 * s.samples for r, s in zip(rs, sc))
        assert np.all(np.isfinite(rs[1].readback()))
    finally:
        for r in rs:
            r.close()


def test_batch_gives_large_frames_their_own_wavefront_call(native_lib):
    # A frame of 2^20 paths fills the GPU by itself: the automatic schedule renders it with a
    # wavefront call of its own and the small frames in the shared launch; either way every frame
    # takes its own paths, so each matches its own single render.
    sc = [configs.mixed(width=1024, height=1024, samples=1), configs.plain_small(),
          configs.room_with_window(width=96, height=54, samples=4, clutter=1024)]
    rs = [GpuRenderer(0) for _ in sc]
    try:
        for r, s in zip(rs, sc):
            r.upload(scene_to_gpu(s))
        for schedule, single in (("auto", ["wavefront", "auto", "auto"]), ("megakernel", ["megakernel"] * 3)):
            st = render_batch(rs, frame_index=21, schedule=schedule)
            assert st["paths"] == sum(s.width * s.height * s.samples for s in sc)
            assert (st["kernel_launches"] > 1) == (schedule == "auto")
            batched = [r.readback_sums()[0] for r in rs]
            for r, b, one in zip(rs, batched, single):
                r.render(frame_index=21, schedule=one)
                assert close(b, r.readback_sums()[0]) > 0.999
    finally:
        for r in rs:
            r.close()


def test_batch_rejects_duplicates_and_options(native_lib):
    r = GpuRenderer(0)
    try:
        r.upload(scene_to_gpu(configs.plain_small()))
        with pytest.raises(TcError, match="twice"):
            render_batch([r, r])
    finally:
        r.close()


def test_autotune_returns_a_working_shape(native_lib):
    with GpuRenderer(0) as r:
        r.upload(scene_to_gpu(configs.mixed(width=320, height=180, samples=4, max_bounces=4)))
        best = r.autotune(probe_samples=2)
        assert best["block_size"] in (64, 128, 256)
        assert best["short_stack"] in (0, 8, 16)
        assert best["refill_lanes"] in (1, 12, 20, 28)
        assert best["samples_per_item"] in (1, 2, 4)
        assert best["schedule"] in ("megakernel", "wavefront")
        assert best["candidates"] >= 6 and best["mpaths_per_s"] > 0
        r.render(block_size=best["block_size"], short_stack=best["short_stack"],
                 refill_lanes=best["refill_lanes"], samples_per_item=best["samples_per_item"],
                 wave_paths=best["wave_paths"], schedule=best["schedule"])
        assert r.stats()["paths"] == 320 * 180 * 4


@pytest.mark.parametrize("refill", [1, 12, 28, 32])
@pytest.mark.parametrize("short_stack", [0, 16])
def test_launch_shapes_trace_the_same_paths(renderer, refill, short_stack):
    # Dynamic fetching and the shared short stack change when and where a lane's traversal runs,
    # not what it computes: the image equals the default shape's up to FP64 summation order.
    scene = configs.mixed(width=96, height=54, samples=8, max_bounces=6)
    renderer.upload(scene_to_gpu(scene))
    renderer.render(frame_index=5)
    a = renderer.readback_sums()[0]
    renderer.render(frame_index=5, refill_lanes=refill, short_stack=short_stack, block_size=256)
    b = renderer.readback_sums()[0]
    assert close(b, a) > 0.999


def test_guided_batch_matches_individual_guided_renders(native_lib):
    # Each frame's queries are inferred by its own network, and every path keeps its seed, so a
    # guided frame traced inside a batch takes the paths of its own guided render.
    from toaster_b200 import guiding_eval

    sc = [configs.room_with_window(width=64, height=36, samples=8, clutter=1024),
          configs.mixed(width=80, height=45, samples=8, max_bounces=6),
          configs.plain_small()]
    for s in sc:
        s.samples = 8
    rs = [GpuRenderer(0) for _ in sc]
    try:
        for i, (r, s) in enumerate(zip(rs, sc)):
            r.upload(scene_to_gpu(s))
            r.guide_set_params(guiding_eval.initial_params(3 + i), configs.scene_bounds(s))
        # A small wave, so the batch runs several waves of whole samples per pixel.
        st = render_batch(rs, frame_index=4, guiding=True, wave_paths=40000)
        assert st["paths"] == sum(s.width * s.height * 8 for s in sc)
        batched = [r.readback_sums()[0] for r in rs]
        for r, s, b in zip(rs, sc, batched):
            r.render(frame_index=4, guiding=True)
            single = r.readback_sums()[0]
            assert close(b, single) > 0.999
            assert b.sum() > 0
    finally:
        for r in rs:
            r.close()


def test_guided_batch_with_a_large_frame(native_lib):
    # The 2^20-path frame gets a guided wavefront call of its own, the small frame the shared
    # guided launch; only the shared launch's frames need one sample count.
    from toaster_b200 import guiding_eval

    sc = [configs.mixed(width=1024, height=1024, samples=1),
          configs.room_with_window(width=64, height=36, samples=8, clutter=1024)]
    rs = [GpuRenderer(0) for _ in sc]
    try:
        for i, (r, s) in enumerate(zip(rs, sc)):
            r.upload(scene_to_gpu(s))
            r.guide_set_params(guiding_eval.initial_params(5 + i), configs.scene_bounds(s))
        st = render_batch(rs, frame_index=5, guiding=True)
        assert st["paths"] == sum(s.width * s.height * s.samples for s in sc)
        batched = [r.readback_sums()[0] for r in rs]
        for r, b, schedule in zip(rs, batched, ("wavefront", "auto")):
            r.render(frame_index=5, guiding=True, schedule=schedule)
            assert close(b, r.readback_sums()[0]) > 0.999
            assert b.sum() > 0
    finally:
        for r in rs:
            r.close()


def test_guided_batch_needs_networks_and_one_sample_count(native_lib):
    from toaster_b200 import guiding_eval

    a, b = GpuRenderer(0), GpuRenderer(0)
    try:
        s = configs.plain_small()
        a.upload(scene_to_gpu(s))
        b.upload(scene_to_gpu(s))
        a.guide_set_params(guiding_eval.initial_params(1), configs.scene_bounds(s))
        with pytest.raises(TcError, match="tc_guide_set_params"):
            render_batch([a, b], guiding=True)
        b.guide_set_params(guiding_eval.initial_params(2), configs.scene_bounds(s))
        with pytest.raises(TcError, match="one sample count"):
            render_batch([a, b], samples=[4, 8], guiding=True)
    finally:
        a.close()
        b.close()
