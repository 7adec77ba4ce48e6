"""The wavefront schedule against the megakernel (needs a B200).

Both schedules trace the same estimator (crates/toaster-cpu/src/integrator.rs:99-244) and every
path draws its random numbers in the same order from the same per-(frame, pixel, sample) seed,
so each path is the same in both up to the compiler's fusing of multiply-adds, which may differ
between the two kernels and, very rarely, tips a borderline decision (a metal reflection grazing
the surface, Schlick against refraction) the other way; elsewhere it moves a path's radiance by
an FP32 rounding or two. So the ray counts must agree within one ray in ten thousand, and all but
1% of the per-pixel sums must agree to 1e-5 relative (a path that went another way moves its pixel
by a few percent; measured: 0.3-0.4% of the pixels of 16- and 32-spp frames hold one).
"""

import numpy as np
import pytest

from toaster_b200 import configs
from toaster_b200.scene import scene_to_gpu

pytestmark = pytest.mark.gpu


def render_both(renderer, samples, max_bounces=None, keep_moments=False, wave_paths=0, refill_lanes=0,
                frame_index=3, ray_sort=0):
    out = {}
    for schedule in ("megakernel", "wavefront"):
        renderer.render(samples=samples, max_bounces=max_bounces, frame_index=frame_index, keep_moments=keep_moments,
                        schedule=schedule, wave_paths=wave_paths,
                        refill_lanes=refill_lanes if schedule == "wavefront" else 0,
                        ray_sort=ray_sort if schedule == "wavefront" else 0)
        s, q, n = renderer.readback_sums(moments=keep_moments)
        out[schedule] = (s, q, renderer.stats())
    return out


def same_fraction(a, b):
    """Fraction of pixels whose three sums agree to FP32 rounding of the paths' radiance."""
    return float(np.mean(np.isclose(a, b, rtol=1e-5, atol=1e-7).all(axis=-1)))


def assert_same_paths(out, scene, samples):
    (s0, q0, st0), (s1, q1, st1) = out["megakernel"], out["wavefront"]
    paths = scene.width * scene.height * samples
    assert st0["paths"] == st1["paths"] == paths
    for key in ("extension_rays", "shadow_rays"):
        assert abs(int(st1[key]) - int(st0[key])) <= 1e-4 * st0[key] + 2, (key, st0[key], st1[key])
    assert same_fraction(s1, s0) >= 0.99, same_fraction(s1, s0)
    if q0 is not None:
        assert same_fraction(q1, q0) >= 0.99
    assert s0.sum() > 0


@pytest.mark.parametrize("make,samples", [(lambda: configs.mixed(width=96, height=54), 32),
                                           (lambda: configs.plain_small(), 4),
                                           (lambda: configs.room_with_window(width=64, height=36, clutter=1024), 32)],
                         ids=["mixed", "plain_small", "window_room"])
def test_wavefront_traces_the_megakernel_paths(renderer, make, samples):
    scene = make()
    renderer.upload(scene_to_gpu(scene))
    assert_same_paths(render_both(renderer, samples), scene, samples)


@pytest.mark.parametrize("bounces", [1, 2, 3])
def test_wavefront_short_paths_and_moments(renderer, bounces):
    scene = configs.mixed(width=64, height=36)
    renderer.upload(scene_to_gpu(scene))
    assert_same_paths(render_both(renderer, 16, max_bounces=bounces, keep_moments=True), scene, 16)


@pytest.mark.parametrize("wave_paths", [32, 1000, 1 << 16])
def test_wavefront_slot_counts(renderer, wave_paths):
    # Fewer slots than paths: slots are refilled many times over, and a partial last warp of slots.
    scene = configs.mixed(width=48, height=27)
    renderer.upload(scene_to_gpu(scene))
    assert_same_paths(render_both(renderer, 8, wave_paths=wave_paths), scene, 8)


@pytest.mark.parametrize("refill_lanes", [8, 16, 28])
def test_wavefront_dynamic_ray_fetching(renderer, refill_lanes):
    # Trace lanes refill from the queue mid-traversal: the same rays, so the same paths.
    scene = configs.mixed(width=64, height=36)
    renderer.upload(scene_to_gpu(scene))
    assert_same_paths(render_both(renderer, 16, refill_lanes=refill_lanes), scene, 16)


@pytest.mark.parametrize("wave_paths", [0, 1000])
def test_wavefront_sorted_rays(renderer, wave_paths):
    # Sorting the queued rays changes the order in which they are traced, not the rays.
    scene = configs.mixed(width=96, height=54)
    renderer.upload(scene_to_gpu(scene))
    assert_same_paths(render_both(renderer, 32, wave_paths=wave_paths, ray_sort=2), scene, 32)


def test_wavefront_progressive_batches(renderer):
    # The progressive contract holds across schedules: a wavefront batch adds to megakernel batches.
    scene = configs.mixed(width=64, height=36)
    renderer.upload(scene_to_gpu(scene))
    renderer.render(samples=8, frame_index=1, schedule="megakernel")
    renderer.render(samples=8, frame_index=1, accumulate=True, schedule="wavefront")
    mixed_sums, _, n = renderer.readback_sums()
    assert n == 16
    renderer.render(samples=8, frame_index=1, schedule="megakernel")
    renderer.render(samples=8, frame_index=1, accumulate=True, schedule="megakernel")
    mega_sums, _, _ = renderer.readback_sums()
    assert same_fraction(mixed_sums, mega_sums) >= 0.99


@pytest.mark.parametrize("fraction", [0.5, 0.85])
def test_guided_wavefront_traces_the_guided_megakernel_paths(renderer, fraction):
    # Guided: the same network infers the same (point, normal) queries in both schedules, and the
    # paths draw in the same order (light NEE, environment NEE, then the one-sample MIS bounce).
    from toaster_b200 import guiding_eval

    scene = configs.room_with_window(width=64, height=36, clutter=1024)
    renderer.upload(scene_to_gpu(scene))
    renderer.guide_set_params(guiding_eval.initial_params(4), configs.scene_bounds(scene))
    out = {}
    for schedule in ("megakernel", "wavefront"):
        renderer.render(samples=16, frame_index=2, guiding=True, guide_fraction=fraction, schedule=schedule)
        out[schedule] = (renderer.readback_sums()[0], None, renderer.stats())
    assert_same_paths(out, scene, 16)


def test_phase_timing_splits_the_wavefront_time(renderer):
    """Per-phase device times of a wavefront render add up to at most its kernel time; a render
    without phase timing, and a megakernel render, report none."""
    scene = configs.mixed(width=256, height=144)
    renderer.upload(scene_to_gpu(scene))
    renderer.render(samples=32, schedule="wavefront", wave_paths=1 << 18, phase_timing=True)
    st = renderer.stats()
    assert st["wf_iterations"] >= scene.max_bounces + 2
    assert st["kernel_launches"] == 3 * st["wf_iterations"]
    assert st["trace_ms"] > 0 and st["logic_ms"] > 0 and st["shade_ms"] > 0 and st["guide_ms"] == 0
    assert st["trace_ms"] + st["logic_ms"] + st["shade_ms"] <= st["kernel_ms"] * 1.001
    renderer.render(samples=32, schedule="wavefront", wave_paths=1 << 18)
    st = renderer.stats()
    assert st["wf_iterations"] > 0 and st["trace_ms"] == 0
    renderer.render(samples=32, schedule="megakernel", phase_timing=True)
    st = renderer.stats()
    assert st["wf_iterations"] == 0 and st["trace_ms"] == 0 and st["kernel_launches"] == 1
