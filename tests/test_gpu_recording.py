"""Guide training samples recorded by the wavefront schedule, and the sample pool (needs a B200).

The wavefront traces the megakernel's paths (same random numbers in the same order), so the
training samples it records from a plain batch are the megakernel's record mode samples; the
pool keeps the samples of every recording batch since the last one that started it; guided
wavefront batches record too, their samples weighted by the mixture pdf their directions were
drawn with.
"""

import numpy as np
import pytest

from toaster_b200 import configs, guiding_eval
from toaster_b200.native import TcError
from toaster_b200.scene import scene_to_gpu

pytestmark = pytest.mark.gpu


def room(width=96, height=54):
    return configs.room_with_window(width=width, height=height, samples=16, clutter=2048)


def keyed(samples):
    """Samples keyed by their rounded position and direction (their order is unspecified)."""
    return {tuple(np.round(np.concatenate([s[0:3], s[8:11]]), 4)): s[3] for s in samples}


def test_wavefront_records_the_megakernel_samples(renderer):
    scene = room()
    renderer.upload(scene_to_gpu(scene))
    renderer.guide_set_params(guiding_eval.initial_params(1), configs.scene_bounds(scene))
    got = {}
    for schedule in ("megakernel", "wavefront"):
        renderer.render(samples=16, frame_index=2, guide_record=1, schedule=schedule)
        got[schedule] = renderer.guide_recorded_samples()
    mk, wf = got["megakernel"], got["wavefront"]
    assert len(mk) > 300
    # Paths tip the other way only at rounding-level differences between the two kernels' fused
    # multiply-adds, so all but a few samples must be the same.
    assert abs(len(wf) - len(mk)) <= 0.01 * len(mk) + 2, (len(wf), len(mk))
    a, b = keyed(mk), keyed(wf)
    same = sum(1 for k, w in b.items() if k in a and abs(a[k] - w) <= 1e-4 * abs(a[k]) + 1e-9)
    assert same >= 0.98 * len(b), (same, len(b))
    assert abs(wf[:, 3].sum() - mk[:, 3].sum()) <= 0.02 * mk[:, 3].sum()


def test_pool_appends_batches_until_restarted(renderer):
    scene = room(64, 36)
    renderer.upload(scene_to_gpu(scene))
    renderer.guide_set_params(guiding_eval.initial_params(1), configs.scene_bounds(scene))
    counts = []
    for frame in (5, 6):
        renderer.render(samples=16, frame_index=frame, guide_record=1, schedule="wavefront")
        counts.append(len(renderer.guide_recorded_samples()))
    renderer.render(samples=16, frame_index=5, guide_record=1, schedule="wavefront")
    renderer.render(samples=16, frame_index=6, guide_record=2, schedule="wavefront")
    pool = renderer.guide_recorded_samples()
    assert len(pool) == sum(counts), (len(pool), counts)
    _, n = renderer.guide_train_recorded(steps=2, batch=1024, lr=1e-3, seed=0)
    assert n == sum(counts)


def test_guided_wavefront_batches_record_and_train(renderer):
    scene = room()
    renderer.upload(scene_to_gpu(scene))
    renderer.guide_set_params(guiding_eval.initial_params(1), configs.scene_bounds(scene))
    renderer.render(samples=16, frame_index=0, guide_record=1, schedule="wavefront")
    losses, n0 = renderer.guide_train_recorded(steps=100, batch=4096, lr=1e-2, seed=5)
    assert n0 > 300 and losses[-10:].mean() < losses[:5].mean()
    renderer.render(samples=16, frame_index=16, accumulate=True, guiding=True, guide_record=2, schedule="wavefront")
    pool = renderer.guide_recorded_samples()
    assert len(pool) > n0
    w = pool[:, 3]
    assert np.all(np.isfinite(w)) and np.all(w > 0)
    assert np.allclose(np.linalg.norm(pool[:, 8:11], axis=1), 1.0, atol=1e-4)
    _, n1 = renderer.guide_train_recorded(steps=20, batch=4096, lr=1e-2, seed=6)
    assert n1 == len(pool)
    assert np.all(np.isfinite(renderer.readback()))


def test_guided_recording_needs_the_wavefront(renderer):
    scene = room(32, 18)
    renderer.upload(scene_to_gpu(scene))
    renderer.guide_set_params(guiding_eval.initial_params(1), configs.scene_bounds(scene))
    with pytest.raises(TcError, match="wavefront"):
        renderer.render(samples=4, guiding=True, guide_record=1, schedule="megakernel")
    with pytest.raises(TcError, match="guide_record"):
        renderer.render(samples=4, guide_record=3)
