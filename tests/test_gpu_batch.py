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


def test_batch_rejects_duplicates_and_options(native_lib):
    r = GpuRenderer(0)
    try:
        r.upload(scene_to_gpu(configs.plain_small()))
        with pytest.raises(TcError, match="twice"):
            render_batch([r, r])
    finally:
        r.close()
