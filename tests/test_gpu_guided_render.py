"""Guided rendering (needs a B200): unbiased against plain sampling, trainable from recorded samples."""

import math

import numpy as np
import pytest

from oracle import guide_net as gn
from toaster_b200 import configs, guiding_eval
from toaster_b200.native import TcError
from toaster_b200.renderer import GpuRenderer
from toaster_b200.scene import scene_to_gpu

pytestmark = pytest.mark.gpu


def test_initial_params_match_the_reference_init():
    assert np.array_equal(guiding_eval.initial_params(3), gn.init_params(3))


def blocks(x, b):
    h, w = x.shape
    return x[: h // b * b, : w // b * b].reshape(h // b, b, w // b, b).sum(axis=(1, 3))


def render_moments(r, spp, **kw):
    r.render(samples=spp, keep_moments=True, **kw)
    s, q, n = r.readback_sums(moments=True)
    w = np.array([0.2126, 0.7152, 0.0722])
    m = s / n
    v = np.maximum(q / n - m * m, 0.0) * n / (n - 1)
    return m @ w, v @ (w**2), n


@pytest.mark.parametrize("make", [lambda: configs.mixed(width=64, height=36, samples=64),
                                  lambda: configs.room_with_window(width=64, height=36, samples=64, clutter=1024)],
                         ids=["mixed", "room"])
@pytest.mark.parametrize("fraction,spp", [(0.0, 2048), (0.85, 8192)], ids=["default_mix", "guide_heavy"])
def test_guided_sampling_is_unbiased(renderer, make, fraction, spp):
    # Untrained (random) network: the one-sample MIS of BSDF and guide sampling must still give
    # the plain estimator's expectation, at the default mixing probability and a guide-heavy one.
    # The sun makes both estimators heavy-tailed, so the guide-heavy case takes more samples for
    # its per-pixel variance estimates to hold.
    scene = make()
    renderer.upload(scene_to_gpu(scene))
    renderer.guide_set_params(guiding_eval.initial_params(7), configs.scene_bounds(scene))
    pl, pv, n = render_moments(renderer, spp, frame_index=3)
    gl, gv, m = render_moments(renderer, spp, frame_index=4, guiding=True, guide_fraction=fraction)
    d = blocks(gl - pl, 2) / 4
    var = (blocks(pv, 2) / n + blocks(gv, 2) / m) / 16
    nz = var > 0
    z = d[nz] / np.sqrt(var[nz])
    assert np.mean(np.abs(z) > 3) <= 0.06, np.mean(np.abs(z) > 3)
    assert abs(np.median(z)) <= 0.35
    se = math.sqrt((pv.sum() / n + gv.sum() / m)) / pv.size
    assert abs(gl.mean() - pl.mean()) <= 6 * se, (gl.mean(), pl.mean(), se)


def test_guide_fraction_outside_unit_interval_is_rejected(renderer):
    scene = configs.mixed(width=16, height=8, samples=4)
    renderer.upload(scene_to_gpu(scene))
    renderer.guide_set_params(guiding_eval.initial_params(7), configs.scene_bounds(scene))
    for bad in (1.0, -0.25, float("nan")):
        with pytest.raises(TcError, match="guide_fraction"):
            renderer.render(samples=4, guiding=True, guide_fraction=bad)


def test_record_train_and_render_guided(renderer):
    scene = configs.room_with_window(width=96, height=54, samples=16, clutter=2048)
    renderer.upload(scene_to_gpu(scene))
    renderer.guide_set_params(guiding_eval.initial_params(1), configs.scene_bounds(scene))
    renderer.render(samples=16, frame_index=0, guide_record=True)
    losses, n = renderer.guide_train_recorded(steps=100, batch=4096, lr=1e-2, seed=5)
    assert n > 300
    assert np.all(np.isfinite(losses))
    assert losses[-10:].mean() < losses[:5].mean()
    renderer.render(samples=16, frame_index=1, accumulate=True, guiding=True)
    assert renderer.accumulated == 32
    img = renderer.readback()
    assert np.all(np.isfinite(img))
    st = renderer.stats()
    assert st["paths"] == 96 * 54 * 16


def test_trained_network_beats_untrained_network(native_lib):
    # What training gains: the same guided estimator (50/50 one-sample MIS with BSDF sampling) at
    # the same sample count, once with the network trained on the GPU from 32 recorded spp and once
    # with its untrained initial weights. The trimmed RMSE (the 0.1% largest pixel errors left out)
    # keeps single bright samples from deciding the comparison.
    scene = configs.room_with_window(width=320, height=180, clutter=2048, metal_fraction=0.0)
    reference = guiding_eval.reference_image(scene, 8192)
    errors = {}
    for trained in (False, True):
        with GpuRenderer(0) as r:
            r.upload(scene_to_gpu(scene))
            r.guide_set_params(guiding_eval.initial_params(0), configs.scene_bounds(scene))
            if trained:
                r.render(samples=32, frame_index=0, guide_record=True)
                _, n = r.guide_train_recorded(guiding_eval.TRAIN_STEPS, 8192, 1e-2, 1)
                assert n > 5000
            r.render(samples=128, frame_index=50_000, guiding=True)
            s, _, cnt = r.readback_sums()
            errors[trained] = guiding_eval.trimmed_rmse(s / cnt, reference)
    assert errors[True] < 0.9 * errors[False], errors
