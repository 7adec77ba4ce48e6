"""Path-guiding network on the tensor cores vs the NumPy restatement (needs a B200).

Forward outputs, the loss, its gradient and an Adam step are compared with
oracle/guide_net.py on the same parameters and inputs. Tolerances cover BF16 activations
whose rounding can flip when the FP32 accumulation order differs (tensor core vs FP64 NumPy).
"""

import numpy as np
import pytest

from oracle import guide_net as gn

pytestmark = pytest.mark.gpu

BOUNDS = (0.1, -0.2, 0.05, 0.5)


def random_queries(n, seed):
    rng = np.random.default_rng(seed)
    p = rng.uniform(-2, 2, (n, 3)).astype(np.float32)
    nrm = rng.normal(size=(n, 3))
    nrm = (nrm / np.linalg.norm(nrm, axis=1, keepdims=True)).astype(np.float32)
    return p, nrm


def reference_outputs(params, p, nrm):
    x = gn.encode(p, nrm, BOUNDS[:3], BOUNDS[3])
    y, cache = gn.forward(params, x)
    return y, cache


def test_guide_inference_matches_reference(renderer):
    params = gn.init_params(seed=3)
    params[gn.N_PARAMS - 32:] = np.random.default_rng(1).normal(0, 0.5, 32)  # nonzero output biases
    renderer.guide_set_params(params, BOUNDS)
    assert np.array_equal(renderer.guide_get_params(), params.astype(np.float32))
    p, nrm = random_queries(1000, 2)  # 8 tiles, the last one partial
    got = renderer.guide_infer(p, nrm)
    y, _ = reference_outputs(params, p, nrm)
    w, kappa, mu = gn.decode(y)
    mu_got = got[:, :32].reshape(-1, 8, 4)
    assert np.abs(mu_got[..., :3] - mu).max() < 0.03
    assert np.max(np.abs(mu_got[..., 3] - kappa) / kappa) < 0.05
    assert np.abs(got[:, 32:] - w).max() < 0.01
    assert np.allclose(np.linalg.norm(mu_got[..., :3], axis=-1), 1.0, atol=1e-5)
    assert np.allclose(got[:, 32:].sum(1), 1.0, atol=1e-5)


def make_samples(n, seed):
    rng = np.random.default_rng(seed)
    p, nrm = random_queries(n, seed)
    om = rng.normal(size=(n, 3))
    om /= np.linalg.norm(om, axis=1, keepdims=True)
    s = rng.uniform(0.2, 2.0, n)
    return np.concatenate([p, nrm, om, s[:, None]], axis=1).astype(np.float32)


def test_guide_loss_and_gradient_match_reference(renderer):
    params = gn.init_params(seed=5)
    params[gn.N_PARAMS - 32:] = np.random.default_rng(2).normal(0, 0.5, 32)
    renderer.guide_set_params(params, BOUNDS)
    samples = make_samples(1000, 7)
    grad, loss = renderer.guide_loss_grad(samples)
    y, cache = reference_outputs(params, samples[:, :3], samples[:, 3:6])
    ref_loss, dy = gn.loss_and_dy(y, samples[:, 6:9], samples[:, 9])
    ref = gn.backward(params, cache, dy)
    assert abs(loss - ref_loss) <= 2e-3 * abs(ref_loss)
    g, r = gn.unpack(grad), gn.unpack(ref)
    for name in g:
        rel = np.linalg.norm(g[name] - r[name]) / max(np.linalg.norm(r[name]), 1e-12)
        assert rel < 0.03, (name, rel)
    assert np.all(g["W1"][:, 75:] == 0.0)


def test_guide_adam_step_matches_reference(renderer):
    params = gn.init_params(seed=9)
    renderer.guide_set_params(params, BOUNDS)
    samples = make_samples(512, 9)
    grad, _ = renderer.guide_loss_grad(samples)
    renderer.guide_adam_step(1e-2)
    got = renderer.guide_get_params()
    ref, _, _ = gn.adam(params, grad, np.zeros_like(params), np.zeros_like(params), 1, lr=1e-2)
    pad = np.zeros(gn.N_PARAMS, bool)
    pad[:64 * 80] = (np.arange(64 * 80) % 80) >= 75
    assert np.allclose(got[~pad], ref[~pad], rtol=1e-5, atol=1e-6)
    assert np.array_equal(got[pad], params[pad])


def test_guide_training_learns_a_directional_distribution(renderer):
    # Radiance arrives from a direction that depends on position: the trained mixture must put
    # most of its mass there, and the loss must fall.
    rng = np.random.default_rng(11)
    n = 1 << 15
    p = rng.uniform(-1, 1, (n, 3)).astype(np.float32)
    nrm = np.tile(np.float32([0, 1, 0]), (n, 1))
    target = np.stack([np.sign(p[:, 0]) * 0.6, np.full(n, 0.8), np.zeros(n)], 1)
    noise = rng.normal(0, 0.1, (n, 3))
    om = target + noise
    om /= np.linalg.norm(om, axis=1, keepdims=True)
    samples = np.concatenate([p, nrm, om, np.ones((n, 1))], 1).astype(np.float32)
    renderer.guide_set_params(gn.init_params(seed=1), (0, 0, 0, 1.0))
    losses = renderer.guide_train(samples, steps=300, batch=4096, lr=1e-2, seed=3)
    assert np.all(np.isfinite(losses))
    assert losses[-20:].mean() < losses[:5].mean() - 1.5
    q_p = np.float32([[0.5, 0.0, 0.2], [-0.5, 0.3, -0.1]])
    dec = renderer.guide_infer(q_p, np.float32([[0, 1, 0], [0, 1, 0]]))
    pdf_at_target = gn.mixture_pdf_from_decoded(dec, np.float32([[0.6, 0.8, 0], [-0.6, 0.8, 0]]))
    pdf_opposite = gn.mixture_pdf_from_decoded(dec, np.float32([[-0.6, 0.8, 0], [0.6, 0.8, 0]]))
    assert np.all(pdf_at_target > 5.0 / (4 * np.pi))
    assert np.all(pdf_at_target > 4 * pdf_opposite)
