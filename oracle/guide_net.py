"""TEST INFRASTRUCTURE ONLY: NumPy reference of the path-guiding network.

The reference renderer has no guiding; this restates, in plain NumPy, exactly what the CUDA
kernels of toaster_b200/csrc/guide.cu compute, so that their forward outputs and gradients can
be checked:

  encoding   q = (p - centre) * scale; for axis i and frequency f_k = 2^(k/2), k in 0..11:
             enc[24 i + 2 k] = sin(pi f_k q_i), enc[24 i + 2 k + 1] = cos(pi f_k q_i);
             enc[72:75] = normal; enc[75:80] = 0                               (80 inputs, bf16)
  network    h1 = relu(W1 x + b1), h2 = relu(W2 h1 + b2), h3 = relu(W3 h2 + b3), y = W4 h3 + b4
             with bf16 inputs/activations, FP32 accumulation and FP32 biases
  decoding   8 lobes j with (a, b, c, d) = y[4j:4j+4]: weight softmax(a), kappa exp(clip(b,-2,7)),
             cos(theta) = tanh(c), phi = pi tanh(d), mu = (sin t cos p, sin t sin p, cos t)
  loss       -s log sum_j w_j vMF(omega; mu_j, kappa_j), averaged over the batch
  backward   dY -> (bf16) -> dH = dZ W, dZ = dH * [h > 0] (bf16), dW = dZ^T H, db = sum dZ

bf16 rounding is emulated at the same points as the kernels (round to nearest even).
"""

from __future__ import annotations

import numpy as np

N_IN, N_HID, N_OUT, N_LOBES, N_FREQ = 80, 64, 32, 8, 12
SHAPES = [("W1", (N_HID, N_IN)), ("b1", (N_HID,)), ("W2", (N_HID, N_HID)), ("b2", (N_HID,)),
          ("W3", (N_HID, N_HID)), ("b3", (N_HID,)), ("W4", (N_OUT, N_HID)), ("b4", (N_OUT,))]
N_PARAMS = sum(int(np.prod(s)) for _, s in SHAPES)
KAPPA_LO, KAPPA_HI = -2.0, 7.0
FREQS = np.float32(2.0) ** (np.arange(N_FREQ, dtype=np.float32) / np.float32(2.0))  # f32 values the kernels use


def bf16(x):
    """Round float32 values to bfloat16 (nearest even) and return them as float32."""
    x = np.asarray(x, np.float32)
    b = x.view(np.uint32).astype(np.uint64)
    rounded = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return rounded.astype(np.uint32).view(np.float32)


def unpack(flat):
    out, o = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = np.asarray(flat[o:o + n], np.float32).reshape(shape)
        o += n
    return out


def pack(params):
    return np.concatenate([np.asarray(params[name], np.float32).reshape(-1) for name, _ in SHAPES])


def init_params(seed=0):
    """He-uniform hidden layers, a 10x smaller output layer, zero biases, zero padded inputs."""
    rng = np.random.default_rng(seed)
    p = {}
    for name, shape in SHAPES:
        if name.startswith("b"):
            p[name] = np.zeros(shape, np.float32)
            continue
        fan_in = 75 if name == "W1" else shape[1]
        bound = np.sqrt(6.0 / fan_in) * (0.1 if name == "W4" else 1.0)
        p[name] = rng.uniform(-bound, bound, shape).astype(np.float32)
    p["W1"][:, 75:] = 0.0
    return pack(p)


def encode(points, normals, centre, scale):
    q = (np.asarray(points, np.float64) - np.asarray(centre, np.float64)) * float(scale)
    n = points.shape[0]
    enc = np.zeros((n, N_IN), np.float64)
    for i in range(3):
        for k in range(N_FREQ):
            ang = np.pi * FREQS[k] * q[:, i]
            enc[:, 24 * i + 2 * k] = np.sin(ang)
            enc[:, 24 * i + 2 * k + 1] = np.cos(ang)
    enc[:, 72:75] = normals
    return bf16(enc.astype(np.float32))


def forward(flat, x):
    P = unpack(flat)
    W1, W2, W3, W4 = (bf16(P[k]) for k in ("W1", "W2", "W3", "W4"))
    z1 = x.astype(np.float64) @ W1.T.astype(np.float64) + P["b1"]
    h1 = bf16(np.maximum(z1, 0.0).astype(np.float32))
    z2 = h1.astype(np.float64) @ W2.T.astype(np.float64) + P["b2"]
    h2 = bf16(np.maximum(z2, 0.0).astype(np.float32))
    z3 = h2.astype(np.float64) @ W3.T.astype(np.float64) + P["b3"]
    h3 = bf16(np.maximum(z3, 0.0).astype(np.float32))
    y = (h3.astype(np.float64) @ W4.T.astype(np.float64) + P["b4"]).astype(np.float32)
    return y, (x, h1, h2, h3)


def decode(y):
    y = y.reshape(-1, N_LOBES, 4).astype(np.float64)
    a, b, c, d = y[..., 0], y[..., 1], y[..., 2], y[..., 3]
    a = a - a.max(axis=1, keepdims=True)
    w = np.exp(a) / np.exp(a).sum(axis=1, keepdims=True)
    kappa = np.exp(np.clip(b, KAPPA_LO, KAPPA_HI))
    ct = np.tanh(c)
    st = np.sqrt(np.maximum(0.0, 1.0 - ct * ct))
    ph = np.pi * np.tanh(d)
    mu = np.stack([st * np.cos(ph), st * np.sin(ph), ct], axis=-1)
    return w, kappa, mu


def log_vmf(kappa, cosang):
    """log of kappa / (2 pi (1 - exp(-2 kappa))) exp(kappa (cos - 1))."""
    return np.log(kappa) - np.log(2.0 * np.pi) - np.log1p(-np.exp(-2.0 * kappa)) + kappa * (cosang - 1.0)


def mixture_pdf(y, omega):
    w, kappa, mu = decode(y)
    cosang = np.einsum("nlc,nc->nl", mu, np.asarray(omega, np.float64))
    return (w * np.exp(log_vmf(kappa, cosang))).sum(axis=1)


def loss_and_dy(y, omega, s):
    """Mean weighted negative log-likelihood and its gradient with respect to y."""
    y64 = y.reshape(-1, N_LOBES, 4).astype(np.float64)
    w, kappa, mu = decode(y)
    om = np.asarray(omega, np.float64)
    cosang = np.einsum("nlc,nc->nl", mu, om)
    lv = log_vmf(kappa, cosang)
    lw = np.log(w)
    t = lw + lv
    m = t.max(axis=1, keepdims=True)
    logq = (m + np.log(np.exp(t - m).sum(axis=1, keepdims=True)))[:, 0]
    r = np.exp(t - logq[:, None])
    n = y.shape[0]
    s = np.asarray(s, np.float64)
    loss = float(-(s * logq).sum() / n)
    g = -(s / n)[:, None]  # d loss / d log q per sample
    dy = np.zeros_like(y64)
    dy[..., 0] = g * (r - w)
    dlv_dk = 1.0 / kappa - 2.0 / np.expm1(2.0 * kappa) + (cosang - 1.0)
    b = y64[..., 1]
    inside = (b > KAPPA_LO) & (b < KAPPA_HI)
    dy[..., 1] = g * r * dlv_dk * kappa * inside
    dmu = (g * r * kappa)[..., None] * om[:, None, :]
    ct = np.tanh(y64[..., 2])
    st = np.sqrt(np.maximum(0.0, 1.0 - ct * ct))
    ph = np.pi * np.tanh(y64[..., 3])
    dmu_dc = np.stack([-ct * st * np.cos(ph), -ct * st * np.sin(ph), st * st], axis=-1)  # d mu / d c
    dmu_dd = np.stack([-st * np.sin(ph), st * np.cos(ph), np.zeros_like(ph)], axis=-1) * (
        np.pi * (1.0 - np.tanh(y64[..., 3]) ** 2))[..., None]
    dy[..., 2] = (dmu * dmu_dc).sum(-1)
    dy[..., 3] = (dmu * dmu_dd).sum(-1)
    return loss, dy.reshape(n, N_OUT).astype(np.float32)


def backward(flat, cache, dy):
    """Parameter gradients (packed like the parameters) for output gradient dy."""
    P = unpack(flat)
    x, h1, h2, h3 = cache
    W2, W3, W4 = (bf16(P[k]) for k in ("W2", "W3", "W4"))
    g = {}
    d4 = bf16(dy)
    g["W4"] = (d4.T.astype(np.float64) @ h3.astype(np.float64)).astype(np.float32)
    g["b4"] = d4.astype(np.float64).sum(0).astype(np.float32)
    d3 = bf16(((d4.astype(np.float64) @ W4.astype(np.float64)) * (h3 > 0)).astype(np.float32))
    g["W3"] = (d3.T.astype(np.float64) @ h2.astype(np.float64)).astype(np.float32)
    g["b3"] = d3.astype(np.float64).sum(0).astype(np.float32)
    d2 = bf16(((d3.astype(np.float64) @ W3.astype(np.float64)) * (h2 > 0)).astype(np.float32))
    g["W2"] = (d2.T.astype(np.float64) @ h1.astype(np.float64)).astype(np.float32)
    g["b2"] = d2.astype(np.float64).sum(0).astype(np.float32)
    d1 = bf16(((d2.astype(np.float64) @ W2.astype(np.float64)) * (h1 > 0)).astype(np.float32))
    g["W1"] = (d1.T.astype(np.float64) @ x.astype(np.float64)).astype(np.float32)
    g["W1"][:, 75:] = 0.0
    g["b1"] = d1.astype(np.float64).sum(0).astype(np.float32)
    return pack(g)


def adam(flat, grad, m, v, step, lr=1e-2, beta1=0.9, beta2=0.999, eps=1e-8):
    m = beta1 * m + (1 - beta1) * grad
    v = beta2 * v + (1 - beta2) * grad * grad
    mh = m / (1 - beta1 ** step)
    vh = v / (1 - beta2 ** step)
    return (flat - lr * mh / (np.sqrt(vh) + eps)).astype(np.float32), m, v


def mixture_pdf_from_decoded(decoded, omega):
    """Mixture density at omega from decoded rows (n, 40): 8 x (mu.xyz, kappa) then 8 weights."""
    d = np.asarray(decoded, np.float64)
    mu = d[:, :32].reshape(-1, 8, 4)
    w = d[:, 32:40]
    cosang = np.einsum("nlc,nc->nl", mu[..., :3], np.asarray(omega, np.float64))
    return (w * np.exp(log_vmf(mu[..., 3], cosang))).sum(axis=1)
