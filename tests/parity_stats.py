"""Statistics of the image-parity tests: two renders of one scene by independent estimators.

Both sides bring per-pixel means and per-pixel sample variances (from sums of squared samples),
so every comparison is scaled by the variance of the *difference* of the two means,
var_gpu / n_gpu + var_oracle / n_oracle, and an estimator that inflates its own variance does not
widen its own band by itself. Reported:

- ``outside_pixel``: fraction of (pixel, channel) z-scores beyond 3 sigma;
- ``outside_block``: the same for the luminance of 2x2 pixel blocks;
- ``median_z``: median block z-score (a consistent bias shifts it);
- ``global_dz``: difference of the image-mean luminances in standard errors, and ``rel_mean`` the
  same difference relative to the oracle's image mean (``rel_se`` is one standard error of it, in
  the same units).

Luminance variances are bounded by the perfectly correlated case, (sum_c w_c sigma_c)^2, because
only per-channel sums of squares are kept and the channels of one path are strongly correlated.

The oracle returns its means as FP32 sums of FP32 samples (relative error up to about 4e-6 over
4,096 terms), so sum_sq / n - mean^2 loses every per-sample variance below about 1e-5 mean^2 to
cancellation: a sky pixel whose jittered samples differ by a part in a thousand shows a variance
of zero or noise. Each side's per-sample variance is therefore floored at 1e-5 mean^2; only pixels
that are zero on both sides are required to agree exactly.
"""

from __future__ import annotations

import numpy as np

LUMA = np.array([0.2126, 0.7152, 0.0722])
VAR_FLOOR = 1e-5


def sample_variance(mean: np.ndarray, sumsq: np.ndarray, n: int) -> np.ndarray:
    """Unbiased per-pixel per-channel sample variance from the mean and the sum of squares."""
    mean = mean.astype(np.float64)
    return np.maximum(sumsq / n - mean**2, 0.0) * n / max(n - 1, 1)


def _blocks(x: np.ndarray, b: int) -> np.ndarray:
    h, w = x.shape
    h2, w2 = h // b * b, w // b * b
    return x[:h2, :w2].reshape(h2 // b, b, w2 // b, b).sum(axis=(1, 3))


def compare(g_mean, g_var, n_g, o_mean, o_var, n_o, block: int = 2) -> dict:
    """Parity statistics of two (height, width, 3) mean images with their sample variances."""
    g_mean = g_mean.astype(np.float64)
    o_mean = o_mean.astype(np.float64)
    # Variance of the difference of the two means, each side's per-sample variance floored at the
    # level that FP32 means leave measurable.
    g_var = np.maximum(g_var, VAR_FLOOR * g_mean**2)
    o_var = np.maximum(o_var, VAR_FLOOR * o_mean**2)
    var = g_var / n_g + o_var / n_o
    diff = g_mean - o_mean
    flat = var <= 0.0
    # Pixels that are zero on both sides (black) must agree exactly.
    const_bad = int(np.sum(diff[flat] != 0.0))
    z = diff[~flat] / np.sqrt(var[~flat])
    sd_l = np.sqrt(var) @ LUMA  # per-pixel luminance standard deviation bound
    d_l = diff @ LUMA
    bd = _blocks(d_l, block)
    bv = _blocks(sd_l**2, block)
    bz = bd[bv > 0] / np.sqrt(bv[bv > 0])
    o_l = o_mean @ LUMA
    se = float(np.sqrt(np.sum(sd_l**2))) / d_l.size
    delta = float(d_l.mean())
    return {
        "outside_pixel": float(np.mean(np.abs(z) > 3.0)) if z.size else 0.0,
        "outside_block": float(np.mean(np.abs(bz) > 3.0)) if bz.size else 0.0,
        "median_z": float(np.median(bz)) if bz.size else 0.0,
        "global_dz": delta / se if se > 0 else 0.0,
        "rel_mean": abs(delta) / max(abs(float(o_l.mean())), 1e-12),
        "rel_se": se / max(abs(float(o_l.mean())), 1e-12),
        "constant_mismatch": const_bad,
        "pixels": int(d_l.size),
    }
