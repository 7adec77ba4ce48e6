"""Equal-time comparison of guided and plain path tracing.

    python -m toaster_b200.guiding_eval [--width W --height H --ref-spp N --plain-spp 256]

Protocol:
- A converged reference is rendered with plain sampling and FP64 accumulation.
- Plain sampling accumulates batches of `batch` spp up to `plain_spp`. After each batch the GPU time
  so far and the RGB RMSE against the reference are recorded.
- Guided sampling starts with `record_spp` plain spp that also record training samples at every
  diffuse scatter (these samples stay in the image). It then trains the network on the GPU with
  Adam, and accumulates guided batches. Training time counts toward the guided timeline.
- The result is the guided time needed to reach the plain method's RMSE at `plain_spp`, as a
  fraction of the plain time.
"""

from __future__ import annotations

import argparse
import json
import time
from pathlib import Path

import numpy as np

from . import configs
from .renderer import GpuRenderer
from .scene import Scene, scene_to_gpu

# Adam steps of the guiding recipe (batch 8,192, lr 1e-2) on the 16 recorded spp. Training acts as
# an early stop: on the window room the per-pixel variance of guided sampling is lowest after 100-200
# steps and rises as the loss keeps falling (the target, a one-sample estimate from 16 spp, rewards
# lobes that are too narrow).
TRAIN_STEPS = 200
# Online training: after every guided batch, that batch's samples (recorded under the guided
# mixture, weighted by cos / (pi p)) join the pool and the network takes ONLINE_STEPS more Adam
# steps of ONLINE_BATCH samples on the whole pool, so the fit sharpens only as fast as its data
# grows (window room, 3 seeds, trimmed time fraction: 0.87-0.96 and one seed that never reached
# plain's error without it; 0.72-0.88 with 25 steps of 8,192; 0.72-0.81 with 100 of 32,768).
ONLINE_STEPS = 100
ONLINE_BATCH = 32768


def initial_params(seed: int = 0) -> np.ndarray:
    """He-uniform hidden layers, a 10x smaller output layer, zero biases, zero padded inputs."""
    rng = np.random.default_rng(seed)
    shapes = [(64, 80), (64,), (64, 64), (64,), (64, 64), (64,), (32, 64), (32,)]
    out = []
    for k, shape in enumerate(shapes):
        if len(shape) == 1:
            out.append(np.zeros(shape, np.float32))
            continue
        fan_in = 75 if k == 0 else shape[1]
        bound = np.sqrt(6.0 / fan_in) * (0.1 if k == 6 else 1.0)
        w = rng.uniform(-bound, bound, shape).astype(np.float32)
        if k == 0:
            w[:, 75:] = 0.0
        out.append(w)
    return np.concatenate([a.reshape(-1) for a in out])


def _image(r: GpuRenderer) -> np.ndarray:
    s, _, n = r.readback_sums()
    return s / n


def reference_image(scene: Scene, spp: int, batch: int = 256, device: int = 0) -> np.ndarray:
    with GpuRenderer(device) as r:
        r.upload(scene_to_gpu(scene))
        done = 0
        while done < spp:
            n = min(batch, spp - done)
            r.render(samples=n, frame_index=1_000_000 + done, accumulate=done > 0)
            done += n
        return _image(r)


def band_rows(height: int, bands: int, rows: int) -> np.ndarray:
    """Image rows of `bands` evenly spaced bands of `rows` rows each (the first band centred in the
    first 1/bands of the image, and so on)."""
    starts = [int((k + 0.5) * height / bands) - rows // 2 for k in range(bands)]
    return np.concatenate([np.arange(max(0, y), min(height, y + rows)) for y in starts])


def reference_bands(scene: Scene, spp: int, bands: int = 4, rows: int = 8, batch: int = 1024,
                    device: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """Plain FP64 reference of `spp` samples per pixel on the rows of `band_rows` only: each band is
    rendered as its own frame whose camera is the full frame's with the image plane cut to the
    band (lower-left corner moved up by the rows below it, vertical extent scaled to its rows),
    so its pixel (x, y') sees what pixel (x, y0 + y') of the full frame sees. Returns (rows, image
    of those rows)."""
    data = scene_to_gpu(scene)
    h = scene.height
    starts = [int((k + 0.5) * h / bands) - rows // 2 for k in range(bands)]
    out = []
    with GpuRenderer(device) as r:
        for band, y0 in enumerate(starts):
            y0, y1 = max(0, y0), min(h, y0 + rows)
            cam = data.camera.copy()
            v = cam["vertical"][0].astype(np.float64)
            cam["lower_left_corner"][0] = (cam["lower_left_corner"][0].astype(np.float64) +
                                           v * (1.0 - y1 / h)).astype(np.float32)
            cam["vertical"][0] = (v * ((y1 - y0) / h)).astype(np.float32)
            params = data.params.copy()
            params["height"] = y1 - y0
            r.upload(type(data)(**{**data.__dict__, "camera": cam, "params": params}))
            done = 0
            while done < spp:
                n = min(batch, spp - done)
                # Each band draws its own streams (pixel indices restart at 0 in every band).
                r.render(samples=n, frame_index=(1 + band) * 1_000_000 + done, accumulate=done > 0)
                done += n
            out.append(_image(r))
    return band_rows(h, bands, rows), np.concatenate(out, axis=0)


def rmse(a: np.ndarray, b: np.ndarray) -> float:
    return float(np.sqrt(np.mean((a - b) ** 2)))


def trimmed_rmse(a: np.ndarray, b: np.ndarray, keep: float = 0.999) -> float:
    """RMSE over the pixels whose squared error is at or below the ``keep`` quantile: the same
    error with the rarest outliers (single bright samples) left out, a steadier statistic for
    comparing two unbiased estimators from one run each."""
    e = ((a - b) ** 2).mean(axis=-1).ravel()
    return float(np.sqrt(e[e <= np.quantile(e, keep)].mean()))


def timeline_plain(scene: Scene, reference: np.ndarray, total_spp: int, batch: int, device: int = 0,
                   frame_offset: int = 0, rows: np.ndarray | None = None):
    points = []
    with GpuRenderer(device) as r:
        r.upload(scene_to_gpu(scene))
        t = 0.0
        done = 0
        while done < total_spp:
            n = min(batch, total_spp - done)
            r.render(samples=n, frame_index=frame_offset + done, accumulate=done > 0)
            t += r.stats()["total_ms"] * 1e-3
            done += n
            img = _image(r) if rows is None else _image(r)[rows]
            points.append((t, done, rmse(img, reference), trimmed_rmse(img, reference)))
    return points


def timeline_guided(scene: Scene, reference: np.ndarray, total_spp: int, batch: int, record_spp: int,
                    train_steps: int, train_batch: int, lr: float = 1e-2, seed: int = 0, device: int = 0,
                    frame_offset: int = 0, rows: np.ndarray | None = None, online_steps: int = 0,
                    online_lr: float | None = None, online_batch: int | None = None, guide_fraction: float = 0.0):
    """Recorded plain batch, training, then guided batches; with ``online_steps`` every guided
    batch but the last also records into the sample pool and is followed by that many Adam steps.
    Training time counts towards the timeline."""
    points = []
    info = {}
    with GpuRenderer(device) as r:
        r.upload(scene_to_gpu(scene))
        r.guide_set_params(initial_params(seed), configs.scene_bounds(scene))
        r.render(samples=record_spp, frame_index=frame_offset, guide_record=True)
        t = r.stats()["total_ms"] * 1e-3
        img = _image(r) if rows is None else _image(r)[rows]
        points.append((t, record_spp, rmse(img, reference), trimmed_rmse(img, reference)))
        t0 = time.perf_counter()
        losses, n = r.guide_train_recorded(train_steps, train_batch, lr, seed)
        train_s = r.stats()["kernel_ms"] * 1e-3
        info.update(train_seconds=train_s, train_host_seconds=time.perf_counter() - t0, samples=n,
                    loss_first=float(losses[:5].mean()), loss_last=float(losses[-5:].mean()))
        t += train_s
        done = record_spp
        online_s = 0.0
        while done < total_spp:
            m = min(batch, total_spp - done)
            learn = online_steps > 0 and done + m < total_spp
            r.render(samples=m, frame_index=frame_offset + done, accumulate=True, guiding=True,
                     guide_record=2 if learn else 0, guide_fraction=guide_fraction)
            t += r.stats()["total_ms"] * 1e-3
            done += m
            img = _image(r) if rows is None else _image(r)[rows]
            points.append((t, done, rmse(img, reference), trimmed_rmse(img, reference)))
            if learn:
                _, n = r.guide_train_recorded(online_steps, online_batch or ONLINE_BATCH, online_lr or lr,
                                              seed * 1_000_003 + done)
                online_s += r.stats()["kernel_ms"] * 1e-3
                t += r.stats()["kernel_ms"] * 1e-3
                info["pool_samples"] = n
        info["online_train_seconds"] = online_s
    return points, info


def time_to_reach(points, target: float, col: int = 2):
    """Earliest (interpolated in log error between batches) time at which the error in column
    ``col`` (2 = RMSE, 3 = trimmed RMSE) is <= target, or None."""
    prev = None
    for p in points:
        t, e = p[0], p[col]
        if e <= target:
            if prev is None or prev[1] <= e:
                return t
            t0, e0 = prev
            f = (np.log(e0) - np.log(target)) / (np.log(e0) - np.log(e))
            return t0 + f * (t - t0)
        prev = (t, e)
    return None


def equal_time_comparison(scene: Scene, ref_spp: int, plain_spp: int = 256, batch: int = 16, record_spp: int = 16,
                          guided_spp: int | None = None, train_steps: int | None = None, train_batch: int = 8192,
                          seed: int = 0, device: int = 0, reference: np.ndarray | None = None,
                          rows: np.ndarray | None = None, online_steps: int | None = None,
                          online_lr: float | None = None, online_batch: int | None = None,
                          guide_fraction: float = 0.0) -> dict:
    """``rows``: the RMSE is taken over these image rows only, against a ``reference`` of them
    (``reference_bands``). ``online_steps``: Adam steps after each guided batch (default
    ONLINE_STEPS; 0 = train once on the recorded batch only)."""
    if reference is None:
        reference = reference_image(scene, ref_spp, device=device)
    train_steps = TRAIN_STEPS if train_steps is None else train_steps
    # Each seed draws its own path samples (frame indices offset by 100,000 per seed).
    plain = timeline_plain(scene, reference, plain_spp, batch, device, frame_offset=100_000 * seed, rows=rows)
    online_steps = ONLINE_STEPS if online_steps is None else online_steps
    guided, info = timeline_guided(scene, reference, guided_spp or plain_spp, batch, record_spp, train_steps,
                                   train_batch, seed=seed, device=device, frame_offset=100_000 * seed, rows=rows,
                                   online_steps=online_steps, online_lr=online_lr, online_batch=online_batch,
                                   guide_fraction=guide_fraction)
    t_plain, _, e_plain, et_plain = plain[-1]
    t_guided = time_to_reach(guided, e_plain)
    tt_guided = time_to_reach(guided, et_plain, col=3)
    e_at, et_at = None, None
    for t, _, e, et in guided:
        if t <= t_plain:
            e_at, et_at = e, et
    return {
        "width": scene.width, "height": scene.height, "max_bounces": scene.max_bounces, "reference_spp": ref_spp,
        "plain_spp": plain_spp, "online_steps": online_steps, "plain_seconds": t_plain, "plain_rmse": e_plain,
        "guided_seconds_to_plain_rmse": t_guided,
        "time_fraction": None if t_guided is None else t_guided / t_plain,
        "guided_rmse_at_plain_time": e_at,
        "plain_trimmed_rmse": et_plain,
        "time_fraction_trimmed": None if tt_guided is None else tt_guided / t_plain,
        "guided_trimmed_rmse_at_plain_time": et_at,
        "plain_timeline": plain, "guided_timeline": guided, **info,
    }


def kernel_timings(width: int = 1280, height: int = 720, record_spp: int = 16, train_steps: int = 600,
                   train_batch: int = 8192, queries: int = 1 << 20, guided_spp: int = 16, device: int = 0) -> dict:
    """Throughput of the network kernels on the guiding workload: training (fused forward +
    backward + Adam per step) on the recorded samples, inference on `queries` recorded
    (position, normal) pairs, and one guided batch. FLOP counts: 30,080 per inference query,
    90,240 per training sample (forward + two backward contractions); rates against the
    measured burst bf16 tensor peak."""
    peaks = json.loads((Path(__file__).resolve().parents[1] / "MEASURED_PEAKS.json").read_text()) \
        if (Path(__file__).resolve().parents[1] / "MEASURED_PEAKS.json").exists() else {}
    peak = float(peaks.get("bf16_tflops", 1590.0))
    scene = configs.room_with_window(width=width, height=height)
    with GpuRenderer(device) as r:
        r.upload(scene_to_gpu(scene))
        r.guide_set_params(initial_params(0), configs.scene_bounds(scene))
        r.render(samples=record_spp, frame_index=0, guide_record=True)
        _, n = r.guide_train_recorded(train_steps, train_batch, 1e-2, 0)
        train_ms = r.stats()["kernel_ms"]
        rec = r.guide_recorded_samples()
        idx = np.resize(np.arange(len(rec)), queries)
        pts, nrm = rec[idx, :3], rec[idx, 4:7]
        infer_ms = []
        for _ in range(5):
            r.guide_infer(pts, nrm)
            infer_ms.append(r.stats()["kernel_ms"])
        r.render(samples=guided_spp, frame_index=record_spp, accumulate=True, guiding=True)
        guided = r.stats()
    train_tflops = train_steps * train_batch * 90240 / (train_ms * 1e-3) / 1e12
    infer = float(np.median(infer_ms))
    infer_tflops = queries * 30080 / (infer * 1e-3) / 1e12
    return {"width": width, "height": height, "training_samples": n, "train_steps": train_steps,
            "train_batch": train_batch, "train_ms": train_ms, "train_us_per_step": train_ms * 1e3 / train_steps,
            "train_tflops": train_tflops, "train_frac_of_measured_peak": train_tflops / peak,
            "infer_queries": queries, "infer_ms": infer, "infer_mqueries_per_s": queries / infer / 1e3,
            "infer_tflops": infer_tflops, "infer_frac_of_measured_peak": infer_tflops / peak,
            "guided_spp": guided_spp, "guided_kernel_ms": guided["kernel_ms"], "guided_total_ms": guided["total_ms"],
            "peak_bf16_tflops": peak}


def main():
    """Defaults are the learned-guiding workload: the window room (8,192 clutter triangles, 30%
    metal) at 1280x720, 8 bounces, a 65,536-spp reference, 256 plain spp, 16 recorded spp."""
    ap = argparse.ArgumentParser()
    ap.add_argument("--width", type=int, default=1280)
    ap.add_argument("--height", type=int, default=720)
    ap.add_argument("--ref-spp", type=int, default=65536)
    ap.add_argument("--plain-spp", type=int, default=256)
    ap.add_argument("--guided-spp", type=int, default=0)
    ap.add_argument("--record-spp", type=int, default=16)
    ap.add_argument("--train-steps", type=int, default=0, help=f"Adam steps (default {TRAIN_STEPS}; --kernels: 600)")
    ap.add_argument("--online-steps", type=int, default=-1,
                    help=f"Adam steps after each guided batch (default {ONLINE_STEPS}; 0 = none)")
    ap.add_argument("--clutter", type=int, default=8192)
    ap.add_argument("--metal", type=float, default=0.3)
    ap.add_argument("--seeds", type=int, default=1)
    ap.add_argument("--timelines", action="store_true")
    ap.add_argument("--kernels", action="store_true",
                    help="only time the network kernels (training, inference, one guided batch)")
    args = ap.parse_args()
    if args.kernels:
        print(json.dumps(kernel_timings(args.width, args.height, args.record_spp, args.train_steps or 600)),
              flush=True)
        return
    scene = configs.room_with_window(width=args.width, height=args.height, clutter=args.clutter,
                                     metal_fraction=args.metal)
    t0 = time.perf_counter()
    reference = reference_image(scene, args.ref_spp)
    print(json.dumps({"reference_spp": args.ref_spp, "reference_seconds": time.perf_counter() - t0}), flush=True)
    for seed in range(args.seeds):
        out = equal_time_comparison(scene, args.ref_spp, args.plain_spp, record_spp=args.record_spp,
                                    guided_spp=args.guided_spp or None, train_steps=args.train_steps or None, seed=seed,
                                    reference=reference, online_steps=None if args.online_steps < 0 else args.online_steps)
        if not args.timelines:
            out.pop("plain_timeline")
            out.pop("guided_timeline")
        out["seed"] = seed
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
