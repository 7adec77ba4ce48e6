"""Batched and animated rendering: throughput and per-frame latency against the plain unbatched path.

    python -m toaster_b200.batch_eval [--frames 240] [--width 1280 --height 720] [--spp 32]

Workloads:
- ``uneven``: 16 independent scenes (triangle counts log-uniform in [128, 262,144], resolutions
  320x180 to 1280x720) rendered by one persistent launch (tc_render_batch) versus one tc_render
  per scene. Reports aggregate Mpaths/s of both.
- ``uneven_guided``: the same scenes with guided sampling on, each scene's network trained on its
  own recorded samples: one guided batched launch against guided and plain renders per scene.
- ``animation``: 240 frames of 64 spheres + 64 boxes on ballistic trajectories. The graph path
  replays one captured CUDA graph per frame (pinned staging -> hierarchy update -> render -> device
  display conversion -> RGBA8 readback): with a device refit of frame 0's tree, with a per-frame
  host rebuild, and with the rebuild and guided sampling (network trained on frame 0); the plain
  unbatched path does what the reference does per frame: a full
  scene upload with a host hierarchy build, a plain render, a float4 readback and display
  conversion on the host. Reports per-frame latency (p50 / p99, from the packed frame records to
  RGBA8 bytes on the host) and aggregate Mpaths/s of each.
Host packing of the evaluated frame (scene_to_gpu) is the same for every path and is reported
separately; it is not part of any latency.
"""

from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import configs, guiding_eval
from .renderer import Animation, GpuRenderer, render_batch
from .scene import scene_to_gpu


def host_display_rgba8(hdr: np.ndarray, exposure_stops: float = 0.0) -> np.ndarray:
    """Host display conversion as the reference does it after readback (color.rs:24-74):
    exposure, ACES fitted, clamp, sRGB transfer, rounding half away from zero, in f32."""
    rgb = hdr[..., :3].astype(np.float32) * np.float32(2.0 ** exposure_stops)
    finite = np.isfinite(rgb)
    c = np.where(finite, rgb, np.float32(0.0))
    np.maximum(c, np.float32(0.0), out=c)
    t = (c * (np.float32(2.51) * c + np.float32(0.03))) / (c * (np.float32(2.43) * c + np.float32(0.59)) + np.float32(0.14))
    np.clip(t, np.float32(0.0), np.float32(1.0), out=t)
    if not finite.all():  # NaN and -inf map to 0, +inf to 1
        t[~finite] = (rgb[~finite] == np.inf).astype(np.float32)
    lin = t <= np.float32(0.0031308)
    srgb = np.empty_like(t)
    srgb[lin] = np.float32(12.92) * t[lin]
    srgb[~lin] = np.float32(1.055) * np.power(t[~lin], np.float32(1.0 / 2.4)) - np.float32(0.055)
    out = np.empty(hdr.shape[:-1] + (4,), np.uint8)
    out[..., :3] = np.floor(np.clip(srgb, 0.0, 1.0) * np.float32(255.0) + np.float32(0.5))
    out[..., 3] = np.floor(np.clip(hdr[..., 3], 0.0, 1.0) * np.float32(255.0) + np.float32(0.5))
    return out


def uneven(count: int = 16, samples: int = 32, max_bounces: int = 8, repeats: int = 3, device: int = 0,
           min_width: int = 320, max_width: int = 1280) -> dict:
    """One batched call over `count` uneven scenes against one call per scene: device time of
    the path kernels (CUDA events) and host time of the synchronous calls (each call waits). The
    batched call runs with the automatic schedule (frames of 2^20 paths or more in wavefront calls
    of their own) and as one shared launch of the megakernel over every frame."""
    scenes = configs.uneven_batch(count=count, samples=samples, max_bounces=max_bounces, min_width=min_width,
                                  max_width=max_width)
    rs = [GpuRenderer(device) for _ in scenes]
    try:
        for r, s in zip(rs, scenes):
            r.upload(scene_to_gpu(s))
        paths = sum(s.width * s.height * s.samples for s in scenes)

        def batched_run(schedule):
            render_batch(rs, frame_index=0, schedule=schedule)  # warm-up
            dev, host = [], []
            for k in range(repeats):
                t0 = time.perf_counter()
                st = render_batch(rs, frame_index=1 + k, schedule=schedule)
                host.append((time.perf_counter() - t0) * 1e3)
                dev.append(st["kernel_ms"])
            return float(np.median(dev)), float(np.median(host))

        b, bh = batched_run("auto")
        b1, b1h = batched_run("megakernel")
        for r in rs:
            r.render(frame_index=0)
        single, single_host = [], []
        for k in range(repeats):
            tot = 0.0
            t0 = time.perf_counter()
            for r in rs:
                r.render(frame_index=1 + k)
                tot += r.stats()["kernel_ms"]
            single_host.append((time.perf_counter() - t0) * 1e3)
            single.append(tot)
        u, uh = float(np.median(single)), float(np.median(single_host))
        return {"scenes": count, "triangles": [s.triangle_count for s in scenes],
                "resolutions": [f"{s.width}x{s.height}" for s in scenes], "spp": samples, "max_bounces": max_bounces,
                "paths": paths, "batched_ms": b, "unbatched_ms": u, "batched_mpaths_per_s": paths / (b * 1e3),
                "unbatched_mpaths_per_s": paths / (u * 1e3), "speedup": u / b,
                "batched_host_ms": bh, "unbatched_host_ms": uh, "host_speedup": uh / bh,
                "one_launch_ms": b1, "one_launch_mpaths_per_s": paths / (b1 * 1e3), "one_launch_host_ms": b1h}
    finally:
        for r in rs:
            r.close()


def uneven_guided(count: int = 16, samples: int = 32, max_bounces: int = 8, repeats: int = 3, record_spp: int = 8,
                  train_steps: int = guiding_eval.TRAIN_STEPS, device: int = 0, min_width: int = 320,
                  max_width: int = 1280) -> dict:
    """The uneven scene set with guided sampling on: every scene trains its own network on its own
    recorded samples (record_spp plain spp, the guiding recipe's Adam steps), then one guided
    batched launch over all scenes (each frame's queries inferred by its own network) against one
    guided tc_render per scene and one plain tc_render per scene. Device time of the path and
    inference kernels; per-scene times of the unbatched calls give their p50 / p99."""
    scenes = configs.uneven_batch(count=count, samples=samples, max_bounces=max_bounces, min_width=min_width,
                                  max_width=max_width)
    rs = [GpuRenderer(device) for _ in scenes]
    try:
        train_ms = 0.0
        for i, (r, s) in enumerate(zip(rs, scenes)):
            r.upload(scene_to_gpu(s))
            r.guide_set_params(guiding_eval.initial_params(i), configs.scene_bounds(s))
            r.render(samples=record_spp, frame_index=0, guide_record=True)
            r.guide_train_recorded(train_steps, 8192, 1e-2, i)
            train_ms += r.stats()["kernel_ms"]
        paths = sum(s.width * s.height * s.samples for s in scenes)
        render_batch(rs, frame_index=1, guiding=True)  # warm-up
        batched = [render_batch(rs, frame_index=2 + k, guiding=True)["kernel_ms"] for k in range(repeats)]
        render_batch(rs, frame_index=1, guiding=True, schedule="megakernel")
        one_launch = [render_batch(rs, frame_index=2 + k, guiding=True, schedule="megakernel")["kernel_ms"]
                      for k in range(repeats)]
        per_scene = {"guided": [], "plain": []}
        totals = {"guided": [], "plain": []}
        for key, guided in (("guided", True), ("plain", False)):
            for r in rs:
                r.render(frame_index=1, guiding=guided)
            for k in range(repeats):
                tot = 0.0
                for r in rs:
                    r.render(frame_index=2 + k, guiding=guided)
                    ms = r.stats()["kernel_ms"]
                    tot += ms
                    per_scene[key].append(ms)
                totals[key].append(tot)
        b = float(np.median(batched))
        g, pl = float(np.median(totals["guided"])), float(np.median(totals["plain"]))
        return {"scenes": count, "spp": samples, "max_bounces": max_bounces, "paths": paths,
                "train_ms_all_scenes": train_ms, "batched_guided_ms": b, "unbatched_guided_ms": g,
                "one_launch_guided_ms": float(np.median(one_launch)),
                "one_launch_guided_mpaths_per_s": paths / (float(np.median(one_launch)) * 1e3),
                "unbatched_plain_ms": pl, "batched_guided_mpaths_per_s": paths / (b * 1e3),
                "unbatched_guided_mpaths_per_s": paths / (g * 1e3), "unbatched_plain_mpaths_per_s": paths / (pl * 1e3),
                "guided_scene_ms_p50": float(np.percentile(per_scene["guided"], 50)),
                "guided_scene_ms_p99": float(np.percentile(per_scene["guided"], 99)),
                "plain_scene_ms_p50": float(np.percentile(per_scene["plain"], 50)),
                "plain_scene_ms_p99": float(np.percentile(per_scene["plain"], 99))}
    finally:
        for r in rs:
            r.close()


def animation(frames: int = 240, width: int = 1280, height: int = 720, samples: int = 32, max_bounces: int = 8,
              guiding: bool = True, train_steps: int = guiding_eval.TRAIN_STEPS, device: int = 0) -> dict:
    anim = configs.BallisticAnimation(width=width, height=height, samples=samples, max_bounces=max_bounces,
                                      frames=frames)
    pack_times = []

    def packed(k):
        t = time.perf_counter()
        data = scene_to_gpu(anim.scene(k))
        pack_times.append((time.perf_counter() - t) * 1e3)
        return data

    first = packed(0)
    paths = width * height * samples
    out = {"frames": frames, "width": width, "height": height, "spp": samples, "max_bounces": max_bounces,
           "primitives": int(anim.n_spheres + 2 + 12 * anim.n_boxes)}
    # Graph paths: refit and per-frame rebuild with plain sampling, then rebuild with guided
    # sampling (network trained on frame 0).
    variants = [("graph_refit", False, False), ("graph", False, True)]
    if guiding:
        variants.append(("graph_guided", True, True))
    for key, guided, rebuild in variants:
        with GpuRenderer(device) as r:
            r.upload(first)
            train_ms = 0.0
            if guided:
                r.guide_set_params(guiding_eval.initial_params(0), configs.scene_bounds(anim.scene(0)))
                r.render(samples=16, frame_index=0, guide_record=True)
                r.guide_train_recorded(train_steps, 8192, 1e-2, 1)
                train_ms = r.stats()["kernel_ms"]
            lat = []
            with Animation(r, first, guiding=guided, update_lights=True, rebuild=rebuild) as a:
                img = np.empty((height, width, 4), np.uint8)
                a.frame(first, 0, img)  # warm-up replay
                for k in range(frames):
                    data = packed(k)
                    t = time.perf_counter()
                    a.frame(data, k, img)
                    lat.append((time.perf_counter() - t) * 1e3)
            lat = np.array(lat)
            out[key] = {
                "guided": guided, "hierarchy": "rebuild" if rebuild else "refit", "train_ms": train_ms,
                "p50_ms": float(np.percentile(lat, 50)),
                "p99_ms": float(np.percentile(lat, 99)), "mean_ms": float(lat.mean()),
                "mpaths_per_s": paths * frames / (lat.sum() * 1e3)}
    # Plain unbatched path (the reference's per-frame flow).
    with GpuRenderer(device) as r:
        lat, conv = [], []
        r.upload(first)
        r.render(frame_index=0)
        for k in range(frames):
            data = packed(k)
            t = time.perf_counter()
            r.upload(data)
            r.render(frame_index=k)
            hdr = r.readback()
            t1 = time.perf_counter()
            host_display_rgba8(hdr)
            t2 = time.perf_counter()
            lat.append((t2 - t) * 1e3)
            conv.append((t2 - t1) * 1e3)
        lat = np.array(lat)
        out["plain_unbatched"] = {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                                  "mean_ms": float(lat.mean()), "mpaths_per_s": paths * frames / (lat.sum() * 1e3),
                                  "host_conversion_ms": float(np.mean(conv))}
    out["host_pack_ms_per_frame"] = float(np.mean(pack_times))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--frames", type=int, default=240)
    ap.add_argument("--width", type=int, default=1280)
    ap.add_argument("--height", type=int, default=720)
    ap.add_argument("--spp", type=int, default=32)
    ap.add_argument("--no-guiding", action="store_true")
    ap.add_argument("--only", choices=["uneven", "uneven_guided", "uneven_small", "animation"], default=None)
    args = ap.parse_args()
    if args.only == "uneven_guided":
        print(json.dumps({"uneven_guided": uneven_guided(samples=args.spp)}), flush=True)
        return
    print(json.dumps({"uneven": uneven(samples=args.spp)}), flush=True)
    if not args.no_guiding:
        print(json.dumps({"uneven_guided": uneven_guided(samples=args.spp)}), flush=True)
    print(json.dumps({"uneven_small": uneven(samples=4, max_bounces=4, min_width=160, max_width=480)}), flush=True)
    print(json.dumps({"animation": animation(args.frames, args.width, args.height, args.spp,
                                             guiding=not args.no_guiding)}), flush=True)


if __name__ == "__main__":
    main()
