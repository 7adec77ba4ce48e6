"""Throughput of the path kernel on the named workloads (one JSON line each).

    python -m toaster_b200.measure [plain_small|mixed|large_mesh|room] [--spp N] [--frames K]
        [--schedule auto|megakernel|wavefront] [--wave-paths N] [--ray-sort] [--guided]

Reports Mpaths/s, Mrays/s (device-counted extension + shadow rays) and the kernel time per frame
(CUDA events on the library's stream), for progressive accumulation of `frames` batches of
`spp` samples per pixel. The scene is uploaded once (hierarchy built on the host).
"""

from __future__ import annotations

import argparse
import json
import statistics
import time

from . import configs
from .renderer import GpuRenderer
from .scene import scene_to_gpu

WORKLOADS = {
    "plain_small": lambda: configs.plain_small(),
    "mixed": lambda: configs.mixed(),
    "large_mesh": lambda: configs.large_mesh(),
    "room": lambda: configs.room_with_window(),
}


def measure(name: str, spp: int | None = None, frames: int = 3, warmup: int = 1, device: int = 0,
            schedule: str = "auto", wave_paths: int = 0, ray_sort: bool = False, guided: bool = False) -> dict:
    """``guided``: guided sampling with the untrained initial network (timing only)."""
    scene = WORKLOADS[name]()
    spp = spp or scene.samples
    t0 = time.perf_counter()
    data = scene_to_gpu(scene)
    opts = dict(schedule=schedule, wave_paths=wave_paths, ray_sort=2 if ray_sort else 0, guiding=guided)
    with GpuRenderer(device) as r:
        r.upload(data)
        upload_s = time.perf_counter() - t0
        if guided:
            from .guiding_eval import initial_params

            r.guide_set_params(initial_params(0), configs.scene_bounds(scene))
        for i in range(warmup):
            r.render(samples=spp, frame_index=i, **opts)
        ms, rays, paths = [], [], []
        for k in range(frames):
            r.render(samples=spp, frame_index=warmup + k, accumulate=k > 0, **opts)
            st = r.stats()
            ms.append(st["kernel_ms"])
            rays.append(st["rays"])
            paths.append(st["paths"])
        depth = r.stats()["bvh_depth"]
    t = sum(ms) * 1e-3
    return {
        "workload": name, "width": scene.width, "height": scene.height, "spp_per_frame": spp, "frames": frames,
        "max_bounces": scene.max_bounces, "triangles": scene.triangle_count, "spheres": scene.sphere_count,
        "bvh_depth": depth, "mpaths_per_s": sum(paths) / t / 1e6, "mrays_per_s": sum(rays) / t / 1e6,
        "rays_per_path": sum(rays) / max(sum(paths), 1), "kernel_ms_per_frame": statistics.mean(ms),
        "kernel_ms_min": min(ms), "upload_s": upload_s, "schedule": schedule, "wave_paths": wave_paths,
        "ray_sort": ray_sort, "guided": guided,
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("workloads", nargs="*", default=list(WORKLOADS))
    ap.add_argument("--spp", type=int, default=0)
    ap.add_argument("--frames", type=int, default=3)
    ap.add_argument("--schedule", choices=["auto", "megakernel", "wavefront"], default="auto")
    ap.add_argument("--wave-paths", type=int, default=0)
    ap.add_argument("--ray-sort", action="store_true")
    ap.add_argument("--guided", action="store_true")
    args = ap.parse_args()
    for name in args.workloads:
        print(json.dumps(measure(name, args.spp or None, args.frames, schedule=args.schedule,
                                 wave_paths=args.wave_paths, ray_sort=args.ray_sort, guided=args.guided)), flush=True)


if __name__ == "__main__":
    main()
