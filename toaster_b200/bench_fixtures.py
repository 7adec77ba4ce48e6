"""toaster's geometry-scaling benchmark suite, regenerated, and its benchmark protocol on the GPU.

The reference publishes GPU timings for seven deterministic fixtures
(README.md:127-148, docs/benchmarks/post-bvh/rtx-2080-ti): terrain meshes of 128 / 2,048 / 8,192
triangles, 64 and 512 spheres, a terrain-plus-128-spheres mix and an environment-lit control, all
at 320x180, 4 spp, 4 bounces, black background, measured as 2 warm-up and 5 measured frames with
frame seed 0 and reported as the median ``dispatch_wait_ms``. ``write_suite`` writes the same
scene and glTF files as the reference's generator (scripts/generate_benchmark_scenes.py: the
analytic terrain height and normal, two triangles per grid cell, the sphere lattice, the shared
camera, materials and light) into a directory laid out like the reference tree, so the
scenes' relative asset paths resolve. The environment control's 4x2 Radiance map is not
generated by that script; a 4x2 stand-in with a bright top row is written in its place.

    python -m toaster_b200.bench_fixtures --out /tmp/suite     # write, load natively, render, report
"""

from __future__ import annotations

import argparse
import base64
import json
import math
import statistics
import struct
import time
from pathlib import Path

RENDER = {"width": 320, "height": 180, "samples": 4, "max_bounces": 4, "background": "black"}
CAMERA = {"position": [0.0, 5.5, 8.0], "look_at": [0.0, 0.0, 0.0], "up": [0.0, 1.0, 0.0], "fov_degrees": 45.0}
MATERIALS = [
    {"name": "surface", "type": "diffuse", "albedo": [0.62, 0.68, 0.74]},
    {"name": "accent", "type": "metal", "albedo": [0.82, 0.48, 0.2], "roughness": 0.2},
    {"name": "light", "type": "emissive", "color": [1.0, 0.92, 0.78], "strength": 14.0},
]
SCENES = ["001_triangles_128.json", "002_triangles_2048.json", "003_triangles_8192.json", "004_spheres_64.json",
          "005_spheres_512.json", "006_mixed_2048t_128s.json", "007_environment_control.json"]

# Published RTX 2080 Ti / Vulkan medians (README.md:135-141): dispatch_wait_ms and total_ms.
PUBLISHED_2080TI = {
    "001_triangles_128.json": (0.597, 1.856),
    "002_triangles_2048.json": (0.968, 2.906),
    "003_triangles_8192.json": (1.457, 6.183),
    "004_spheres_64.json": (1.129, 2.380),
    "005_spheres_512.json": (1.752, 3.142),
    "006_mixed_2048t_128s.json": (2.478, 4.558),
    "007_environment_control.json": (0.671, 1.887),
}


def _dump(path: Path, value) -> None:
    path.parent.mkdir(parents=True, exist_ok=True)
    path.write_text(json.dumps(value, indent=2) + "\n", encoding="utf-8")


def _height(x: float, z: float) -> float:
    return 0.16 * math.sin(0.9 * x) * math.cos(0.9 * z)


def _normal(x: float, z: float) -> tuple:
    dx = 0.144 * math.cos(0.9 * x) * math.cos(0.9 * z)
    dz = -0.144 * math.sin(0.9 * x) * math.sin(0.9 * z)
    n = (-dx, 1.0, -dz)
    length = math.sqrt(sum(c * c for c in n))
    return tuple(c / length for c in n)


def terrain_gltf(subdivisions: int) -> dict:
    """An 8 x 8 terrain grid, two triangles per cell, positions + normals + u16 indices in one
    embedded buffer."""
    extent = 4.0
    pos, nrm = [], []
    for row in range(subdivisions + 1):
        z = -extent + 2.0 * extent * row / subdivisions
        for col in range(subdivisions + 1):
            x = -extent + 2.0 * extent * col / subdivisions
            pos.extend((x, _height(x, z), z))
            nrm.extend(_normal(x, z))
    idx, w = [], subdivisions + 1
    for row in range(subdivisions):
        for col in range(subdivisions):
            ll = row * w + col
            lr, ul = ll + 1, ll + w
            idx.extend((ll, ul, lr))
            idx.extend((lr, ul, ul + 1))
    pb, nb, ib = struct.pack(f"<{len(pos)}f", *pos), struct.pack(f"<{len(nrm)}f", *nrm), struct.pack(f"<{len(idx)}H", *idx)
    payload = pb + nb + ib
    return {
        "asset": {"version": "2.0", "generator": "Toaster benchmark fixture generator"},
        "scene": 0,
        "scenes": [{"nodes": [0]}],
        "nodes": [{"mesh": 0}],
        "meshes": [{"name": f"BenchmarkTerrain{subdivisions}",
                    "primitives": [{"attributes": {"POSITION": 0, "NORMAL": 1}, "indices": 2, "mode": 4}]}],
        "accessors": [
            {"bufferView": 0, "componentType": 5126, "count": len(pos) // 3, "type": "VEC3",
             "min": [-extent, -0.16, -extent], "max": [extent, 0.16, extent]},
            {"bufferView": 1, "componentType": 5126, "count": len(nrm) // 3, "type": "VEC3"},
            {"bufferView": 2, "componentType": 5123, "count": len(idx), "type": "SCALAR"},
        ],
        "bufferViews": [
            {"buffer": 0, "byteOffset": 0, "byteLength": len(pb), "target": 34962},
            {"buffer": 0, "byteOffset": len(pb), "byteLength": len(nb), "target": 34962},
            {"buffer": 0, "byteOffset": len(pb) + len(nb), "byteLength": len(ib), "target": 34963},
        ],
        "buffers": [{"byteLength": len(payload),
                     "uri": "data:application/octet-stream;base64," + base64.b64encode(payload).decode("ascii")}],
    }


def _scene(objects: list) -> dict:
    return {"camera": CAMERA, "render": RENDER, "materials": MATERIALS, "objects": objects}


def _light() -> dict:
    return {"type": "sphere", "center": [0.0, 4.5, 0.5], "radius": 0.65, "material": "light"}


def _terrain(subdivisions: int) -> dict:
    return _scene([{"type": "mesh", "path": f"../../assets/benchmarks/terrain_grid_{subdivisions}.gltf",
                    "material": "surface"}, _light()])


def _spheres(count: int, material: str = "surface") -> list:
    """``count`` spheres on a square lattice over a 7.2 x 7.2 footprint, every fifth one metal."""
    cols = math.ceil(math.sqrt(count))
    rows = math.ceil(count / cols)
    sx, sz = 7.2 / max(cols - 1, 1), 7.2 / max(rows - 1, 1)
    radius = min(sx, sz) * 0.34
    out = []
    for i in range(count):
        x, z = -3.6 + (i % cols) * sx, -3.6 + (i // cols) * sz
        y = radius + 0.08 * math.sin(i * 0.73)
        out.append({"type": "sphere", "center": [round(x, 7), round(y, 7), round(z, 7)], "radius": round(radius, 7),
                    "material": material if i % 5 else "accent"})
    return out


def _ground() -> list:
    return [{"type": "triangle", "vertices": [[-5.0, 0.0, -5.0], [-5.0, 0.0, 5.0], [5.0, 0.0, -5.0]], "material": "surface"},
            {"type": "triangle", "vertices": [[5.0, 0.0, -5.0], [-5.0, 0.0, 5.0], [5.0, 0.0, 5.0]], "material": "surface"}]


def _mixed() -> dict:
    objs = [{"type": "mesh", "path": "../../assets/benchmarks/terrain_grid_32.gltf", "material": "surface"}]
    for s in _spheres(128):
        s["center"][1] = round(float(s["center"][1]) + 0.22, 7)
        s["radius"] = round(float(s["radius"]) * 0.72, 7)
        objs.append(s)
    objs.append(_light())
    return _scene(objs)


def _environment_control() -> dict:
    sc = _scene([{"type": "sphere", "center": [-1.2, 0.7, 0.0], "radius": 0.7, "material": "accent"},
                 {"type": "sphere", "center": [0.0, 0.7, -0.2], "radius": 0.7, "material": "surface"},
                 {"type": "sphere", "center": [1.2, 0.7, 0.0], "radius": 0.7, "material": "accent"},
                 {"type": "sphere", "center": [0.0, -1000.0, 0.0], "radius": 1000.0, "material": "surface"}])
    sc["camera"] = {"position": [0.0, 1.25, 5.5], "look_at": [0.0, 0.65, 0.0], "up": [0.0, 1.0, 0.0], "fov_degrees": 42.0}
    render = dict(RENDER)
    render["background"] = {"type": "environment", "path": "../../assets/environments/studio_test.hdr",
                            "intensity": 8.0, "rotation_degrees": 20.0}
    sc["render"] = render
    return sc


def _standin_hdr() -> bytes:
    """4 x 2 flat RGBE pixels: a warm bright top row, a dim blue bottom row."""
    top, bottom = bytes([200, 180, 150, 129]), bytes([40, 60, 120, 127])
    return b"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n-Y 2 +X 4\n" + top * 4 + bottom * 4


def write_suite(root) -> Path:
    """Writes scenes/benchmarks/*.json and assets/benchmarks/*.gltf (plus the environment
    stand-in) under ``root``; returns the scene directory."""
    root = Path(root)
    for n in (8, 32, 64):
        _dump(root / "assets" / "benchmarks" / f"terrain_grid_{n}.gltf", terrain_gltf(n))
    env = root / "assets" / "environments" / "studio_test.hdr"
    env.parent.mkdir(parents=True, exist_ok=True)
    env.write_bytes(_standin_hdr())
    scenes = dict(zip(SCENES, [_terrain(8), _terrain(32), _terrain(64), _scene(_ground() + _spheres(64) + [_light()]),
                               _scene(_ground() + _spheres(512) + [_light()]), _mixed(), _environment_control()]))
    out = root / "scenes" / "benchmarks"
    for name, sc in scenes.items():
        _dump(out / name, sc)
    return out


def run(root, warmup: int = 2, measured: int = 5, device: int = 0) -> list:
    """The reference's benchmark protocol on every fixture: native load, upload, then warm-up and
    measured static frames at seed 0 through the frame loop. Reports the median dispatch wait
    (render call, host clock, synchronous), the median device kernel time, the median whole frame
    (dispatch + RGBA8 readback with the display conversion on the device) and Mpaths/s."""
    from .frames import GpuBenchmarkConfig, StaticSceneEvaluator, benchmark_gpu_evaluator
    from .renderer import GpuRenderer
    from .scene import load_scene_gpu

    scene_dir = write_suite(root)
    rows = []
    with GpuRenderer(device) as r:
        for name in SCENES:
            t0 = time.perf_counter()
            data, exposure = load_scene_gpu(scene_dir / name)
            load_ms = (time.perf_counter() - t0) * 1e3
            res = benchmark_gpu_evaluator(StaticSceneEvaluator(data, exposure), GpuBenchmarkConfig(warmup, measured),
                                          renderer=r)
            paths = 320 * 180 * 4
            dispatch = statistics.median(f.dispatch_wait for f in res.frames) * 1e3
            kernel = statistics.median(f.kernel_ms for f in res.frames)
            total = statistics.median(f.total for f in res.frames) * 1e3
            ref_dispatch, ref_total = PUBLISHED_2080TI[name]
            rows.append({"scene": name, "load_ms": load_ms, "dispatch_ms": dispatch, "kernel_ms": kernel,
                         "total_ms": total, "mpaths_per_s_dispatch": paths / dispatch / 1e3,
                         "mpaths_per_s_kernel": paths / kernel / 1e3,
                         "published_2080ti_dispatch_ms": ref_dispatch, "published_2080ti_total_ms": ref_total,
                         "dispatch_speedup_vs_published": ref_dispatch / dispatch,
                         "total_speedup_vs_published": ref_total / total})
    return rows


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--out", type=Path, required=True, help="directory for the regenerated suite")
    ap.add_argument("--write-only", action="store_true")
    a = ap.parse_args()
    if a.write_only:
        print(write_suite(a.out))
        return
    for row in run(a.out):
        print(json.dumps(row))


if __name__ == "__main__":
    main()
