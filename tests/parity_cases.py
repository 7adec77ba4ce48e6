"""Scenes of the image-parity tests, shared by tests/test_gpu_parity.py and the oracle-against-itself
calibration (tests/calibrate_parity.py) that sets their thresholds.

Each case renders one scene on the GPU at ``gpu_spp`` and with the oracle at ``cpu_spp``; the
calibration replaces the GPU side by the oracle with an independent seed at ``gpu_spp``.
"""

from __future__ import annotations

import base64
import tempfile
from dataclasses import dataclass
from pathlib import Path
from typing import Callable

import numpy as np

from test_scene_loader import Gltf, png_bytes, scene_doc, write_scene
from toaster_b200 import configs, gpu_types as gt
from toaster_b200.scene import Material, Scene, load_scene


def sky_dielectric_metal() -> Scene:
    mats = [Material.dielectric(1.5), Material.metal((0.9, 0.6, 0.3), 0.3), Material.diffuse((0.6, 0.7, 0.8)),
            Material.emissive((1.0, 0.9, 0.8), 6.0)]
    return Scene(camera_position=(0, 1, 5), camera_look_at=(0, 0.3, 0), width=48, height=32, samples=64,
                 max_bounces=6, background=gt.SKY, materials=mats,
                 sphere_centers=np.array([(-0.8, 0.5, 0), (0.8, 0.5, 0), (0, -100, 0), (0, 3, 0)], np.float32),
                 sphere_radii=np.array([0.5, 0.5, 99.9, 0.4], np.float32),
                 sphere_materials=np.array([0, 1, 2, 3], np.uint32))


def plain_small() -> Scene:
    s = configs.plain_small()
    s.width, s.height = 80, 45
    return s


def window_room_sky() -> Scene:
    # The guiding workload's plain estimator with the sun left out and 1,024 clutter triangles.
    env = configs.sky_environment(width=256, height=128, sun_radiance=0.0)
    return configs.room_with_window(width=48, height=27, samples=64, clutter=1024, environment=env)


def window_room_sun() -> Scene:
    # The guiding workload itself: 8,192 clutter triangles (30% metal), the 1024x512 sky with its
    # 0.5-degree sun of radiance 1e4, 8 bounces; a 96x54 frame of the same view.
    return configs.room_with_window(width=96, height=54, samples=64)


def large_mesh() -> Scene:
    # The 1024 x 1024 fBm heightfield (2,093,058 triangles) with 512 glass and metal spheres and the
    # sky + sun, 8 bounces; a 96x54 frame of the same view.
    return configs.large_mesh(width=96, height=54, samples=64)


def textured_scene(tmp_path: Path) -> Path:
    """A scene file with a textured, smooth-shaded glTF floor (a checker PNG, per-vertex normals
    tilted towards the centre), a glass and a gold sphere and an emissive triangle under the sky."""
    g = Gltf()
    checker = np.zeros((4, 4, 3), np.uint8)
    checker[(np.add.outer(np.arange(4), np.arange(4)) % 2) == 0] = (230, 60, 40)
    checker[(np.add.outer(np.arange(4), np.arange(4)) % 2) == 1] = (40, 200, 90)
    g.doc["images"] = [{"uri": "data:image/png;base64," + base64.b64encode(png_bytes(checker, 2)).decode()}]
    g.doc["textures"] = [{"source": 0}]
    g.doc["materials"] = [{"pbrMetallicRoughness": {"baseColorFactor": [0.9, 0.9, 0.9, 1.0],
                                                    "baseColorTexture": {"index": 0}}}]
    # A gently curved floor: 8 x 8 quads with per-vertex normals tilted towards the centre.
    n = 9
    xs = np.linspace(-2, 2, n, dtype=np.float32)
    gx, gz = np.meshgrid(xs, xs)
    pos = np.stack([gx, 0.05 * (gx ** 2 + gz ** 2) - 0.5, gz], -1).reshape(-1, 3).astype(np.float32)
    nrm = np.stack([-0.1 * gx, np.ones_like(gx), -0.1 * gz], -1).reshape(-1, 3).astype(np.float32)
    uv = (np.stack([gx, gz], -1).reshape(-1, 2) * 0.5 + 0.5).astype(np.float32)
    idx = []
    for r in range(n - 1):
        for c in range(n - 1):
            a, b, d, e = r * n + c, r * n + c + 1, (r + 1) * n + c, (r + 1) * n + c + 1
            idx += [a, d, b, b, d, e]
    prim = {"attributes": {"POSITION": g.accessor(pos, 5126, "VEC3"), "NORMAL": g.accessor(nrm, 5126, "VEC3"),
                           "TEXCOORD_0": g.accessor(uv, 5126, "VEC2")},
            "indices": g.accessor(np.array(idx, np.uint16), 5123, "SCALAR"), "material": 0}
    g.doc["meshes"] = [{"primitives": [prim]}]
    g.doc["nodes"] = [{"mesh": 0}]
    g.doc["scenes"] = [{"nodes": [0]}]
    g.write(tmp_path / "floor.gltf")
    mats = [{"name": "glass", "type": "dielectric", "ior": 1.5},
            {"name": "gold", "type": "metal", "albedo": [0.9, 0.7, 0.3], "roughness": 0.2},
            {"name": "lamp", "type": "emissive", "color": [1.0, 0.95, 0.9], "strength": 8.0}]
    objs = [{"type": "mesh", "path": "floor.gltf"},
            {"type": "sphere", "center": [-0.6, 0.0, 0.2], "radius": 0.45, "material": "glass"},
            {"type": "sphere", "center": [0.7, -0.05, -0.3], "radius": 0.4, "material": "gold"},
            {"type": "triangle", "vertices": [[-1, 2.5, -1], [1, 2.5, -1], [0, 2.5, 1]], "material": "lamp"}]
    doc = scene_doc(objs, mats, background="sky", display={"exposure_stops": 0.5})
    doc["render"].update({"width": 48, "height": 32, "samples": 64, "max_bounces": 6})
    return write_scene(tmp_path, doc)



def textured_scene_file() -> Scene:
    return load_scene(textured_scene(Path(tempfile.mkdtemp())))


@dataclass(frozen=True)
class Case:
    name: str
    make: Callable[[], Scene]
    gpu_spp: int
    cpu_spp: int


CASES = [
    Case("plain_small", plain_small, 4096, 256),
    Case("mixed", lambda: configs.mixed(width=64, height=36, samples=64), 4096, 256),
    Case("sky_dielectric_metal", sky_dielectric_metal, 4096, 256),
    Case("window_room_sky", window_room_sky, 4096, 1024),
    Case("window_room_sun", window_room_sun, 4096, 1024),
    Case("large_mesh", large_mesh, 4096, 256),
    Case("textured_scene_file", textured_scene_file, 4096, 256),
]
BY_NAME = {c.name: c for c in CASES}
