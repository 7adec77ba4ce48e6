"""Scene files through the native loader on the GPU (needs a B200).

A scene file with a textured, smooth-shaded glTF mesh is loaded by tc_scene_load and uploaded
straight from the library's buffers (GpuRenderer.upload_file); its image must agree with the
oracle's render of the same file loaded by the Python loader, within the statistical band of the
image parity tests. The file renderer's PNG holds exactly the device-converted RGBA8 bytes.
"""

import base64
import json

import numpy as np
import pytest

from test_gpu_parity import statistical_parity
from test_scene_loader import Gltf, png_bytes, scene_doc, write_scene
from toaster_b200.render_file import render_file
from toaster_b200.scene import _decode_png, load_scene
from toaster_b200.stream import encode_png

pytestmark = pytest.mark.gpu


def textured_scene(tmp_path):
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


def test_scene_file_image_matches_oracle(renderer, tmp_path):
    path = textured_scene(tmp_path)
    statistical_parity(renderer, load_scene(path), upload=lambda: renderer.upload_file(path))


def test_render_file_writes_the_device_converted_bytes(renderer, tmp_path):
    path = textured_scene(tmp_path)
    exposure = renderer.upload_file(path)
    assert exposure == 0.5
    renderer.render(samples=16, frame_index=3)
    rgba = renderer.readback_rgba8(exposure)
    w, h, ch, img = _decode_png(encode_png(rgba))
    assert (w, h, ch) == (48, 32, 4) and np.array_equal(img, rgba)
    out = render_file(path, tmp_path / "frame.png", spp=16)
    w, h, ch, img = _decode_png((tmp_path / "frame.png").read_bytes())
    assert (w, h) == (48, 32) and img[..., 3].min() == 255 and img[..., :3].max() > 0
    assert out["samples"] == 16
    jpg = render_file(path, tmp_path / "frame.jpg", spp=16)
    data = (tmp_path / "frame.jpg").read_bytes()
    assert data[:2] == b"\xff\xd8" and jpg["bytes"] == len(data)
