"""The native scene-file loader (tc_scene_load) against the Python loader and known answers (CPU).

Both loaders restate toaster's ``load_scene`` + ``scene_to_gpu`` (crates/toaster-scene/src/loader.rs:534-971,
crates/toaster-assets/src/gltf_loader.rs:11-233, crates/toaster-gpu/src/scene_upload.rs:54-294): every packed record
must be byte-identical between them. The fixtures are written here (PNG with every filter type, Adam7 interlacing,
palettes and transparency keys; flat, run-length and new run-length Radiance files; glTF with external and embedded
buffers, GLB, node hierarchies, sparse accessors and normalised texture coordinates), so the pixel, texel and vertex
values they hold are known answers. The reference's own scene files, when present next to this repository's
checkout, add the reference tests' golden values.
"""

import base64
import json
import math
import os
import struct
import zlib
from pathlib import Path

import numpy as np
import pytest
from conftest import reference_checkout

from toaster_b200 import gpu_types as gt
from toaster_b200.native import TcError
from toaster_b200.scene import load_scene, load_scene_gpu, scene_to_gpu

FIELDS = ["params", "camera", "spheres", "triangles", "triangle_attributes", "materials", "lights",
          "environment_pixels", "texture_pixels"]
REFERENCE_SCENES = reference_checkout() / "scenes"


def both(path):
    """(native records, exposure), (python records, exposure)."""
    native, exposure = load_scene_gpu(path)
    scene = load_scene(path)
    return (native, exposure), (scene_to_gpu(scene), scene.exposure_stops)


def assert_identical(path):
    (n, ne), (p, pe) = both(path)
    for f in FIELDS:
        a, b = getattr(n, f), getattr(p, f)
        if a is None or b is None:
            assert (a is None or a.size == 0) and (b is None or b.size == 0), f
            continue
        assert a.tobytes() == b.tobytes(), f"{path.name}: {f} differs"
    assert np.float32(ne) == np.float32(pe)
    return n


def assert_both_reject(path, match=None):
    with pytest.raises(TcError) as e:
        load_scene_gpu(path)
    if match:
        assert match in str(e.value), str(e.value)
    with pytest.raises((ValueError, KeyError, TypeError, OSError, zlib.error)):
        scene_to_gpu(load_scene(path))


# ------------------------------------------------------------------------------------- PNG writer
def _filter_row(kind, raw, prev, bpp):
    out = bytearray(len(raw))
    for i, x in enumerate(raw):
        left = raw[i - bpp] if i >= bpp else 0
        up = prev[i]
        ul = prev[i - bpp] if i >= bpp else 0
        if kind == 0:
            pred = 0
        elif kind == 1:
            pred = left
        elif kind == 2:
            pred = up
        elif kind == 3:
            pred = (left + up) >> 1
        else:
            p = left + up - ul
            pa, pb, pc = abs(p - left), abs(p - up), abs(p - ul)
            pred = left if pa <= pb and pa <= pc else (up if pb <= pc else ul)
        out[i] = (x - pred) & 0xFF
    return bytes([kind]) + bytes(out)


def _pack_row(samples, depth):
    if depth == 8:
        return bytes(int(v) for v in samples)
    out, acc, bits = bytearray(), 0, 0
    for v in samples:
        acc = (acc << depth) | int(v)
        bits += depth
        if bits == 8:
            out.append(acc)
            acc, bits = 0, 0
    if bits:
        out.append(acc << (8 - bits))
    return bytes(out)


def png_bytes(samples, color, depth=8, palette=None, trns=None, interlace=False):
    """samples: (h, w, channels) sample values (palette indices for colour type 3). Rows use
    filter types 0..4 in turn, so decoding exercises every reconstruction rule."""
    h, w, ch = samples.shape
    bpp = max(1, ch * depth // 8)
    passes = [(0, 0, 1, 1)] if not interlace else [(0, 0, 8, 8), (4, 0, 8, 8), (0, 4, 4, 8), (2, 0, 4, 4),
                                                   (0, 2, 2, 4), (1, 0, 2, 2), (0, 1, 1, 2)]
    raw, k = bytearray(), 0
    for x0, y0, dx, dy in passes:
        sub = samples[y0::dy, x0::dx]
        if sub.size == 0:
            continue
        rb = (sub.shape[1] * ch * depth + 7) // 8
        prev = bytes(rb)
        for row in sub:
            r = _pack_row(row.reshape(-1), depth)
            raw += _filter_row(k % 5, r, prev, bpp)
            prev = r
            k += 1

    def chunk(kind, body):
        return struct.pack(">I", len(body)) + kind + body + struct.pack(">I", zlib.crc32(kind + body))

    out = b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, depth, color, 0, 0, int(interlace)))
    if palette is not None:
        out += chunk(b"PLTE", bytes(np.asarray(palette, np.uint8).reshape(-1)))
    if trns is not None:
        out += chunk(b"tRNS", bytes(trns))
    return out + chunk(b"IDAT", zlib.compress(bytes(raw))) + chunk(b"IEND", b"")


# ------------------------------------------------------------------------------- Radiance writer
def _rle_channel(values):
    out, i, n = bytearray(), 0, len(values)
    while i < n:
        run = 1
        while i + run < n and run < 127 and values[i + run] == values[i]:
            run += 1
        if run >= 3:
            out += bytes([128 + run, values[i]])
            i += run
            continue
        j = i
        while j < n and j - i < 128 and not (j + 2 < n and values[j] == values[j + 1] == values[j + 2]):
            j += 1
        out += bytes([j - i]) + bytes(values[i:j])
        i = j
    return bytes(out)


def hdr_bytes(rgbe, mode="rle"):
    """rgbe: (h, w, 4) uint8. mode "rle" (new run-length scanlines), "flat", or "old" (flat with
    (1, 1, 1, k) repeats wherever a pixel equals its predecessor)."""
    h, w, _ = rgbe.shape
    out = bytearray(b"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\nEXPOSURE=1.0\n\n" + f"-Y {h} +X {w}\n".encode())
    for y in range(h):
        row = rgbe[y]
        if mode == "rle":
            out += bytes([2, 2, w >> 8, w & 0xFF])
            for c in range(4):
                out += _rle_channel(list(int(v) for v in row[:, c]))
        elif mode == "flat":
            out += row.tobytes()
        else:
            x = 0
            while x < w:
                if x > 0 and np.array_equal(row[x], row[x - 1]):
                    run = 1
                    while x + run < w and run < 255 and np.array_equal(row[x + run], row[x - 1]):
                        run += 1
                    out += bytes([1, 1, 1, run])
                    x += run
                else:
                    out += row[x].tobytes()
                    x += 1
    return bytes(out)


def rgbe_expected(rgbe):
    e = rgbe[..., 3].astype(np.int64)
    scale = np.where(e > 0, np.ldexp(1.0, e - 136), 0.0)
    return (rgbe[..., :3] * scale[..., None]).astype(np.float32)


# ----------------------------------------------------------------------------------- glTF writer
class Gltf:
    def __init__(self):
        self.doc = {"asset": {"version": "2.0"}, "buffers": [], "bufferViews": [], "accessors": [], "meshes": [],
                    "nodes": [], "scenes": []}
        self.blob = bytearray()

    def view(self, data: bytes, stride=None):
        while len(self.blob) % 4:
            self.blob.append(0)
        v = {"buffer": 0, "byteOffset": len(self.blob), "byteLength": len(data)}
        if stride:
            v["byteStride"] = stride
        self.blob += data
        self.doc["bufferViews"].append(v)
        return len(self.doc["bufferViews"]) - 1

    def accessor(self, arr, ctype, shape, normalized=False, sparse=None, stride=None):
        arr = np.ascontiguousarray(arr)
        count = arr.shape[0]
        data = arr.tobytes()
        if stride:  # interleave with padding bytes
            elem = arr.itemsize * (arr.shape[1] if arr.ndim > 1 else 1)
            data = b"".join(arr[i].tobytes() + bytes(stride - elem) for i in range(count))
        a = {"bufferView": self.view(data, stride), "componentType": ctype, "count": count, "type": shape}
        if normalized:
            a["normalized"] = True
        if sparse is not None:
            idx, vals = sparse
            a["sparse"] = {"count": len(idx),
                           "indices": {"bufferView": self.view(np.asarray(idx, np.uint16).tobytes()), "componentType": 5123},
                           "values": {"bufferView": self.view(np.ascontiguousarray(vals).tobytes())}}
        self.doc["accessors"].append(a)
        return len(self.doc["accessors"]) - 1

    def write(self, path: Path, external=False):
        if external:
            (path.parent / (path.stem + ".bin")).write_bytes(bytes(self.blob))
            self.doc["buffers"] = [{"uri": path.stem + ".bin", "byteLength": len(self.blob)}]
        else:
            uri = "data:application/octet-stream;base64," + base64.b64encode(bytes(self.blob)).decode()
            self.doc["buffers"] = [{"uri": uri, "byteLength": len(self.blob)}]
        path.write_text(json.dumps(self.doc))

    def write_glb(self, path: Path):
        self.doc["buffers"] = [{"byteLength": len(self.blob)}]
        js = json.dumps(self.doc).encode()
        js += b" " * (-len(js) % 4)
        binary = bytes(self.blob) + bytes(-len(self.blob) % 4)
        total = 12 + 8 + len(js) + 8 + len(binary)
        path.write_bytes(b"glTF" + struct.pack("<II", 2, total) + struct.pack("<I", len(js)) + b"JSON" + js +
                         struct.pack("<I", len(binary)) + b"BIN\0" + binary)


def quad(z=0.0):
    pos = np.array([[-1, -1, z], [1, -1, z], [1, 1, z], [-1, 1, z]], np.float32)
    return pos, np.array([0, 1, 2, 0, 2, 3], np.uint16)


def scene_doc(objects, materials=None, background="sky", **extra):
    doc = {"camera": {"position": [0.3, 1.2, 4.0], "look_at": [0.0, 0.2, 0.0], "fov_degrees": 40.0},
           "render": {"width": 64, "height": 36, "samples": 4, "max_bounces": 5, "background": background},
           "materials": materials if materials is not None else [
               {"name": "white", "type": "diffuse", "albedo": [0.7, 0.7, 0.7]},
               {"name": "light", "type": "emissive", "color": [1.0, 0.9, 0.8], "strength": 12.5}],
           "objects": objects}
    doc.update(extra)
    return doc


def write_scene(tmp_path, doc, name="scene.json"):
    p = tmp_path / name
    p.write_text(json.dumps(doc))
    return p


# ------------------------------------------------------------------------------- identical packing
def test_primitives_materials_and_display(tmp_path):
    mats = [{"name": "matte", "type": "diffuse", "albedo": [0.2, 0.3, 0.4]},
            {"name": "rough", "type": "metal", "albedo": [0.8, 0.8, 0.8], "roughness": 2.0},
            {"name": "glass", "type": "dielectric", "ior": 1.5},
            {"name": "lamp", "type": "emissive", "color": [1, 0.8, 0.6], "strength": 5},
            {"name": "dark", "type": "emissive", "color": [0, 0, 0], "strength": 5}]
    objs = [{"type": "sphere", "center": [0, -100.5, 0], "radius": 100, "material": "matte"},
            {"type": "sphere", "center": [0.7, 0.2, 0], "radius": 0.3, "material": "glass", "id": "ball"},
            {"type": "sphere", "center": [0, 2, 0], "radius": 0.25, "material": "lamp", "group": "lights"},
            {"type": "box", "center": [-0.6, 0.1, 0.2], "size": [0.4, 0.8, 0.3], "material": "rough"},
            {"type": "triangle", "vertices": [[-1, 1.9, -1], [1, 1.9, -1], [0, 1.9, 1]], "material": "lamp"},
            {"type": "triangle", "vertices": [[-1, 1.8, -1], [1, 1.8, -1], [0, 1.8, 1]], "material": "dark"}]
    doc = scene_doc(objs, mats, background="black", display={"exposure_stops": -2.0})
    doc["camera"]["vertical_fov_degrees"] = doc["camera"].pop("fov_degrees")
    doc["render"]["samples_per_pixel"] = doc["render"].pop("samples")
    doc["animation"] = {"tracks": [{"type": "translation", "target": {"type": "group", "name": "lights"}}]}
    n = assert_identical(write_scene(tmp_path, doc))
    p = n.params[0]
    assert (p["sphere_count"], p["triangle_count"], p["material_count"]) == (3, 14, 5)
    assert p["background_kind"] == gt.BLACK and p["samples"] == 4
    assert n.materials[1]["params"][0] == 1.0  # roughness clamped (loader.rs tests, accepts_all_material_types)
    assert n.materials[2]["kind"] == gt.DIELECTRIC and n.materials[2]["params"][1] == np.float32(1.5)
    assert tuple(n.materials[2]["albedo"]) == (1, 1, 1, 1)
    # Lights: the emissive triangle first, then the sphere; the zero-weight triangle is left out.
    assert list(n.lights["kind"]) == [0, 1] and p["light_count"] == 2
    assert n.lights["area_weight_cumulative"][1][2] == p["total_light_weight"]
    assert load_scene_gpu(write_scene(tmp_path, doc))[1] == -2.0


def _texture_variants():
    rng = np.random.default_rng(5)
    rgba = rng.integers(0, 256, (5, 7, 4), dtype=np.uint8)
    rgb = rng.integers(0, 256, (3, 6, 3), dtype=np.uint8)
    grey4 = rng.integers(0, 16, (4, 9, 1), dtype=np.uint8)
    grey_key = np.array([[[0], [77]], [[77], [200]]], np.uint8)
    pal_idx = rng.integers(0, 3, (6, 5, 1), dtype=np.uint8)
    palette = [(255, 0, 0), (0, 255, 0), (10, 20, 30)]
    rgb_key = np.array([[[1, 2, 3], [4, 5, 6]]], np.uint8)
    out = [
        ("rgba_interlaced", png_bytes(rgba, 6, interlace=True), rgba),
        ("rgb", png_bytes(rgb, 2), np.concatenate([rgb, np.full(rgb.shape[:2] + (1,), 255, np.uint8)], 2)),
        ("grey4", png_bytes(grey4, 0, depth=4), np.repeat(grey4 * 17, 3, 2)),
        ("grey_key", png_bytes(grey_key, 0, trns=[0, 77]), None),
        ("palette_trns", png_bytes(pal_idx, 3, depth=2, palette=palette, trns=[128, 255]), None),
        ("rgb_key", png_bytes(rgb_key, 2, trns=[0, 4, 0, 5, 0, 6]), None),
    ]
    expect = []
    for name, data, px in out:
        if name == "grey_key":
            g = grey_key[..., 0]
            px = np.stack([g, g, g, np.where(g == 77, 0, 255)], -1).astype(np.uint8)
        elif name == "palette_trns":
            pal = np.array(palette, np.uint8)[pal_idx[..., 0]]
            alpha = np.array([128, 255, 255], np.uint8)[pal_idx[..., 0]]
            px = np.concatenate([pal, alpha[..., None]], -1)
        elif name == "rgb_key":
            px = np.array([[[1, 2, 3, 255], [4, 5, 6, 0]]], np.uint8)
        elif px.shape[-1] == 3:
            px = np.concatenate([px, np.full(px.shape[:2] + (1,), 255, np.uint8)], -1)
        expect.append((name, data, px))
    return expect


def test_gltf_textures_hierarchy_sparse_and_normalised_uvs(tmp_path):
    """Every PNG variant becomes one textured material; the atlas holds each texture's RGBA8 texels
    in little-endian words, in texture order."""
    variants = _texture_variants()
    g = Gltf()
    g.doc["images"], g.doc["textures"], g.doc["materials"] = [], [], []
    pos, idx = quad()
    for i, (name, data, _) in enumerate(variants):
        if i % 2:
            (tmp_path / f"{name}.png").write_bytes(data)
            g.doc["images"].append({"uri": f"{name}.png"})
        else:
            g.doc["images"].append({"uri": "data:image/png;base64," + base64.b64encode(data).decode()})
        g.doc["textures"].append({"source": i})
        g.doc["materials"].append({"pbrMetallicRoughness": {"baseColorFactor": [0.5, 0.25 + 0.1 * i, 1.0, 1.0],
                                                            "baseColorTexture": {"index": i}}})
    # Vertices: positions with a sparse override of vertex 2, normals, u8 normalised UVs (strided).
    uv8 = np.array([[0, 255], [255, 255], [255, 0], [0, 128]], np.uint8)
    a_pos = g.accessor(pos, 5126, "VEC3", sparse=([2], np.array([[1.5, 1.25, 0.0]], np.float32)))
    a_nrm = g.accessor(np.tile(np.array([[0, 0, 1]], np.float32), (4, 1)), 5126, "VEC3")
    a_uv = g.accessor(uv8, 5121, "VEC2", normalized=True, stride=4)
    a_idx = g.accessor(idx, 5123, "SCALAR")
    prims = [{"attributes": {"POSITION": a_pos, "NORMAL": a_nrm, "TEXCOORD_0": a_uv}, "indices": a_idx, "material": m}
             for m in range(len(variants))]
    a_tri = g.accessor(pos[:3], 5126, "VEC3")
    prims.append({"attributes": {"POSITION": a_tri}})  # no material, no indices: default material, 1 triangle
    g.doc["meshes"] = [{"primitives": prims[:3]}, {"primitives": prims[3:]}]
    s = math.sin(math.radians(15)), math.cos(math.radians(15))  # quaternion of a 30-degree turn about y
    g.doc["nodes"] = [
        {"translation": [0.0, 0.5, -1.0], "rotation": [0.0, s[0], 0.0, s[1]], "scale": [0.5, 0.5, 0.5],
         "children": [1], "mesh": 0},
        {"matrix": [1, 0, 0, 0, 0, 0, 1, 0, 0, -1, 0, 0, 0.25, 0.0, 0.5, 1], "mesh": 1},
    ]
    g.doc["scenes"] = [{"nodes": [0]}]
    g.doc["scene"] = 0
    g.write(tmp_path / "mesh.gltf", external=True)
    doc = scene_doc([{"type": "mesh", "path": "mesh.gltf", "group": "m"},
                     {"type": "triangle", "vertices": [[-1, 2, -1], [1, 2, -1], [0, 2, 1]], "material": "light"}])
    n = assert_identical(write_scene(tmp_path, doc))
    # 6 textured quads (12 triangles), the default-material triangle, the light triangle.
    assert n.params[0]["triangle_count"] == 14
    assert n.params[0]["material_count"] == 2 + len(variants) + 1
    offset = 0
    for i, (name, _, px) in enumerate(variants):
        m = n.materials[2 + i]
        h, w = px.shape[:2]
        assert (m["texture_offset"], m["texture_width"], m["texture_height"]) == (offset, w, h), name
        words = n.texture_pixels[offset:offset + w * h]
        assert np.array_equal(words.view(np.uint8).reshape(h, w, 4), px), name
        assert np.allclose(m["albedo"][:3], [0.5, np.float32(0.25 + 0.1 * i), 1.0])
        offset += w * h
    assert len(n.texture_pixels) == offset
    # The default material (no glTF material) is white diffuse, after the imported ones.
    last = n.materials[2 + len(variants)]
    assert last["kind"] == gt.DIFFUSE and tuple(last["albedo"]) == (1, 1, 1, 1) and last["texture_width"] == 0
    attrs = n.triangle_attributes
    assert list(attrs["flags"][:12]) == [3] * 12 and attrs["flags"][12] == 0
    assert tuple(attrs["uv0"][0]) == (0.0, 1.0) and attrs["uv0"][1][1] == np.float32(1.0)
    assert attrs["uv2"][1][1] == np.float32(128) / np.float32(255)
    # Node 0: scale 0.5, 30 degrees about y, then translation; vertex 0 (-1, -1, 0).
    v0 = n.triangles["v0"][0][:3]
    c, sn = math.cos(math.radians(30)), math.sin(math.radians(30))
    assert np.allclose(v0, [-0.5 * c + 0.0, 0.5 - 0.5, -1.0 + 0.5 * sn], atol=1e-6)
    # Its normals are the rotated +z, unit length.
    assert np.allclose(attrs["n0"][0][:3], [sn, 0.0, c], atol=1e-6)


def test_glb_buffers_images_from_buffer_views_and_override_material(tmp_path):
    variants = _texture_variants()[:2]
    g = Gltf()
    pos, idx = quad(0.5)
    g.doc["images"] = [{"bufferView": g.view(variants[1][1]), "mimeType": "image/png"}]
    g.doc["textures"] = [{"source": 0}]
    g.doc["materials"] = [{"pbrMetallicRoughness": {"baseColorTexture": {"index": 0}}}]
    a_pos = g.accessor(pos, 5126, "VEC3")
    a_uv = g.accessor(np.array([[0, 0], [65535, 0], [65535, 65535], [0, 65535]], np.uint16), 5123, "VEC2",
                      normalized=True)
    a_idx = g.accessor(idx.astype(np.uint32), 5125, "SCALAR")
    g.doc["meshes"] = [{"primitives": [{"attributes": {"POSITION": a_pos, "TEXCOORD_0": a_uv}, "indices": a_idx,
                                        "material": 0}]}]
    g.doc["nodes"] = [{"mesh": 0}, {"mesh": 0, "translation": [0, 0, -2]}]
    g.doc["scenes"] = [{"nodes": [1]}, {"nodes": [0]}]  # no default scene: all scenes, in order
    g.write_glb(tmp_path / "quad.glb")
    imported = assert_identical(write_scene(tmp_path, scene_doc([{"type": "mesh", "path": "quad.glb"}])))
    assert imported.params[0]["triangle_count"] == 4
    assert imported.triangles["v0"][0][2] == np.float32(-1.5)  # scene 0 (node 1) first
    assert imported.materials[2]["texture_width"] == variants[1][2].shape[1]
    assert imported.triangle_attributes["uv1"][0][0] == np.float32(1.0)
    # With an override the glTF materials and textures are not imported.
    over = assert_identical(write_scene(tmp_path, scene_doc([{"type": "mesh", "path": "quad.glb",
                                                              "material": "white"}])))
    assert over.params[0]["material_count"] == 2 and over.texture_pixels is None
    assert set(over.triangles["material_index"]) == {0}


@pytest.mark.parametrize("mode", ["rle", "flat", "old"])
def test_radiance_environment_known_answer(tmp_path, mode):
    rng = np.random.default_rng(11)
    h, w = 16, 40
    rgbe = rng.integers(0, 256, (h, w, 4), dtype=np.uint8)
    rgbe[..., 3] = rng.integers(120, 140, (h, w))
    rgbe[2:5, 10:30] = rgbe[2, 10]  # long runs for the run-length forms
    rgbe[7, :, 3] = 0  # zero exponent: black
    (tmp_path / "sky.hdr").write_bytes(hdr_bytes(rgbe, mode))
    bg = {"type": "environment", "path": "sky.hdr", "intensity": 2.5, "rotation_degrees": -30.0}
    n = assert_identical(write_scene(tmp_path, scene_doc([{"type": "sphere", "center": [0, 0, 0], "radius": 1,
                                                           "material": "white"}], background=bg)))
    p = n.params[0]
    assert (p["environment_width"], p["environment_height"]) == (w, h)
    assert p["environment_intensity"] == np.float32(2.5) and p["environment_rotation_degrees"] == np.float32(330.0)
    env = n.environment_pixels.reshape(h, w, 4)
    assert np.array_equal(env[..., :3], rgbe_expected(rgbe))
    cdf = env[..., 3].reshape(-1)
    assert cdf[-1] == 1.0 and np.all(np.diff(cdf) >= 0)


def test_png_environment_is_srgb_decoded(tmp_path):
    grey = np.arange(24, dtype=np.uint8).reshape(4, 6, 1) * 10
    (tmp_path / "env.png").write_bytes(png_bytes(grey, 0))
    bg = {"type": "environment", "path": "env.png"}
    n = assert_identical(write_scene(tmp_path, scene_doc([{"type": "sphere", "center": [0, 0, 0], "radius": 1,
                                                           "material": "white"}], background=bg)))
    x = grey[..., 0].astype(np.float64) / 255.0
    lin = np.where(x <= 0.04045, x / 12.92, ((x + 0.055) / 1.055) ** 2.4)
    assert np.allclose(n.environment_pixels[:, 0].reshape(4, 6), lin, rtol=1e-6, atol=1e-7)


# ------------------------------------------------------------------------------------- rejections
BAD_MATERIALS = [  # loader.rs tests rejects_invalid_material_parameters, plus the other material rules
    {"name": "bad", "type": "diffuse", "albedo": [1.1, 0, 0]},
    {"name": "bad", "type": "dielectric", "ior": 0},
    {"name": "bad", "type": "metal", "albedo": [0.5, 0.5, 0.5]},
    {"name": "bad", "type": "emissive", "color": [1, 1, 1], "strength": -1},
    {"name": "bad", "type": "plastic", "albedo": [0.5, 0.5, 0.5]},
]


@pytest.mark.parametrize("material", BAD_MATERIALS, ids=["albedo", "ior", "roughness_missing", "strength", "type"])
def test_invalid_materials_are_rejected(tmp_path, material):
    doc = scene_doc([{"type": "sphere", "center": [0, 0, 0], "radius": 1, "material": "bad"}], [material])
    assert_both_reject(write_scene(tmp_path, doc))


def _sphere():
    return {"type": "sphere", "center": [0, 0, 0], "radius": 1, "material": "white"}


@pytest.mark.parametrize("case", [
    "unknown_material", "exposure_overflow", "duplicate_material", "collinear", "fov_180", "up_parallel",
    "display_field", "box_size", "radius", "duplicate_id", "empty", "triangle_physics", "physics_without_id",
])
def test_invalid_scenes_are_rejected(tmp_path, case):
    doc = scene_doc([_sphere()])
    if case == "unknown_material":  # loader.rs tests rejects_unknown_materials
        doc["objects"] = [{"type": "sphere", "center": [0, 0, 0], "radius": 1, "material": "missing"}]
    elif case == "exposure_overflow":  # rejects_invalid_display_settings
        text = json.dumps(doc)[:-1] + ', "display": {"exposure_stops": 1e400}}'
        p = tmp_path / "scene.json"
        p.write_text(text)
        return assert_both_reject(p)
    elif case == "duplicate_material":
        doc["materials"].append(dict(doc["materials"][0]))
    elif case == "collinear":
        doc["objects"].append({"type": "triangle", "vertices": [[0, 0, 0], [1, 1, 1], [2, 2, 2]], "material": "white"})
    elif case == "fov_180":
        doc["camera"]["fov_degrees"] = 180
    elif case == "up_parallel":
        doc["camera"]["up"] = [0.6, 2.4, 8.0]
        doc["camera"]["look_at"] = [0, 0, 0]
    elif case == "display_field":
        doc["display"] = {"gamma": 2.2}
    elif case == "box_size":
        doc["objects"].append({"type": "box", "center": [0, 0, 0], "size": [1, 0, 1], "material": "white"})
    elif case == "radius":
        doc["objects"][0]["radius"] = -1
    elif case == "duplicate_id":
        doc["objects"] = [dict(_sphere(), id="a"), dict(_sphere(), id="a")]
    elif case == "empty":  # loads, but the GPU packing needs an object
        doc["objects"] = []
    elif case == "triangle_physics":
        doc["objects"].append({"type": "triangle", "vertices": [[0, 0, 0], [1, 0, 0], [0, 1, 0]], "material": "white",
                               "physics": {"type": "dynamic"}})
    elif case == "physics_without_id":
        doc["objects"][0]["physics"] = {"type": "dynamic"}
    assert_both_reject(write_scene(tmp_path, doc))


@pytest.mark.parametrize("case", ["mode", "index", "no_uv_texture", "crc", "png16", "jpeg", "missing_file",
                                  "no_triangles"])
def test_invalid_meshes_are_rejected(tmp_path, case):
    g = Gltf()
    pos, idx = quad()
    a_pos = g.accessor(pos, 5126, "VEC3")
    prim = {"attributes": {"POSITION": a_pos}, "indices": g.accessor(idx, 5123, "SCALAR")}
    if case == "mode":
        prim["mode"] = 1
    elif case == "index":
        prim["indices"] = g.accessor(np.array([0, 1, 9], np.uint16), 5123, "SCALAR")
    elif case in ("no_uv_texture", "crc", "png16", "jpeg"):
        data = png_bytes(np.zeros((2, 2, 4), np.uint8), 6)
        if case == "crc":
            data = data[:-20] + bytes([data[-20] ^ 1]) + data[-19:]
        elif case == "png16":
            data = png_bytes(np.zeros((2, 2, 3), np.uint8), 2)
            data = data[:24] + bytes([16]) + data[25:]  # bit depth byte of IHDR
            body = data[12:29]
            data = data[:29] + struct.pack(">I", zlib.crc32(body)) + data[33:]
        elif case == "jpeg":
            data = b"\xff\xd8\xff\xe0" + bytes(32)
        g.doc["images"] = [{"uri": "data:image/png;base64," + base64.b64encode(data).decode()}]
        g.doc["textures"] = [{"source": 0}]
        g.doc["materials"] = [{"pbrMetallicRoughness": {"baseColorTexture": {"index": 0}}}]
        prim["material"] = 0
    g.doc["meshes"] = [{"primitives": [prim]}]
    g.doc["nodes"] = [{"mesh": 0}] if case != "no_triangles" else [{}]
    g.doc["scenes"] = [{"nodes": [0]}]
    g.write(tmp_path / "m.gltf")
    path = "m.gltf" if case != "missing_file" else "absent.gltf"
    assert_both_reject(write_scene(tmp_path, scene_doc([{"type": "mesh", "path": path}])),
                       "JPEG" if case == "jpeg" else None)


def test_error_message_names_the_field(tmp_path):
    doc = scene_doc([_sphere()])
    del doc["render"]["max_bounces"]
    with pytest.raises(TcError, match="max_bounces"):
        load_scene_gpu(write_scene(tmp_path, doc))
    p = tmp_path / "broken.json"
    p.write_text('{"camera": {"position": [0, 0, 1],, }')
    with pytest.raises(TcError, match="line 1 column"):
        load_scene_gpu(p)


# ------------------------------------------------------------------ the reference's own scene files
def _reference_files():
    if not REFERENCE_SCENES.is_dir():
        return []
    return sorted(REFERENCE_SCENES.glob("*.json")) + sorted(REFERENCE_SCENES.glob("benchmarks/*.json"))


@pytest.mark.skipif(not REFERENCE_SCENES.is_dir(), reason="the reference's scene files are not present")
def test_reference_scene_files_pack_identically():
    loaded = 0
    for path in _reference_files():
        text = path.read_text()
        if json.loads(text) == {}:  # placeholder files: both loaders reject them
            assert_both_reject(path, "camera")
            continue
        assert_identical(path)
        loaded += 1
    assert loaded >= 20


@pytest.mark.skipif(not REFERENCE_SCENES.is_dir(), reason="the reference's scene files are not present")
def test_reference_known_answers():
    s = REFERENCE_SCENES
    # scene_upload.rs:511-551 loads_materials_scene_into_gpu_layout
    n, _ = load_scene_gpu(s / "002_materials.json")
    assert tuple(n.camera["origin"][0]) == (0.0, np.float32(1.4), 6.0, 0.0)
    assert tuple(n.spheres["center_radius"][3]) == (np.float32(1.2), 0.5, 0.0, 0.5)
    assert n.materials[2]["kind"] == 2 and n.materials[2]["params"][1] == np.float32(1.5)
    assert n.materials[3]["kind"] == 1 and n.materials[3]["params"][0] == np.float32(0.08)
    assert n.materials[4]["kind"] == 3 and n.materials[4]["params"][2] == 6.0
    assert len(n.lights) == 1 and n.lights[0]["kind"] == 1 and n.lights[0]["material_index"] == 4
    # :553-575 loads_cornell_box_triangles_into_gpu_layout
    n, _ = load_scene_gpu(s / "003_cornell_box.json")
    assert len(n.triangles) == 12
    assert tuple(n.triangles["v0"][0]) == (-2.0, 0.0, 0.0, 0.0) and tuple(n.triangles["v1"][0]) == (2.0, 0.0, -4.0, 0.0)
    assert [n.triangles["material_index"][i] for i in (0, 6, 8, 10)] == [0, 1, 2, 3]
    assert len(n.lights) == 2 and set(n.lights["kind"]) == {0}
    # :577-622 loads_mesh_room_into_gpu_layout
    n, _ = load_scene_gpu(s / "004_mesh.json")
    p = n.params[0]
    assert (p["sphere_count"], p["triangle_count"], p["material_count"]) == (0, 24, 6)
    assert [n.materials[i]["kind"] for i in (3, 4, 5)] == [0, 1, 3] and len(n.lights) == 2
    # :624-636 and gltf_loader.rs:240-256 (tetrahedron vertices after the node transform)
    n, _ = load_scene_gpu(s / "008_gltf_tetrahedron.json")
    assert (n.params[0]["sphere_count"], n.params[0]["triangle_count"], n.params[0]["light_count"]) == (1, 6, 1)
    assert n.triangles["material_index"][2] == 1
    assert tuple(n.triangles["v0"][2]) == (0.0, 0.75, -2.0, 0.0)
    assert tuple(n.triangles["v1"][2][:3]) == (-0.75, -0.75, -1.25)
    # :638-656 uploads_textured_gltf_material_and_triangle_attributes, loader.rs:1846-1872
    n, _ = load_scene_gpu(s / "009_gltf_textured_quad.json")
    a = n.triangle_attributes
    assert n.params[0]["triangle_count"] == 4 and len(a) == 4 and a["flags"][0] == 3
    assert tuple(a["n0"][0]) == (0.0, 0.0, 1.0, 0.0) and tuple(a["uv0"][0]) == (0.0, 1.0)
    m = n.materials[1]
    assert (m["texture_offset"], m["texture_width"], m["texture_height"]) == (0, 2, 2)
    assert tuple(m["albedo"][:3]) == (np.float32(0.8), 1.0, np.float32(0.6))
    assert len(n.texture_pixels) == 4 and n.texture_pixels[0] == 0xFF0000FF and n.params[0]["light_count"] == 2
    assert set(n.triangles["material_index"][:2]) == {1}
    # :699-716 uploads_float_environment_map_and_metadata, loader.rs:1874-1889
    n, _ = load_scene_gpu(s / "010_environment_map.json")
    p = n.params[0]
    assert p["background_kind"] == 2 and (p["environment_width"], p["environment_height"]) == (4, 2)
    assert p["environment_intensity"] == 8.0 and p["environment_rotation_degrees"] == 20.0
    assert len(n.environment_pixels) == 8 and abs(n.environment_pixels[-1, 3] - 1.0) < 1e-6
    assert np.any(n.environment_pixels[:, :3] > 0)
    # loader.rs:1891-1916 loads_generated_benchmark_suite_with_expected_geometry_counts
    for name, tris, spheres, env in [("001_triangles_128.json", 128, 1, False), ("002_triangles_2048.json", 2048, 1, False),
                                     ("003_triangles_8192.json", 8192, 1, False), ("004_spheres_64.json", 2, 65, False),
                                     ("005_spheres_512.json", 2, 513, False),
                                     ("006_mixed_2048t_128s.json", 2048, 129, False),
                                     ("007_environment_control.json", 0, 4, True)]:
        n, _ = load_scene_gpu(s / "benchmarks" / name)
        p = n.params[0]
        assert (p["triangle_count"], p["sphere_count"], p["background_kind"] == 2) == (tris, spheres, env), name
        assert (p["width"], p["height"], p["samples"], p["max_bounces"]) == (320, 180, 4, 4), name


def test_c_abi_arguments_and_error_truncation(tmp_path):
    import ctypes

    from toaster_b200 import native

    lib = native.load_library()
    out = ctypes.c_void_p()
    err = ctypes.create_string_buffer(16)
    assert lib.tc_scene_load(None, ctypes.byref(out), err, len(err)) == native.TC_ERR_INVALID
    assert lib.tc_scene_load(b"x.json", None, err, len(err)) == native.TC_ERR_INVALID
    missing = str(tmp_path / "absent.json").encode()
    assert lib.tc_scene_load(missing, ctypes.byref(out), err, len(err)) == native.TC_ERR_INVALID
    assert not out.value and len(err.value) == 15 and err.value.startswith(b"failed to open")
    assert lib.tc_scene_load(missing, ctypes.byref(out), None, 0) == native.TC_ERR_INVALID
    assert lib.tc_loaded_scene_data(None) is None or not lib.tc_loaded_scene_data(None)
    exposure = ctypes.c_float()
    assert lib.tc_loaded_scene_display(None, ctypes.byref(exposure)) == native.TC_ERR_INVALID
    assert lib.tc_loaded_scene_free(None) == native.TC_OK


def test_mutated_files_are_loaded_or_rejected(tmp_path):
    """Seeded byte mutations of every input kind (scene JSON, glTF JSON, its buffer, GLB, PNG,
    Radiance): each load must return OK or TC_ERR_INVALID with a message, never crash."""
    import random

    rng = random.Random(2024)
    g = Gltf()
    pos, idx = quad()
    tex = png_bytes(np.arange(48, dtype=np.uint8).reshape(4, 3, 4) * 5, 6, interlace=True)
    g.doc["images"] = [{"uri": "t.png"}]
    g.doc["textures"] = [{"source": 0}]
    g.doc["materials"] = [{"pbrMetallicRoughness": {"baseColorTexture": {"index": 0}}}]
    a_pos = g.accessor(pos, 5126, "VEC3", sparse=([1], np.array([[0.5, -1, 0]], np.float32)))
    a_uv = g.accessor(np.array([[0, 0], [255, 0], [255, 255], [0, 255]], np.uint8), 5121, "VEC2", normalized=True,
                      stride=4)
    g.doc["meshes"] = [{"primitives": [{"attributes": {"POSITION": a_pos, "TEXCOORD_0": a_uv},
                                        "indices": g.accessor(idx, 5123, "SCALAR"), "material": 0}]}]
    g.doc["nodes"] = [{"mesh": 0, "rotation": [0, 0.2, 0, 0.98], "children": [1]}, {"mesh": 0, "translation": [1, 0, 0]}]
    g.doc["scenes"] = [{"nodes": [0]}]
    g.write(tmp_path / "m.gltf", external=True)
    g.write_glb(tmp_path / "m.glb")
    rgbe = np.random.default_rng(1).integers(0, 256, (6, 12, 4), dtype=np.uint8)
    rgbe[..., 3] = 130
    scene = scene_doc([{"type": "mesh", "path": "m.gltf"}, {"type": "mesh", "path": "m.glb", "material": "white"},
                       {"type": "sphere", "center": [0, 0, 0], "radius": 1, "material": "light"}],
                      background={"type": "environment", "path": "e.hdr", "intensity": 2})
    base = {"m.gltf": (tmp_path / "m.gltf").read_bytes(), "m.bin": (tmp_path / "m.bin").read_bytes(),
            "m.glb": (tmp_path / "m.glb").read_bytes(), "t.png": tex, "e.hdr": hdr_bytes(rgbe, "rle"),
            "scene.json": json.dumps(scene).encode()}

    def mutate(b):
        b = bytearray(b)
        for _ in range(rng.randint(1, 8)):
            i = rng.randrange(len(b))
            op = rng.random()
            if op < 0.4:
                b[i] = rng.randrange(256)
            elif op < 0.6:
                del b[i:i + rng.randint(1, 16)]
            elif op < 0.8:
                b[i:i] = bytes(rng.randrange(256) for _ in range(rng.randint(1, 8)))
            else:
                j = rng.randrange(len(b))
                b[i:i + 4] = b[j:j + 4]
        return bytes(b) or b"x"

    outcomes = {}
    for _ in range(300):
        files = dict(base)
        target = rng.choice(sorted(files))
        files[target] = mutate(files[target])
        for name, data in files.items():
            (tmp_path / name).write_bytes(data)
        try:
            load_scene_gpu(tmp_path / "scene.json")
            outcomes["ok"] = outcomes.get("ok", 0) + 1
        except TcError as e:
            assert e.code == -1 and len(str(e)) > 25
            outcomes["rejected"] = outcomes.get("rejected", 0) + 1
    assert outcomes.get("ok", 0) > 0 and outcomes.get("rejected", 0) > 0
