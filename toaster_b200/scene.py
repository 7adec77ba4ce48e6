"""Renderer-neutral scene model, toaster JSON loading and packing into GPU records.

The model mirrors ``toaster_scene::Scene`` (crates/toaster-scene/src/scene.rs:19-90) with
geometry held as NumPy arrays so million-triangle scenes stay cheap. ``scene_to_gpu`` is the
equivalent of ``toaster_gpu::scene_upload::scene_to_gpu`` (scene_upload.rs:79-294): it packs the
scene into the ``#[repr(C)]`` records of gpu_types.rs that the CUDA library consumes.
"""

from __future__ import annotations

import base64
import dataclasses
import json
import math
import struct
import urllib.parse
import zlib
from pathlib import Path
from typing import Optional

import numpy as np

from . import gpu_types as gt

F32_EPSILON = np.float32(np.finfo(np.float32).eps)


@dataclasses.dataclass
class Material:
    """One runtime material (crates/toaster-scene/src/material.rs:7-39)."""

    kind: int  # gpu_types DIFFUSE / METAL / DIELECTRIC / EMISSIVE
    albedo: tuple = (1.0, 1.0, 1.0)  # diffuse/metal albedo, emissive colour
    roughness: float = 0.0
    ior: float = 1.5
    strength: float = 0.0
    name: str = ""
    texture: Optional[int] = None  # base-colour texture (index into Scene.textures) of a textured diffuse

    @staticmethod
    def diffuse(albedo, name=""):
        return Material(gt.DIFFUSE, tuple(float(a) for a in albedo), name=name)

    @staticmethod
    def metal(albedo, roughness, name=""):
        return Material(gt.METAL, tuple(float(a) for a in albedo), roughness=float(roughness), name=name)

    @staticmethod
    def dielectric(ior, name=""):
        return Material(gt.DIELECTRIC, (1.0, 1.0, 1.0), ior=float(ior), name=name)

    @staticmethod
    def emissive(color, strength, name=""):
        return Material(gt.EMISSIVE, tuple(float(c) for c in color), strength=float(strength), name=name)


@dataclasses.dataclass
class EnvironmentMap:
    """Lat-long linear-radiance map (crates/toaster-scene/src/environment.rs:9-24)."""

    width: int
    height: int
    pixels: np.ndarray  # (height, width, 3) float32, row-major, y down
    intensity: float = 1.0
    rotation_degrees: float = 0.0

    def __post_init__(self):
        self.pixels = np.ascontiguousarray(self.pixels, dtype=np.float32).reshape(self.height, self.width, 3)
        if self.width <= 0 or self.height <= 0:
            raise ValueError("environment dimensions must be nonzero")
        if not np.all(np.isfinite(self.pixels)) or np.any(self.pixels < 0):
            raise ValueError("environment pixels must be finite and non-negative")
        if not math.isfinite(self.intensity) or self.intensity < 0:
            raise ValueError("environment intensity must be finite and non-negative")
        if not math.isfinite(self.rotation_degrees):
            raise ValueError("environment rotation_degrees must be finite")

    def importance_cdf(self) -> np.ndarray:
        """Flat row-major CDF (environment.rs:245-278): f64 accumulation, f32 storage, last = 1."""
        h, w = self.height, self.width
        sin_theta = np.array([math.sin(math.pi * (y + 0.5) / h) for y in range(h)], np.float64)
        px = self.pixels.astype(np.float64)
        lum = 0.2126 * px[..., 0] + 0.7152 * px[..., 1] + 0.0722 * px[..., 2]
        weights = (lum * sin_theta[:, None] * float(np.float32(self.intensity))).reshape(-1)
        total = np.cumsum(weights)[-1]  # sequential, as the reference sums
        if not (total > 0) or not np.isfinite(total):
            return np.zeros(w * h, dtype=np.float32)
        cdf = np.cumsum(weights / total).astype(np.float32)
        cdf[-1] = 1.0
        return cdf


@dataclasses.dataclass
class Scene:
    """Renderer-neutral scene: camera, render settings, materials and primitive arrays."""

    camera_position: tuple
    camera_look_at: tuple
    camera_up: tuple = (0.0, 1.0, 0.0)
    fov_degrees: float = 45.0
    width: int = 320
    height: int = 180
    samples: int = 4
    max_bounces: int = 4
    background: int = gt.SKY
    materials: list = dataclasses.field(default_factory=list)
    sphere_centers: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros((0, 3), np.float32))
    sphere_radii: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros((0,), np.float32))
    sphere_materials: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros((0,), np.uint32))
    triangles: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros((0, 3, 3), np.float32))
    triangle_materials: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros((0,), np.uint32))
    triangle_normals: Optional[np.ndarray] = None  # (n, 3, 3) or None
    triangle_uvs: Optional[np.ndarray] = None  # (n, 3, 2) or None
    triangle_attr_flags: Optional[np.ndarray] = None  # (n,) bit0 normals, bit1 uvs
    environment: Optional[EnvironmentMap] = None
    texture_pixels: Optional[np.ndarray] = None  # packed RGBA8 atlas (u32), when ``textures`` is empty
    textures: list = dataclasses.field(default_factory=list)  # (width, height, RGBA8 uint8 array)
    exposure_stops: float = 0.0  # display block of a loaded scene file

    def __post_init__(self):
        self.sphere_centers = np.ascontiguousarray(self.sphere_centers, np.float32).reshape(-1, 3)
        self.sphere_radii = np.ascontiguousarray(self.sphere_radii, np.float32).reshape(-1)
        self.sphere_materials = np.ascontiguousarray(self.sphere_materials, np.uint32).reshape(-1)
        self.triangles = np.ascontiguousarray(self.triangles, np.float32).reshape(-1, 3, 3)
        self.triangle_materials = np.ascontiguousarray(self.triangle_materials, np.uint32).reshape(-1)

    @property
    def sphere_count(self) -> int:
        return int(self.sphere_radii.shape[0])

    @property
    def triangle_count(self) -> int:
        return int(self.triangles.shape[0])

    def material_index(self, name: str) -> int:
        for i, m in enumerate(self.materials):
            if m.name == name:
                return i
        raise KeyError(f"unknown material {name!r}")


# --------------------------------------------------------------------------- f32 vector helpers
def _f32(v) -> np.ndarray:
    return np.asarray(v, dtype=np.float32)


def _dot(a, b):
    return np.float32(a[0] * b[0]) + np.float32(a[1] * b[1]) + np.float32(a[2] * b[2])


def _cross(a, b):
    return _f32([a[1] * b[2] - b[1] * a[2], a[2] * b[0] - b[2] * a[0], a[0] * b[1] - b[0] * a[1]])


def _normalize(a):
    inv = np.float32(1.0) / np.sqrt(np.float32(_dot(a, a)))
    return _f32(a * inv)


def make_camera(position, look_at, up, fov_degrees: float, aspect: float) -> np.ndarray:
    """Pinhole viewport basis in f32 (scene_upload.rs:352-368 == camera.rs:54-91)."""
    position, look_at, up = _f32(position), _f32(look_at), _f32(up)
    view = _f32(position - look_at)
    if not np.all(np.isfinite(view)) or _dot(view, view) <= F32_EPSILON:
        raise ValueError("camera position and look_at must differ")
    if not (0.0 < fov_degrees < 180.0) or not math.isfinite(aspect) or aspect <= 0:
        raise ValueError("camera FOV and aspect ratio must be positive and finite")
    backward = _normalize(view)
    right = _cross(up, backward)
    if not np.all(np.isfinite(right)) or _dot(right, right) <= F32_EPSILON:
        raise ValueError("camera up vector must not be parallel to the view direction")
    right = _normalize(right)
    true_up = _cross(backward, right)
    radians = np.float32(fov_degrees) * np.float32(np.float32(math.pi) / np.float32(180.0))
    vh = np.float32(2.0) * np.float32(math.tan(np.float32(0.5) * radians))
    vw = np.float32(aspect) * vh
    horizontal = _f32(vw * right)
    vertical = _f32(vh * true_up)
    lower_left = _f32(position - horizontal * np.float32(0.5) - vertical * np.float32(0.5) - backward)
    cam = np.zeros(1, gt.CAMERA)
    cam["origin"][0, :3] = position
    cam["lower_left_corner"][0, :3] = lower_left
    cam["horizontal"][0, :3] = horizontal
    cam["vertical"][0, :3] = vertical
    return cam


@dataclasses.dataclass
class SceneGpuData:
    """Packed records (scene_upload.rs:17-40)."""

    params: np.ndarray
    camera: np.ndarray
    spheres: np.ndarray
    triangles: np.ndarray
    triangle_attributes: np.ndarray
    materials: np.ndarray
    lights: np.ndarray
    bvh_nodes: Optional[np.ndarray]
    bvh_primitives: Optional[np.ndarray]
    texture_pixels: Optional[np.ndarray]
    environment_pixels: Optional[np.ndarray]

    def host_bytes(self) -> int:
        """Bytes of all packed arrays (the host-to-device upload volume)."""
        total = 0
        for a in (
            self.params,
            self.camera,
            self.spheres,
            self.triangles,
            self.triangle_attributes,
            self.materials,
            self.lights,
            self.bvh_nodes,
            self.bvh_primitives,
            self.texture_pixels,
            self.environment_pixels,
        ):
            if a is not None:
                total += a.nbytes
        return total


def lights_to_gpu(scene: Scene):
    """Emissive primitives with cumulative power weights (scene_upload.rs:412-475)."""
    mats = scene.materials
    emissive = np.array([m.kind == gt.EMISSIVE for m in mats], dtype=bool)
    strength = np.array([m.strength for m in mats], dtype=np.float32)
    color = np.array([m.albedo for m in mats], dtype=np.float32).reshape(-1, 3)
    lum = (np.float32(0.2126) * color[:, 0] + np.float32(0.7152) * color[:, 1]) + np.float32(0.0722) * color[:, 2]
    records = []
    cumulative = np.float32(0.0)
    tri_idx = np.nonzero(emissive[scene.triangle_materials])[0] if scene.triangle_count else np.zeros(0, int)
    for i in tri_idx:
        v = scene.triangles[i]
        m = int(scene.triangle_materials[i])
        c = _cross(_f32(v[1] - v[0]), _f32(v[2] - v[0]))
        area = np.float32(0.5) * np.sqrt(np.float32(_dot(c, c)))
        weight = np.float32(area * lum[m]) * strength[m]
        if weight <= 0:
            continue
        cumulative = np.float32(cumulative + weight)
        rec = np.zeros(1, gt.LIGHT)
        rec["kind"], rec["material_index"] = 0, m
        rec["v0"][0, :3], rec["v1"][0, :3], rec["v2"][0, :3] = v[0], v[1], v[2]
        rec["area_weight_cumulative"][0] = (area, weight, cumulative, 0.0)
        records.append(rec)
    sph_idx = np.nonzero(emissive[scene.sphere_materials])[0] if scene.sphere_count else np.zeros(0, int)
    for i in sph_idx:
        m = int(scene.sphere_materials[i])
        r = scene.sphere_radii[i]
        area = np.float32(np.float32(4.0) * np.float32(math.pi)) * r * r
        weight = np.float32(area * lum[m]) * strength[m]
        if weight <= 0:
            continue
        cumulative = np.float32(cumulative + weight)
        rec = np.zeros(1, gt.LIGHT)
        rec["kind"], rec["material_index"] = 1, m
        rec["center_radius"][0] = (*scene.sphere_centers[i], r)
        rec["area_weight_cumulative"][0] = (area, weight, cumulative, 0.0)
        records.append(rec)
    lights = np.concatenate(records) if records else np.zeros(0, gt.LIGHT)
    return lights, float(cumulative)


def scene_to_gpu(scene: Scene, bvh: Optional[tuple] = None) -> SceneGpuData:
    """Validates and packs ``scene`` (scene_upload.rs:79-294).

    ``bvh`` may be ``(nodes, primitive_refs)`` in GpuBvhNode / GpuPrimitiveRef records; when
    omitted the library builds the identical median-split hierarchy itself.
    """
    if scene.sphere_count == 0 and scene.triangle_count == 0:
        raise ValueError("GPU renderer requires at least one object")
    if not scene.materials:
        raise ValueError("GPU renderer requires at least one material")
    camera = make_camera(
        scene.camera_position, scene.camera_look_at, scene.camera_up, scene.fov_degrees,
        float(np.float32(scene.width) / np.float32(scene.height)),
    )
    spheres = np.zeros(scene.sphere_count, gt.SPHERE)
    spheres["center_radius"][:, :3] = scene.sphere_centers
    spheres["center_radius"][:, 3] = scene.sphere_radii
    spheres["material_index"] = scene.sphere_materials
    tris = np.zeros(scene.triangle_count, gt.TRIANGLE)
    tris["v0"][:, :3] = scene.triangles[:, 0]
    tris["v1"][:, :3] = scene.triangles[:, 1]
    tris["v2"][:, :3] = scene.triangles[:, 2]
    tris["material_index"] = scene.triangle_materials
    attrs = np.zeros(scene.triangle_count, gt.TRIANGLE_ATTRIBUTES)
    flags = np.zeros(scene.triangle_count, np.uint32)
    if scene.triangle_normals is not None:
        n = np.asarray(scene.triangle_normals, np.float32).reshape(-1, 3, 3)
        attrs["n0"][:, :3], attrs["n1"][:, :3], attrs["n2"][:, :3] = n[:, 0], n[:, 1], n[:, 2]
        flags |= 1
    if scene.triangle_uvs is not None:
        uv = np.asarray(scene.triangle_uvs, np.float32).reshape(-1, 3, 2)
        attrs["uv0"], attrs["uv1"], attrs["uv2"] = uv[:, 0], uv[:, 1], uv[:, 2]
        flags |= 2
    if scene.triangle_attr_flags is not None:
        flags &= np.asarray(scene.triangle_attr_flags, np.uint32)
    attrs["flags"] = flags
    # Texture atlas: textures back to back, one little-endian RGBA8 word per texel.
    texels = scene.texture_pixels
    tex_meta = []
    if scene.textures:
        offset, words = 0, []
        for w, h, rgba in scene.textures:
            if w <= 0 or h <= 0 or len(rgba) != w * h * 4:
                raise ValueError("texture dimensions must be nonzero and match its pixel data")
            tex_meta.append((offset, w, h))
            words.append(np.ascontiguousarray(rgba, np.uint8).view("<u4"))
            offset += w * h
        texels = np.concatenate(words).astype(np.uint32)
    mats = np.zeros(len(scene.materials), gt.MATERIAL)
    for i, m in enumerate(scene.materials):
        mats[i]["kind"] = m.kind
        if m.texture is not None:
            if m.texture >= len(tex_meta):
                raise ValueError("material references an unknown texture")
            mats[i]["texture_offset"], mats[i]["texture_width"], mats[i]["texture_height"] = tex_meta[m.texture]
        if m.kind == gt.DIELECTRIC:
            mats[i]["albedo"] = (1.0, 1.0, 1.0, 1.0)
        else:
            mats[i]["albedo"] = (*m.albedo, 1.0)
        if m.kind == gt.METAL:
            mats[i]["params"] = (m.roughness, 0, 0, 0)
        elif m.kind == gt.DIELECTRIC:
            mats[i]["params"] = (0, m.ior, 0, 0)
        elif m.kind == gt.EMISSIVE:
            mats[i]["params"] = (0, 0, m.strength, 0)
    if scene.sphere_count and int(scene.sphere_materials.max()) >= len(scene.materials):
        raise ValueError("sphere references an unknown material")
    if scene.triangle_count and int(scene.triangle_materials.max()) >= len(scene.materials):
        raise ValueError("triangle references an unknown material")
    lights, total_weight = lights_to_gpu(scene)
    env = scene.environment
    env_pixels = None
    if scene.background == gt.ENVIRONMENT:
        if env is None:
            raise ValueError("environment background requires an environment map")
    if env is not None:
        env_pixels = np.zeros((env.width * env.height, 4), np.float32)
        env_pixels[:, :3] = env.pixels.reshape(-1, 3)
        env_pixels[:, 3] = env.importance_cdf()
    params = np.zeros(1, gt.RENDER_PARAMS)
    p = params[0]
    p["width"], p["height"], p["samples"], p["max_bounces"] = scene.width, scene.height, scene.samples, scene.max_bounces
    p["sphere_count"], p["triangle_count"], p["material_count"] = scene.sphere_count, scene.triangle_count, len(scene.materials)
    p["background_kind"] = scene.background
    p["light_count"], p["total_light_weight"] = len(lights), total_weight
    if scene.background == gt.ENVIRONMENT and env is not None:
        p["environment_width"], p["environment_height"] = env.width, env.height
        p["environment_intensity"] = env.intensity
        rot = np.fmod(np.float32(env.rotation_degrees), np.float32(360.0))  # f32::rem_euclid(360.0)
        p["environment_rotation_degrees"] = rot + np.float32(360.0) if rot < 0 else rot
    nodes, prims = (None, None) if bvh is None else bvh
    if nodes is not None:
        p["bvh_node_count"], p["bvh_primitive_count"] = len(nodes), len(prims)
    return SceneGpuData(
        params=params,
        camera=camera,
        spheres=spheres,
        triangles=tris,
        triangle_attributes=attrs,
        materials=mats,
        lights=lights,
        bvh_nodes=nodes,
        bvh_primitives=prims,
        texture_pixels=texels,
        environment_pixels=env_pixels,
    )


# --------------------------------------------------------------------------- JSON scene loading
def box_triangles(center, size) -> np.ndarray:
    """Twelve triangles of an axis-aligned box (crates/toaster-scene/src/loader.rs:1541-1568)."""
    c, half = _f32(center), _f32(size) * np.float32(0.5)
    signs = [(-1, -1, -1), (-1, -1, 1), (-1, 1, -1), (-1, 1, 1), (1, -1, -1), (1, -1, 1), (1, 1, -1), (1, 1, 1)]
    verts = [_f32(c + _f32([sx * half[0], sy * half[1], sz * half[2]])) for sx, sy, sz in signs]
    faces = [(1, 5, 7), (1, 7, 3), (4, 0, 2), (4, 2, 6), (0, 1, 3), (0, 3, 2), (5, 4, 6), (5, 6, 7), (3, 7, 6),
             (3, 6, 2), (0, 4, 5), (0, 5, 1)]
    return np.array([[verts[i] for i in f] for f in faces], dtype=np.float32)


def triangle_is_valid(v: np.ndarray) -> bool:
    """Finite and non-collinear (loader.rs:1584-1593)."""
    if not np.all(np.isfinite(v)):
        return False
    c = _cross(_f32(v[1] - v[0]), _f32(v[2] - v[0]))
    return bool(_dot(c, c) > F32_EPSILON)


def _triangles_valid(v: np.ndarray) -> np.ndarray:
    """triangle_is_valid over an (n, 3, 3) array."""
    e1, e2 = v[:, 1] - v[:, 0], v[:, 2] - v[:, 0]
    c = np.stack([e1[:, 1] * e2[:, 2] - e2[:, 1] * e1[:, 2], e1[:, 2] * e2[:, 0] - e2[:, 2] * e1[:, 0],
                  e1[:, 0] * e2[:, 1] - e2[:, 0] * e1[:, 1]], axis=1)
    with np.errstate(invalid="ignore", over="ignore"):
        d = (c[:, 0] * c[:, 0] + c[:, 1] * c[:, 1]) + c[:, 2] * c[:, 2]
        return np.all(np.isfinite(v), axis=(1, 2)) & (d > F32_EPSILON)


# f32 matrix arithmetic of the glTF importer (glam's operation order): column-major 4 x 4,
# m[column, row]. Every product and sum below is a float32 operation.
def _m4_mul(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """a * b, column j = ((a0 * b_j.x + a1 * b_j.y) + a2 * b_j.z) + a3 * b_j.w."""
    r = np.zeros((4, 4), np.float32)
    for j in range(4):
        v = a[0] * b[j, 0]
        v = v + a[1] * b[j, 1]
        v = v + a[2] * b[j, 2]
        v = v + a[3] * b[j, 3]
        r[j] = v
    return r


def _transform_points(m: np.ndarray, p: np.ndarray) -> np.ndarray:
    """Mat4::transform_point3 on rows of p: ((x * p.x + y * p.y) + z * p.z) + w."""
    out = np.empty_like(p)
    for row in range(3):
        v = m[0, row] * p[:, 0]
        v = m[1, row] * p[:, 1] + v
        v = m[2, row] * p[:, 2] + v
        out[:, row] = m[3, row] + v
    return out


def _normals_to_world(m: np.ndarray, n: np.ndarray) -> np.ndarray:
    """Mat3::from_mat4(m).inverse().transpose() * n, then normalize_or_zero, in f32."""
    x, y, z = m[0, :3], m[1, :3], m[2, :3]
    t0, t1, t2 = _cross(y, z), _cross(z, x), _cross(x, y)
    inv_det = np.float32(1.0) / _dot(z, t2)
    c0, c1, c2 = t0 * inv_det, t1 * inv_det, t2 * inv_det
    r = c0[None, :] * n[:, 0:1]
    r = r + c1[None, :] * n[:, 1:2]
    r = r + c2[None, :] * n[:, 2:3]
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        d = (r[:, 0] * r[:, 0] + r[:, 1] * r[:, 1]) + r[:, 2] * r[:, 2]
        rcp = np.float32(1.0) / np.sqrt(d)
        ok = np.isfinite(rcp) & (rcp > 0)
        return np.where(ok[:, None], r * rcp[:, None], np.float32(0.0)).astype(np.float32)


def _trs_matrix(node: dict) -> np.ndarray:
    """A node's local matrix: ``matrix`` as given, else T * R * S with the quaternion expanded
    as the importer's math expands it."""
    if "matrix" in node:
        m = _f32(node["matrix"])
        if m.shape != (16,):
            raise ValueError("glTF node matrix must have 16 components")
        return m.reshape(4, 4).copy()
    t = _f32(node.get("translation", [0.0, 0.0, 0.0]))
    x, y, z, w = (np.float32(v) for v in node.get("rotation", [0.0, 0.0, 0.0, 1.0]))
    s = _f32(node.get("scale", [1.0, 1.0, 1.0]))
    one = np.float32(1.0)
    tm = np.eye(4, dtype=np.float32)
    tm[3, :3] = t
    x2, y2, z2 = x + x, y + y, z + z
    xx2, xy2, xz2 = x2 * x, x2 * y, x2 * z
    yy2, yz2, zz2 = y2 * y, y2 * z, z2 * z
    sy2, sz2, sx2 = y2 * w, z2 * w, x2 * w
    rm = np.zeros((4, 4), np.float32)
    rm[0, :3] = (one - yy2 - zz2, xy2 + sz2, xz2 - sy2)
    rm[1, :3] = (xy2 - sz2, one - xx2 - zz2, yz2 + sx2)
    rm[2, :3] = (xz2 + sy2, yz2 - sx2, one - xx2 - yy2)
    rm[3, 3] = one
    sm = np.zeros((4, 4), np.float32)
    sm[0, 0], sm[1, 1], sm[2, 2], sm[3, 3] = s[0], s[1], s[2], one
    return _m4_mul(_m4_mul(tm, rm), sm)


def _decode_png(data: bytes):
    """8-bit PNG as (width, height, channels, uint8 pixels) after png's EXPAND transform:
    palettes to RGB (RGBA with tRNS), grey of depth 1/2/4 scaled to 8 bits, a tRNS colour key
    to an alpha channel. 16-bit images are rejected (image_to_rgba8, gltf_loader.rs:200-233)."""
    if data[:8] != b"\x89PNG\r\n\x1a\n":
        raise ValueError("not a PNG image")
    pos, idat, palette, trns, ihdr = 8, bytearray(), b"", b"", None
    while pos + 12 <= len(data):
        n = struct.unpack(">I", data[pos:pos + 4])[0]
        ctype = data[pos + 4:pos + 8]
        body = data[pos + 8:pos + 8 + n]
        if len(body) != n or pos + 12 + n > len(data):
            raise ValueError("truncated PNG chunk")
        if zlib.crc32(data[pos + 4:pos + 8 + n]) != struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])[0]:
            raise ValueError("PNG chunk CRC mismatch")
        if ctype == b"IHDR":
            ihdr = struct.unpack(">IIBBBBB", body)
        elif ctype == b"PLTE":
            palette = body
        elif ctype == b"tRNS":
            trns = body
        elif ctype == b"IDAT":
            idat += body
        elif ctype == b"IEND":
            break
        elif not ctype[0] & 0x20:
            raise ValueError("unknown critical PNG chunk")
        pos += n + 12
    if ihdr is None:
        raise ValueError("truncated PNG")
    w, h, depth, color, comp, filt, interlace = ihdr
    if comp != 0 or filt != 0 or interlace > 1:
        raise ValueError("unsupported PNG compression, filter or interlace method")
    if w == 0 or h == 0:
        raise ValueError("PNG dimensions must be nonzero")
    if depth == 16:
        raise ValueError("unsupported 16-bit image; use an 8-bit image")
    samples = {0: 1, 2: 3, 3: 1, 4: 2, 6: 4}.get(color)
    if samples is None or (color in (2, 4, 6) and depth != 8) or depth not in (1, 2, 4, 8):
        raise ValueError("invalid PNG colour type or bit depth")
    raw = zlib.decompress(bytes(idat))
    if color == 0:
        out_ch = 2 if len(trns) >= 2 else 1
    elif color == 2:
        out_ch = 4 if len(trns) >= 6 else 3
    elif color == 3:
        out_ch = 4 if trns else 3
    else:
        out_ch = samples
    img = np.zeros((h, w, out_ch), np.uint8)
    passes = [(0, 0, 1, 1)] if interlace == 0 else [(0, 0, 8, 8), (4, 0, 8, 8), (0, 4, 4, 8), (2, 0, 4, 4),
                                                     (0, 2, 2, 4), (1, 0, 2, 2), (0, 1, 1, 2)]
    bpp = max(1, samples * depth // 8)
    off = 0
    for x0, y0, dx, dy in passes:
        pw = (w - x0 + dx - 1) // dx if w > x0 else 0
        ph = (h - y0 + dy - 1) // dy if h > y0 else 0
        if pw == 0 or ph == 0:
            continue
        rb = (pw * samples * depth + 7) // 8
        prev = bytearray(rb)
        for py in range(ph):
            ftype = raw[off]
            cur = bytearray(raw[off + 1:off + 1 + rb])
            if len(cur) != rb:
                raise ValueError("corrupt PNG image data")
            off += rb + 1
            for i in range(rb):
                left = cur[i - bpp] if i >= bpp else 0
                up = prev[i]
                if ftype == 1:
                    cur[i] = (cur[i] + left) & 0xFF
                elif ftype == 2:
                    cur[i] = (cur[i] + up) & 0xFF
                elif ftype == 3:
                    cur[i] = (cur[i] + ((left + up) >> 1)) & 0xFF
                elif ftype == 4:
                    ul = prev[i - bpp] if i >= bpp else 0
                    p = left + up - ul
                    pa, pb, pc = abs(p - left), abs(p - up), abs(p - ul)
                    pred = left if (pa <= pb and pa <= pc) else (up if pb <= pc else ul)
                    cur[i] = (cur[i] + pred) & 0xFF
                elif ftype != 0:
                    raise ValueError("invalid PNG filter type")
            prev = cur
            y = y0 + py * dy
            for px in range(pw):
                x = x0 + px * dx
                if color in (0, 3):
                    if depth == 8:
                        v = cur[px]
                    else:
                        bit = px * depth
                        v = (cur[bit >> 3] >> (8 - depth - (bit & 7))) & ((1 << depth) - 1)
                    if color == 0:
                        img[y, x, 0] = v if depth == 8 else v * (255 // ((1 << depth) - 1))
                        if out_ch == 2:
                            img[y, x, 1] = 0 if v == (trns[0] << 8 | trns[1]) else 255
                    else:
                        if 3 * v + 2 >= len(palette):
                            raise ValueError("PNG palette index out of range")
                        img[y, x, :3] = tuple(palette[3 * v:3 * v + 3])
                        if out_ch == 4:
                            img[y, x, 3] = trns[v] if v < len(trns) else 255
                elif color == 2:
                    r, g, b = cur[3 * px:3 * px + 3]
                    img[y, x, :3] = (r, g, b)
                    if out_ch == 4:
                        keyed = (trns[0], trns[1], trns[2], trns[3], trns[4], trns[5]) == (0, r, 0, g, 0, b)
                        img[y, x, 3] = 0 if keyed else 255
                else:
                    img[y, x] = tuple(cur[samples * px:samples * px + samples])
    return w, h, out_ch, img


def _rgba8(w: int, h: int, ch: int, img: np.ndarray) -> np.ndarray:
    """gltf_loader.rs:200-233 image_to_rgba8: grey (+alpha), RGB and RGBA to RGBA8."""
    out = np.full((h, w, 4), 255, np.uint8)
    if ch <= 2:
        out[..., 0] = out[..., 1] = out[..., 2] = img[..., 0]
        if ch == 2:
            out[..., 3] = img[..., 1]
    else:
        out[..., :ch] = img
    return out.reshape(-1)


def _gltf_uri(uri: str, base: Path) -> bytes:
    if uri.startswith("data:"):
        head, _, payload = uri.partition(",")
        if ";base64" not in head:
            raise ValueError("only base64 data URIs are supported")
        return base64.b64decode(payload + "=" * (-len(payload) % 4))
    if "://" in uri:
        raise ValueError("unsupported URI scheme")
    return (base / urllib.parse.unquote(uri)).read_bytes()


def _load_gltf(path: Path) -> dict:
    """glTF / GLB triangle import (crates/toaster-assets/src/gltf_loader.rs:11-197).

    Returns positions, normals and texture coordinates per vertex (world space), triangles as
    vertex-index triples with their glTF material index (-1 for none), the glTF materials as
    (base colour factor, texture index or -1) and the textures as (width, height, RGBA8 bytes).
    """
    blob = path.read_bytes()
    bin_chunk = None
    if blob[:4] == b"glTF":
        version, total = struct.unpack("<II", blob[4:12])
        if version != 2:
            raise ValueError(f"{path}: unsupported GLB version")
        pos, text = 12, None
        while pos + 8 <= min(total, len(blob)):
            n, ctype = struct.unpack("<II", blob[pos:pos + 8])
            if text is None:
                if ctype != 0x4E4F534A:
                    raise ValueError(f"{path}: GLB does not start with a JSON chunk")
                text = blob[pos + 8:pos + 8 + n].decode("utf-8")
            elif ctype == 0x004E4942 and bin_chunk is None:
                bin_chunk = blob[pos + 8:pos + 8 + n]
            pos += 8 + n
        doc = json.loads(text)
    else:
        doc = json.loads(blob.decode("utf-8"))
    base = path.parent
    buffers = []
    for i, b in enumerate(doc.get("buffers") or []):
        if b.get("uri") is not None:
            data = _gltf_uri(b["uri"], base)
        elif i == 0 and bin_chunk is not None:
            data = bin_chunk
        else:
            raise ValueError(f"{path}: buffer without a URI outside a GLB")
        if len(data) < b["byteLength"]:
            raise ValueError(f"{path}: buffer is shorter than its byteLength")
        buffers.append(data[:b["byteLength"]])

    comp = {5120: "<i1", 5121: "<u1", 5122: "<i2", 5123: "<u2", 5125: "<u4", 5126: "<f4"}
    shapes = {"SCALAR": 1, "VEC2": 2, "VEC3": 3, "VEC4": 4}

    def view(i):
        v = doc["bufferViews"][i]
        data = buffers[v["buffer"]]
        off, n = v.get("byteOffset", 0), v["byteLength"]
        if off + n > len(data):
            raise ValueError(f"{path}: bufferView exceeds its buffer")
        return data[off:off + n], v.get("byteStride", 0)

    def accessor(i, ncomp):
        a = doc["accessors"][i]
        dt = np.dtype(comp[a["componentType"]])
        if shapes[a["type"]] != ncomp:
            raise ValueError(f"{path}: accessor has type {a['type']}")
        count = a["count"]
        out = np.zeros((count, ncomp), np.float64)
        elem = dt.itemsize * ncomp
        if a.get("bufferView") is not None:
            data, stride = view(a["bufferView"])
            stride = stride or elem
            off = a.get("byteOffset", 0)
            if count and off + stride * (count - 1) + elem > len(data):
                raise ValueError(f"{path}: accessor exceeds its bufferView")
            for k in range(count):
                out[k] = np.frombuffer(data, dt, ncomp, off + k * stride)
        sp = a.get("sparse")
        if sp:
            n = sp["count"]
            idt = np.dtype(comp[sp["indices"]["componentType"]])
            idata, _ = view(sp["indices"]["bufferView"])
            vdata, _ = view(sp["values"]["bufferView"])
            idx = np.frombuffer(idata, idt, n, sp["indices"].get("byteOffset", 0)).astype(np.int64)
            vals = np.frombuffer(vdata, dt, n * ncomp, sp["values"].get("byteOffset", 0)).reshape(n, ncomp)
            if np.any(idx >= count):
                raise ValueError(f"{path}: sparse index out of range")
            out[idx] = vals
        return a["componentType"], out

    def floats(i, ncomp):
        ctype, raw = accessor(i, ncomp)
        if ctype != 5126:
            raise ValueError(f"{path}: expected float components")
        return raw.astype(np.float32)

    def tex_coords(i):
        ctype, raw = accessor(i, 2)
        if ctype == 5126:
            return raw.astype(np.float32)
        if ctype in (5121, 5123):
            return raw.astype(np.float32) / np.float32(255.0 if ctype == 5121 else 65535.0)
        raise ValueError(f"{path}: invalid TEXCOORD_0 component type")

    materials = []
    for m in doc.get("materials") or []:
        pbr = m.get("pbrMetallicRoughness") or {}
        factor = tuple(float(np.float32(c)) for c in (pbr.get("baseColorFactor") or (1.0, 1.0, 1.0, 1.0)))
        tex = (pbr.get("baseColorTexture") or {}).get("index", -1)
        materials.append((factor, tex))
    images = []
    for i, im in enumerate(doc.get("images") or []):
        if im.get("uri") is not None:
            data = _gltf_uri(im["uri"], base)
        elif im.get("bufferView") is not None:
            data = view(im["bufferView"])[0]
        else:
            raise ValueError(f"{path}: image {i} without a URI or bufferView")
        if data[:3] == b"\xff\xd8\xff":
            raise ValueError(f"{path}: JPEG textures are not supported by this loader; use PNG")
        w, h, ch, img = _decode_png(bytes(data))
        images.append((w, h, _rgba8(w, h, ch, img)))
    textures = []
    for t in doc.get("textures") or []:
        if t.get("source") is None or t["source"] >= len(images):
            raise ValueError(f"{path}: texture references an unknown image")
        textures.append(images[t["source"]])
    for _, tex in materials:
        if tex >= len(textures):
            raise ValueError(f"{path}: material references an unknown texture")

    positions, normals, has_normal, uvs, has_uv, tris, tri_mats = [], [], [], [], [], [], []
    n_vertices = 0

    def load_node(index, parent, depth):
        nonlocal n_vertices
        if depth > 256:
            raise ValueError(f"{path}: node hierarchy is too deep or cyclic")
        node = doc["nodes"][index]
        world = _m4_mul(parent, _trs_matrix(node))
        if node.get("mesh") is not None:
            mi = node["mesh"]
            for pi, prim in enumerate(doc["meshes"][mi]["primitives"]):
                ctx = f"glTF mesh {mi} primitive {pi}"
                if prim.get("mode", 4) != 4:
                    raise ValueError(f"{ctx} uses unsupported mode {prim['mode']}; only triangles are supported")
                attrs = prim["attributes"]
                if attrs.get("POSITION") is None:
                    raise ValueError(f"{ctx} has no POSITION attribute")
                pos = _transform_points(world, floats(attrs["POSITION"], 3))
                if not np.all(np.isfinite(pos)):
                    raise ValueError(f"{ctx} produces non-finite positions")
                nrm = floats(attrs["NORMAL"], 3) if attrs.get("NORMAL") is not None else None
                uv = tex_coords(attrs["TEXCOORD_0"]) if attrs.get("TEXCOORD_0") is not None else None
                if (nrm is not None and len(nrm) != len(pos)) or (uv is not None and len(uv) != len(pos)):
                    raise ValueError(f"{ctx} has mismatched vertex attribute counts")
                if prim.get("indices") is not None:
                    ctype, raw = accessor(prim["indices"], 1)
                    if ctype not in (5121, 5123, 5125):
                        raise ValueError(f"{ctx}: invalid index component type")
                    idx = raw.reshape(-1).astype(np.int64)
                else:
                    idx = np.arange(len(pos), dtype=np.int64)
                if len(idx) % 3:
                    raise ValueError(f"{ctx} has an index count that is not divisible by three")
                if len(idx) and int(idx.max()) >= len(pos):
                    raise ValueError(f"{ctx} contains an out-of-bounds index")
                if nrm is not None:
                    nrm = _normals_to_world(world, nrm)
                    if not np.all(np.isfinite(nrm)) or np.any(np.all(nrm == 0, axis=1)):
                        raise ValueError(f"{ctx} produces an invalid normal")
                if uv is not None and not np.all(np.isfinite(uv)):
                    raise ValueError(f"{ctx} contains non-finite texture coordinates")
                material = prim.get("material")
                if material is not None and material >= len(materials):
                    raise ValueError(f"{ctx} references an unknown material")
                n = len(pos)
                positions.append(pos)
                normals.append(nrm if nrm is not None else np.zeros((n, 3), np.float32))
                has_normal.append(np.full(n, nrm is not None))
                uvs.append(uv if uv is not None else np.zeros((n, 2), np.float32))
                has_uv.append(np.full(n, uv is not None))
                tris.append(idx.reshape(-1, 3) + n_vertices)
                tri_mats.append(np.full(len(idx) // 3, -1 if material is None else material, np.int64))
                n_vertices += n
        for c in node.get("children") or []:
            load_node(c, world, depth + 1)

    scenes = doc.get("scenes") or []
    chosen = [scenes[doc["scene"]]] if doc.get("scene") is not None else scenes
    for sc in chosen:
        for r in sc.get("nodes") or []:
            load_node(r, np.eye(4, dtype=np.float32), 0)
    if sum(len(t) for t in tris) == 0:
        raise ValueError(f"glTF {path} contains no triangle primitives")
    return {"positions": np.concatenate(positions), "normals": np.concatenate(normals),
            "has_normal": np.concatenate(has_normal), "uvs": np.concatenate(uvs), "has_uv": np.concatenate(has_uv),
            "triangles": np.concatenate(tris), "triangle_materials": np.concatenate(tri_mats),
            "materials": materials, "textures": textures}


def _read_hdr(path: Path) -> EnvironmentMap:
    """Radiance RGBE (.hdr) reader: flat, original run-length and new run-length scanlines."""
    data = path.read_bytes()
    if not (data.startswith(b"#?RADIANCE") or data.startswith(b"#?RGBE")):
        raise ValueError(f"{path}: not a Radiance image")
    pos = 0
    while True:
        end = data.index(b"\n", pos)
        line = data[pos:end].rstrip(b"\r")
        pos = end + 1
        if not line:
            break
        if line.startswith(b"FORMAT=") and line != b"FORMAT=32-bit_rle_rgbe":
            raise ValueError(f"{path}: unsupported Radiance format")
    end = data.index(b"\n", pos)
    parts = data[pos:end].rstrip(b"\r").split()
    pos = end + 1
    if len(parts) != 4 or parts[0] != b"-Y" or parts[2] != b"+X":
        raise ValueError(f"{path}: unsupported Radiance orientation")
    h, w = int(parts[1]), int(parts[3])
    rgbe = np.zeros((h, w, 4), np.uint8)
    for y in range(h):
        if 8 <= w < 0x8000 and data[pos] == 2 and data[pos + 1] == 2 and not data[pos + 2] & 0x80 and \
                (data[pos + 2] << 8 | data[pos + 3]) == w:
            pos += 4
            for c in range(4):
                x = 0
                while x < w:
                    count = data[pos]
                    pos += 1
                    if count > 128:
                        count -= 128
                        if count > w - x:
                            raise ValueError(f"{path}: bad Radiance run length")
                        rgbe[y, x:x + count, c] = data[pos]
                        pos += 1
                    else:
                        if count == 0 or count > w - x:
                            raise ValueError(f"{path}: bad Radiance run length")
                        rgbe[y, x:x + count, c] = np.frombuffer(data, np.uint8, count, pos)
                        pos += count
                    x += count
        else:
            x, shift = 0, 0
            while x < w:
                p = data[pos:pos + 4]
                pos += 4
                if p[0] == 1 and p[1] == 1 and p[2] == 1:
                    if x == 0:
                        raise ValueError(f"{path}: Radiance run without a preceding pixel")
                    count = p[3] << shift
                    if count > w - x:
                        raise ValueError(f"{path}: bad Radiance run length")
                    rgbe[y, x:x + count] = rgbe[y, x - 1]
                    x += count
                    shift += 8
                else:
                    rgbe[y, x] = tuple(p)
                    x += 1
                    shift = 0
    e = rgbe[..., 3].astype(np.int32)
    scale = np.where(e > 0, np.ldexp(1.0, e - 136), 0.0)
    pixels = (rgbe[..., :3].astype(np.float64) * scale[..., None]).astype(np.float32)
    return EnvironmentMap(w, h, pixels)


_SRGB_LUT = None


def _srgb_to_linear(v: np.ndarray) -> np.ndarray:
    """texture.rs:84-91 in f32, with the C library's powf as the reference's f32::powf uses it."""
    global _SRGB_LUT
    if _SRGB_LUT is None:
        import ctypes
        import ctypes.util

        libm = ctypes.CDLL(ctypes.util.find_library("m"))
        libm.powf.argtypes = [ctypes.c_float, ctypes.c_float]
        libm.powf.restype = ctypes.c_float
        lut = np.zeros(256, np.float32)
        for i in range(256):
            x = np.float32(i) / np.float32(255.0)
            if x <= np.float32(0.04045):
                lut[i] = x / np.float32(12.92)
            else:
                lut[i] = libm.powf(float((x + np.float32(0.055)) / np.float32(1.055)), 2.4)
        _SRGB_LUT = lut
    return _SRGB_LUT[np.asarray(v, np.uint8)]


def _load_environment(path: Path) -> EnvironmentMap:
    """environment.rs:94-128: Radiance maps as linear f32, 8-bit PNG maps through sRGB decoding."""
    head = path.read_bytes()[:16]
    if head.startswith(b"#?RADIANCE") or head.startswith(b"#?RGBE"):
        return _read_hdr(path)
    if head.startswith(b"\x89PNG"):
        w, h, ch, img = _decode_png(path.read_bytes())
        rgb = np.repeat(img[..., :1], 3, axis=2) if ch <= 2 else img[..., :3]
        return EnvironmentMap(w, h, _srgb_to_linear(rgb))
    raise ValueError(f"unsupported environment map format (Radiance .hdr and PNG are read): {path}")


def _vec3(v, what: str) -> np.ndarray:
    if not isinstance(v, (list, tuple)) or len(v) != 3 or not all(isinstance(c, (int, float)) and
                                                                 not isinstance(c, bool) for c in v):
        raise ValueError(f"{what}: expected an array of 3 numbers")
    return _f32(v)


def _color_ok(c: np.ndarray) -> bool:
    return bool(np.all(np.isfinite(c)) and np.all(c >= 0) and np.all(c <= 1))


def load_scene(path) -> Scene:
    """Loads a toaster scene JSON file (crates/toaster-scene/src/loader.rs:534-971).

    Camera, render and display settings, named materials, and sphere / box / triangle / glTF
    mesh objects (imported glTF materials and PNG base-colour textures included), with sky /
    black / environment backgrounds (Radiance .hdr or PNG maps), validated with the reference
    loader's rules. Animation, physics, triggers, spawn points and event reactions do not
    change the rendered records and are skipped. The library's native loader (tc_scene_load,
    ``load_scene_gpu``) follows the same rules and produces the same packed records.
    """
    path = Path(path)
    doc = json.loads(path.read_text(encoding="utf-8"))
    if not isinstance(doc, dict):
        raise ValueError("the scene must be a JSON object")
    for key in ("camera", "render", "materials", "objects"):
        if key not in doc:
            raise ValueError(f"missing field `{key}`")
    cam, render = doc["camera"], doc["render"]
    position = _vec3(cam["position"], "camera position")
    look_at = _vec3(cam["look_at"], "camera look_at")
    up = _vec3(cam["up"], "camera up") if cam.get("up") is not None else _f32([0.0, 1.0, 0.0])
    fov = np.float32(cam["fov_degrees"] if "fov_degrees" in cam else cam["vertical_fov_degrees"])
    width, height = int(render["width"]), int(render["height"])
    samples = int(render["samples"] if "samples" in render else render["samples_per_pixel"])
    max_bounces = int(render["max_bounces"])
    if width <= 0 or height <= 0:
        raise ValueError("render width and height must be greater than zero")
    if samples <= 0:
        raise ValueError("render samples must be greater than zero")
    if not (np.float32(0.0) <= fov < np.float32(180.0)):
        raise ValueError("camera fov_degrees must be between 0 and 180")
    view = _f32(position - look_at)
    if not (np.all(np.isfinite(position)) and np.all(np.isfinite(look_at)) and np.all(np.isfinite(up))) or \
            np.all(np.abs(view) <= F32_EPSILON):
        raise ValueError("camera vectors are invalid")
    c = _cross(up, view)
    if not _dot(c, c) > F32_EPSILON:
        raise ValueError("camera up vector must not be parallel to its view direction")
    display = doc.get("display") or {}
    unknown = set(display) - {"exposure_stops", "tone_mapper"}
    if unknown:
        raise ValueError(f"display: unknown field `{sorted(unknown)[0]}`")
    if display.get("tone_mapper", "aces") != "aces":
        raise ValueError("display: unknown tone mapper")
    exposure = np.float32(display.get("exposure_stops") or 0.0)
    if not np.isfinite(exposure):
        raise ValueError("display exposure_stops must be finite")

    scene = Scene(camera_position=tuple(float(v) for v in position), camera_look_at=tuple(float(v) for v in look_at),
                  camera_up=tuple(float(v) for v in up), fov_degrees=float(fov), width=width, height=height,
                  samples=samples, max_bounces=max_bounces)
    scene.exposure_stops = float(exposure)
    names = {}
    for m in doc["materials"]:
        name, kind = m["name"], m["type"]
        if name in names:
            raise ValueError(f"duplicate material name '{name}'")
        if kind == "diffuse":
            albedo = _vec3(m["albedo"], f"material '{name}' albedo")
            if not _color_ok(albedo):
                raise ValueError(f"material '{name}' albedo must be between 0 and 1")
            mat = Material.diffuse(albedo, name)
        elif kind == "metal":
            albedo = _vec3(m["albedo"], f"material '{name}' albedo")
            rough = np.float32(m["roughness"])
            if not _color_ok(albedo):
                raise ValueError(f"material '{name}' albedo must be between 0 and 1")
            if not np.isfinite(rough):
                raise ValueError(f"material '{name}' roughness must be finite")
            mat = Material.metal(albedo, float(min(max(rough, np.float32(0.0)), np.float32(1.0))), name)
        elif kind == "dielectric":
            ior = np.float32(m["ior"])
            if not (np.isfinite(ior) and ior > 0):
                raise ValueError(f"material '{name}' ior must be finite and greater than zero")
            mat = Material.dielectric(float(ior), name)
        elif kind == "emissive":
            color = _vec3(m["color"], f"material '{name}' color")
            strength = np.float32(m["strength"])
            if not _color_ok(color):
                raise ValueError(f"material '{name}' color must be between 0 and 1")
            if not (np.isfinite(strength) and strength >= 0):
                raise ValueError(f"material '{name}' strength must be finite and non-negative")
            mat = Material.emissive(color, float(strength), name)
        else:
            raise ValueError(f"material '{name}': unknown material type `{kind}`")
        names[name] = len(scene.materials)
        scene.materials.append(mat)

    def material_of(obj, what):
        if obj.get("material") not in names:
            raise ValueError(f"{what} references unknown material '{obj.get('material')}'")
        return names[obj["material"]]

    centers, radii, smat = [], [], []
    tris, tmat, tnorm, tuv, tflags = [], [], [], [], []
    ids = set()
    zero_n, zero_uv = np.zeros((3, 3), np.float32), np.zeros((3, 2), np.float32)
    for obj in doc["objects"]:
        kind = obj["type"]
        if kind not in ("sphere", "box", "triangle", "mesh"):
            raise ValueError(f"unknown object type `{kind}`")
        physics = obj.get("physics") is not None
        if obj.get("id") is not None:
            if obj["id"] == "":
                raise ValueError("physics entity id must not be empty")
            if obj["id"] in ids:
                raise ValueError(f"duplicate physics entity id '{obj['id']}'")
            ids.add(obj["id"])
        elif physics and kind != "triangle":
            raise ValueError("physics objects require a nonempty object id")
        if obj.get("group") == "":
            raise ValueError("object group name must not be empty")
        if kind == "sphere":
            center, radius = _vec3(obj["center"], "sphere center"), np.float32(obj["radius"])
            if not (np.all(np.isfinite(center)) and np.isfinite(radius) and radius > 0):
                raise ValueError("sphere radius must be positive and its center must be finite")
            centers.append(center)
            radii.append(radius)
            smat.append(material_of(obj, "sphere"))
        elif kind == "box":
            center, size = _vec3(obj["center"], "box center"), _vec3(obj["size"], "box size")
            if not (np.all(np.isfinite(center)) and np.all(np.isfinite(size)) and np.all(size > 0)):
                raise ValueError("box center must be finite and size components must be positive")
            mi = material_of(obj, "box")
            for v in box_triangles(center, size):
                tris.append(v)
                tmat.append(mi)
                tnorm.append(zero_n)
                tuv.append(zero_uv)
                tflags.append(0)
        elif kind == "triangle":
            if physics:
                raise ValueError("triangle objects do not support physics in the rigid-body MVP")
            vs = obj["vertices"]
            if len(vs) != 3:
                raise ValueError("triangle vertices: expected an array of 3 points")
            v = np.stack([_vec3(p, "triangle vertex") for p in vs])
            if not triangle_is_valid(v):
                raise ValueError("triangle vertices must be finite and non-collinear")
            tris.append(v)
            tmat.append(material_of(obj, "triangle"))
            tnorm.append(zero_n)
            tuv.append(zero_uv)
            tflags.append(0)
        else:
            override = material_of(obj, "mesh") if obj.get("material") is not None else None
            mesh_path = path.parent / obj["path"]
            mesh = _load_gltf(mesh_path)
            imported = []
            if override is None:
                base = len(scene.textures)
                scene.textures.extend(mesh["textures"])
                for factor, tex in mesh["materials"]:
                    mat = Material.diffuse(factor[:3])
                    if tex >= 0:
                        mat.texture = base + tex
                    scene.materials.append(mat)
                    imported.append(len(scene.materials) - 1)
            tri, tm = mesh["triangles"], mesh["triangle_materials"]
            default = None
            if override is None and np.any(tm < 0):
                scene.materials.append(Material.diffuse((1.0, 1.0, 1.0)))
                default = len(scene.materials) - 1
            v = mesh["positions"][tri]
            valid = _triangles_valid(v)
            if not np.all(valid):
                raise ValueError(f"mesh {mesh_path} contains invalid triangle {int(np.argmin(valid))}")
            if override is not None:
                mi = np.full(len(tri), override, np.int64)
            else:
                lut = np.array(imported + [default if default is not None else -1], np.int64)
                mi = lut[np.where(tm < 0, len(imported), tm)]
            has_n = np.all(mesh["has_normal"][tri], axis=1)
            has_uv = np.all(mesh["has_uv"][tri], axis=1)
            textured = np.array([scene.materials[m].texture is not None for m in mi], bool)
            if np.any(textured & ~has_uv):
                k = int(np.argmax(textured & ~has_uv))
                raise ValueError(f"mesh {mesh_path} triangle {k} uses a base-color texture without TEXCOORD_0")
            tris.extend(v)
            tmat.extend(int(m) for m in mi)
            tnorm.extend(np.where(has_n[:, None, None], mesh["normals"][tri], np.float32(0.0)))
            tuv.extend(np.where(has_uv[:, None, None], mesh["uvs"][tri], np.float32(0.0)))
            tflags.extend((has_n.astype(np.uint32) | (has_uv.astype(np.uint32) << 1)).tolist())

    background = render.get("background")
    if background is None or background == "sky":
        scene.background = gt.SKY
    elif background == "black":
        scene.background = gt.BLACK
    elif isinstance(background, dict) and background.get("type") == "environment":
        intensity = np.float32(background["intensity"]) if background.get("intensity") is not None else np.float32(1.0)
        rotation = np.float32(background["rotation_degrees"]) if background.get("rotation_degrees") is not None \
            else np.float32(0.0)
        env = _load_environment(path.parent / background["path"])
        env.intensity, env.rotation_degrees = float(intensity), float(rotation)
        env.__post_init__()
        scene.environment = env
        scene.background = gt.ENVIRONMENT
    else:
        raise ValueError(f"render background: unknown variant {background!r}")
    if centers:
        scene.sphere_centers = _f32(centers)
        scene.sphere_radii = _f32(radii)
        scene.sphere_materials = np.array(smat, np.uint32)
    if tris:
        scene.triangles = np.array(tris, np.float32)
        scene.triangle_materials = np.array(tmat, np.uint32)
        if any(tflags):
            scene.triangle_normals = np.array(tnorm, np.float32)
            scene.triangle_uvs = np.array(tuv, np.float32)
            scene.triangle_attr_flags = np.array(tflags, np.uint32)
    return scene


def load_scene_gpu(path) -> tuple:
    """Loads and packs a scene file with the library's native loader (tc_scene_load).

    Returns ``(SceneGpuData, exposure_stops)``: the records the reference's ``load_scene`` +
    ``scene_to_gpu`` would produce (hierarchy left to the upload), copied out of the library.
    """
    import ctypes

    from . import native

    def copy(ptr, count, dtype):
        if not ptr or not count:
            return np.zeros(0, dtype)
        dt = np.dtype(dtype)
        raw = (ctypes.c_uint8 * (count * dt.itemsize)).from_address(ptr)
        return np.frombuffer(raw, dt, count).copy()

    with native.LoadedScene(path) as loaded:
        sd = loaded.data()
        params = np.frombuffer(bytes(sd.params), gt.RENDER_PARAMS, 1).copy()
        camera = np.frombuffer(bytes(sd.camera), gt.CAMERA, 1).copy()
        texels = copy(sd.texture_pixels, sd.texture_pixel_count, np.uint32)
        env = copy(sd.environment_pixels, sd.environment_pixel_count * 4, np.float32)
        data = SceneGpuData(
            params=params,
            camera=camera,
            spheres=copy(sd.spheres, sd.sphere_count, gt.SPHERE),
            triangles=copy(sd.triangles, sd.triangle_count, gt.TRIANGLE),
            triangle_attributes=copy(sd.triangle_attributes, sd.triangle_attribute_count, gt.TRIANGLE_ATTRIBUTES),
            materials=copy(sd.materials, sd.material_count, gt.MATERIAL),
            lights=copy(sd.lights, sd.light_count, gt.LIGHT),
            bvh_nodes=None,
            bvh_primitives=None,
            texture_pixels=texels if texels.size else None,
            environment_pixels=env.reshape(-1, 4) if env.size else None,
        )
        return data, loaded.exposure_stops()


def save_scene_json(scene: Scene, path, environment_file: Optional[str] = None) -> None:
    """Writes ``scene`` in the reference's JSON format (explicit triangles and spheres)."""
    mats = []
    for i, m in enumerate(scene.materials):
        name = m.name or f"m{i}"
        if m.kind == gt.DIFFUSE:
            mats.append({"name": name, "type": "diffuse", "albedo": list(map(float, m.albedo))})
        elif m.kind == gt.METAL:
            mats.append({"name": name, "type": "metal", "albedo": list(map(float, m.albedo)), "roughness": m.roughness})
        elif m.kind == gt.DIELECTRIC:
            mats.append({"name": name, "type": "dielectric", "ior": m.ior})
        else:
            mats.append({"name": name, "type": "emissive", "color": list(map(float, m.albedo)), "strength": m.strength})
    objs = []
    for c, r, mi in zip(scene.sphere_centers, scene.sphere_radii, scene.sphere_materials):
        objs.append({"type": "sphere", "center": [float(x) for x in c], "radius": float(r), "material": mats[mi]["name"]})
    for v, mi in zip(scene.triangles, scene.triangle_materials):
        objs.append({"type": "triangle", "vertices": [[float(x) for x in p] for p in v], "material": mats[mi]["name"]})
    if scene.background == gt.ENVIRONMENT:
        bg = {"type": "environment", "path": environment_file or "environment.hdr",
              "intensity": scene.environment.intensity, "rotation_degrees": scene.environment.rotation_degrees}
    else:
        bg = {gt.SKY: "sky", gt.BLACK: "black"}[scene.background]
    doc = {
        "camera": {"position": list(map(float, scene.camera_position)), "look_at": list(map(float, scene.camera_look_at)),
                   "up": list(map(float, scene.camera_up)), "fov_degrees": scene.fov_degrees},
        "render": {"width": scene.width, "height": scene.height, "samples": scene.samples,
                   "max_bounces": scene.max_bounces, "background": bg},
        "materials": mats,
        "objects": objs,
    }
    Path(path).write_text(json.dumps(doc) + "\n", encoding="utf-8")
