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
        y = np.arange(h, dtype=np.float64)
        sin_theta = np.sin(np.pi * (y + 0.5) / h)
        px = self.pixels.astype(np.float64)
        lum = 0.2126 * px[..., 0] + 0.7152 * px[..., 1] + 0.0722 * px[..., 2]
        weights = (lum * sin_theta[:, None] * float(np.float32(self.intensity))).reshape(-1)
        total = weights.sum()
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
    texture_pixels: Optional[np.ndarray] = None  # packed RGBA8 atlas (u32)

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
        if not weight > 0:
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
        if not weight > 0:
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
    mats = np.zeros(len(scene.materials), gt.MATERIAL)
    for i, m in enumerate(scene.materials):
        mats[i]["kind"] = m.kind
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
        p["environment_rotation_degrees"] = float(np.float32(env.rotation_degrees) % np.float32(360.0))
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
        texture_pixels=scene.texture_pixels,
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


def _load_gltf_meshes(path: Path):
    """Minimal glTF 2.0 reader for indexed triangle meshes with embedded or external buffers.

    Supports POSITION, NORMAL and TEXCOORD_0 float accessors, u8/u16/u32 indices and node
    matrices / TRS transforms, which is what the reference's benchmark fixtures and sample
    meshes use (crates/toaster-assets/src/gltf_loader.rs:11).
    """
    doc = json.loads(path.read_text(encoding="utf-8"))
    buffers = []
    for b in doc.get("buffers", []):
        uri = b["uri"]
        if uri.startswith("data:"):
            buffers.append(base64.b64decode(uri.split(",", 1)[1]))
        else:
            buffers.append((path.parent / uri).read_bytes())

    def accessor(i):
        a = doc["accessors"][i]
        view = doc["bufferViews"][a["bufferView"]]
        comp = {5126: ("<f4", 4), 5123: ("<u2", 2), 5125: ("<u4", 4), 5121: ("u1", 1)}[a["componentType"]]
        ncomp = {"SCALAR": 1, "VEC2": 2, "VEC3": 3, "VEC4": 4}[a["type"]]
        start = view.get("byteOffset", 0) + a.get("byteOffset", 0)
        stride = view.get("byteStride", comp[1] * ncomp)
        raw = buffers[view["buffer"]]
        count = a["count"]
        if stride == comp[1] * ncomp:
            arr = np.frombuffer(raw, dtype=comp[0], count=count * ncomp, offset=start).reshape(count, ncomp)
        else:
            arr = np.stack([np.frombuffer(raw, dtype=comp[0], count=ncomp, offset=start + k * stride) for k in range(count)])
        return arr

    def node_matrix(node):
        if "matrix" in node:
            return np.array(node["matrix"], dtype=np.float64).reshape(4, 4).T
        m = np.eye(4)
        t = node.get("translation", [0, 0, 0])
        r = node.get("rotation", [0, 0, 0, 1])
        s = node.get("scale", [1, 1, 1])
        x, y, z, w = r
        rot = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])
        m[:3, :3] = rot * np.array(s)[None, :]
        m[:3, 3] = t
        return m

    out = []
    scene_index = doc.get("scene", 0)
    roots = doc["scenes"][scene_index]["nodes"] if doc.get("scenes") else list(range(len(doc.get("nodes", []))))
    stack = [(r, np.eye(4)) for r in roots]
    while stack:
        ni, parent = stack.pop()
        node = doc["nodes"][ni]
        world = parent @ node_matrix(node)
        for c in node.get("children", []):
            stack.append((c, world))
        if "mesh" not in node:
            continue
        for prim in doc["meshes"][node["mesh"]]["primitives"]:
            if prim.get("mode", 4) != 4 or "indices" not in prim:
                continue
            pos = accessor(prim["attributes"]["POSITION"]).astype(np.float64)
            pos = (pos @ world[:3, :3].T + world[:3, 3]).astype(np.float32)
            idx = accessor(prim["indices"]).reshape(-1, 3).astype(np.int64)
            nrm = None
            if "NORMAL" in prim["attributes"]:
                n = accessor(prim["attributes"]["NORMAL"]).astype(np.float64)
                normal_matrix = np.linalg.inv(world[:3, :3]).T
                n = n @ normal_matrix.T
                n /= np.linalg.norm(n, axis=1, keepdims=True)
                nrm = n.astype(np.float32)[idx]
            uv = None
            if "TEXCOORD_0" in prim["attributes"]:
                uv = accessor(prim["attributes"]["TEXCOORD_0"]).astype(np.float32)[idx]
            out.append((pos[idx], nrm, uv))
    return out


def _read_hdr(path: Path) -> EnvironmentMap:
    """Radiance RGBE (.hdr) reader: flat and new-style run-length encoded scanlines."""
    data = path.read_bytes()
    pos = 0
    while True:
        end = data.index(b"\n", pos)
        line = data[pos:end].strip()
        pos = end + 1
        if line.startswith(b"-Y") or line.startswith(b"+Y"):
            parts = line.split()
            h, w = int(parts[1]), int(parts[3])
            break
    rgbe = np.zeros((h, w, 4), np.uint8)
    for y in range(h):
        if w >= 8 and w < 32768 and data[pos] == 2 and data[pos + 1] == 2 and (data[pos + 2] << 8 | data[pos + 3]) == w:
            pos += 4
            for c in range(4):
                x = 0
                while x < w:
                    count = data[pos]
                    pos += 1
                    if count > 128:
                        count -= 128
                        rgbe[y, x:x + count, c] = data[pos]
                        pos += 1
                    else:
                        rgbe[y, x:x + count, c] = np.frombuffer(data, np.uint8, count, pos)
                        pos += count
                    x += count
        else:
            rgbe[y] = np.frombuffer(data, np.uint8, w * 4, pos).reshape(w, 4)
            pos += w * 4
    e = rgbe[..., 3].astype(np.int32)
    scale = np.where(e > 0, np.ldexp(1.0, e - 136), 0.0)
    pixels = (rgbe[..., :3].astype(np.float64) * scale[..., None]).astype(np.float32)
    return EnvironmentMap(w, h, pixels)


def load_scene(path) -> Scene:
    """Loads the JSON subset of docs/scene_format.md used by the GPU path.

    Camera, render, materials (diffuse/metal/dielectric/emissive) and sphere / triangle / box /
    glTF mesh objects, with sky / black / environment backgrounds (Radiance .hdr maps).
    Physics, animation, triggers and textures are outside the GPU path and ignored.
    """
    path = Path(path)
    doc = json.loads(path.read_text(encoding="utf-8"))
    cam = doc["camera"]
    render = doc["render"]
    fov = cam.get("fov_degrees", cam.get("vertical_fov_degrees"))
    scene = Scene(
        camera_position=tuple(cam["position"]),
        camera_look_at=tuple(cam["look_at"]),
        camera_up=tuple(cam.get("up", [0.0, 1.0, 0.0])),
        fov_degrees=float(fov),
        width=int(render["width"]),
        height=int(render["height"]),
        samples=int(render.get("samples", render.get("samples_per_pixel", 1))),
        max_bounces=int(render["max_bounces"]),
    )
    bg = render.get("background", "sky")
    if isinstance(bg, str):
        scene.background = {"sky": gt.SKY, "black": gt.BLACK}[bg]
    else:
        if bg.get("type") != "environment":
            raise ValueError(f"unsupported background {bg!r}")
        env = _read_hdr((path.parent / bg["path"]).resolve())
        env.intensity = float(bg.get("intensity", 1.0))
        env.rotation_degrees = float(bg.get("rotation_degrees", 0.0))
        scene.environment = env
        scene.background = gt.ENVIRONMENT
    names = {}
    for m in doc["materials"]:
        kind = m["type"]
        if kind == "diffuse":
            mat = Material.diffuse(m["albedo"], m["name"])
        elif kind == "metal":
            mat = Material.metal(m["albedo"], m.get("roughness", 0.0), m["name"])
        elif kind == "dielectric":
            mat = Material.dielectric(m["ior"], m["name"])
        elif kind == "emissive":
            mat = Material.emissive(m["color"], m.get("strength", 1.0), m["name"])
        else:
            raise ValueError(f"unsupported material type {kind!r}")
        names[m["name"]] = len(scene.materials)
        scene.materials.append(mat)
    centers, radii, smat = [], [], []
    tris, tmat, tnorm, tuv, tflags = [], [], [], [], []
    for obj in doc["objects"]:
        kind = obj["type"]
        if kind == "sphere":
            centers.append(obj["center"])
            radii.append(obj["radius"])
            smat.append(names[obj["material"]])
        elif kind == "triangle":
            v = _f32(obj["vertices"])
            if not triangle_is_valid(v):
                raise ValueError("triangle vertices must be finite and non-collinear")
            tris.append(v)
            tmat.append(names[obj["material"]])
            tnorm.append(np.zeros((3, 3), np.float32))
            tuv.append(np.zeros((3, 2), np.float32))
            tflags.append(0)
        elif kind == "box":
            for v in box_triangles(obj["center"], obj["size"]):
                tris.append(v)
                tmat.append(names[obj["material"]])
                tnorm.append(np.zeros((3, 3), np.float32))
                tuv.append(np.zeros((3, 2), np.float32))
                tflags.append(0)
        elif kind == "mesh":
            if "material" not in obj:
                default = len(scene.materials)
                scene.materials.append(Material.diffuse((1.0, 1.0, 1.0), "__gltf_default"))
            mi = names[obj["material"]] if "material" in obj else default
            for pos, nrm, uv in _load_gltf_meshes((path.parent / obj["path"]).resolve()):
                for k in range(pos.shape[0]):
                    if not triangle_is_valid(pos[k]):
                        raise ValueError("triangle vertices must be finite and non-collinear")
                tris.extend(pos)
                tmat.extend([mi] * pos.shape[0])
                tnorm.extend(nrm if nrm is not None else np.zeros((pos.shape[0], 3, 3), np.float32))
                tuv.extend(uv if uv is not None else np.zeros((pos.shape[0], 3, 2), np.float32))
                flag = (1 if nrm is not None else 0) | (2 if uv is not None else 0)
                tflags.extend([flag] * pos.shape[0])
        else:
            raise ValueError(f"unsupported object type {kind!r}")
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
