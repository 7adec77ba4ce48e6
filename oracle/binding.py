"""TEST INFRASTRUCTURE ONLY: build recipe and ctypes binding of the CPU oracle (oracle.cpp)."""

from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SRC = HERE / "oracle.cpp"
BUILD_DIR = HERE / "_build"
LIB = BUILD_DIR / "liboracle.so"


def build(force: bool = False) -> Path:
    """g++ -O2 -ffp-contract=off -fopenmp (no fused multiply-adds: Rust f32 semantics)."""
    BUILD_DIR.mkdir(exist_ok=True)
    if force or not LIB.exists() or LIB.stat().st_mtime < SRC.stat().st_mtime:
        tmp = LIB.with_suffix(".so.tmp")
        subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-shared",
                        "-fPIC", str(SRC), "-o", str(tmp)], check=True)
        tmp.replace(LIB)
    return LIB


def library_path() -> Path:
    return LIB


_lib = None


def _load():
    global _lib
    if _lib is None:
        build()
        lib = ctypes.CDLL(str(LIB))
        vp, u32, u64, f32, i32 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_float, ctypes.c_int
        lib.orc_scene_create.restype = vp
        lib.orc_scene_create.argtypes = [vp, u32, vp, u32, vp, vp, u32, vp, u32, vp, vp, u32, u32, f32, f32, u32]
        lib.orc_scene_destroy.argtypes = [vp]
        lib.orc_bvh_node_count.argtypes = [vp]
        lib.orc_bvh_node_count.restype = u32
        lib.orc_bvh_prim_count.argtypes = [vp]
        lib.orc_bvh_prim_count.restype = u32
        lib.orc_bvh_export.argtypes = [vp, vp, vp, vp]
        lib.orc_trace_closest.argtypes = [vp, vp, u64, f32, vp, vp, vp, vp, i32]
        lib.orc_ray_color.argtypes = [vp, vp, u64, u32, i32, f32, u64, vp]
        lib.orc_render.argtypes = [vp, u64, u32, u32, u32, i32, vp, vp, vp]
        lib.orc_camera_basis.argtypes = [vp, vp, vp, f32, f32, vp]
        lib.orc_camera_basis.restype = i32
        lib.orc_scatter.argtypes = [vp, vp, vp, u64, vp]
        lib.orc_scatter.restype = i32
        lib.orc_refract.argtypes = [vp, vp, f32, vp]
        lib.orc_reflectance.argtypes = [f32, f32]
        lib.orc_reflectance.restype = f32
        lib.orc_power_heuristic.argtypes = [f32, f32]
        lib.orc_power_heuristic.restype = f32
        lib.orc_direct.argtypes = [vp, vp, vp, i32, u64, u32, vp]
        lib.orc_lights.argtypes = [vp, vp, vp]
        lib.orc_lights.restype = u32
        lib.orc_sample_lights.argtypes = [vp, u64, u32, vp]
        lib.orc_env_create.restype = vp
        lib.orc_env_create.argtypes = [u32, u32, vp, f32, f32]
        lib.orc_env_destroy.argtypes = [vp]
        lib.orc_env_cdf.argtypes = [vp, vp]
        lib.orc_env_rotation.argtypes = [vp]
        lib.orc_env_rotation.restype = f32
        lib.orc_env_lookup.argtypes = [vp, vp, u32, vp, vp]
        lib.orc_env_sample.argtypes = [vp, vp, u32, vp]
        lib.orc_env_direction_to_uv.argtypes = [vp, vp, vp]
        lib.orc_env_direction_to_uv.restype = i32
        lib.orc_num_threads.restype = i32
        lib.orc_aabb_intersects.argtypes = [vp, vp, vp, vp, f32, f32]
        lib.orc_aabb_intersects.restype = i32
        lib.orc_display_rgba8.argtypes = [vp, u64, f32, vp]
        _lib = lib
    return _lib


class _Settings(ctypes.Structure):
    _fields_ = [
        ("camera_position", ctypes.c_float * 3),
        ("camera_look_at", ctypes.c_float * 3),
        ("camera_up", ctypes.c_float * 3),
        ("fov_degrees", ctypes.c_float),
        ("width", ctypes.c_uint32),
        ("height", ctypes.c_uint32),
        ("samples", ctypes.c_uint32),
        ("max_bounces", ctypes.c_uint32),
        ("background", ctypes.c_uint32),
    ]


def _c(a, dtype=np.float32):
    return np.ascontiguousarray(a, dtype)


class Oracle:
    """CPU scene: hierarchy, lights and integrator of the reference CPU renderer."""

    def __init__(self, scene, max_leaf: int = 4):
        """``scene`` is a ``toaster_b200.scene.Scene`` (its packed records are what the oracle reads)."""
        from toaster_b200.scene import scene_to_gpu

        self.lib = _load()
        self.scene = scene
        data = scene_to_gpu(scene)
        self._keep = [data]
        st = _Settings()
        st.camera_position[:] = [float(x) for x in scene.camera_position]
        st.camera_look_at[:] = [float(x) for x in scene.camera_look_at]
        st.camera_up[:] = [float(x) for x in scene.camera_up]
        st.fov_degrees = scene.fov_degrees
        st.width, st.height, st.samples, st.max_bounces = scene.width, scene.height, scene.samples, scene.max_bounces
        st.background = scene.background
        env = scene.environment
        env_rgb = None
        if env is not None:
            env_rgb = _c(env.pixels.reshape(-1, 3))
            self._keep.append(env_rgb)

        def p(a):
            return None if a is None or len(a) == 0 else a.ctypes.data

        self.handle = self.lib.orc_scene_create(
            p(data.spheres), len(data.spheres), p(data.triangles), len(data.triangles), p(data.triangle_attributes),
            p(data.materials), len(data.materials), p(data.texture_pixels),
            0 if data.texture_pixels is None else len(data.texture_pixels), ctypes.byref(st),
            None if env_rgb is None else env_rgb.ctypes.data, 0 if env is None else env.width,
            0 if env is None else env.height, 0.0 if env is None else env.intensity,
            0.0 if env is None else env.rotation_degrees, max_leaf)

    def close(self):
        if self.handle:
            self.lib.orc_scene_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def bvh(self):
        """(bounds (n, 8) f32, links (n, 2) u32, prims (m, 2) u32) in GpuBvhNode order."""
        n = self.lib.orc_bvh_node_count(self.handle)
        m = self.lib.orc_bvh_prim_count(self.handle)
        bounds = np.zeros((n, 8), np.float32)
        links = np.zeros((n, 2), np.uint32)
        prims = np.zeros((m, 2), np.uint32)
        self.lib.orc_bvh_export(self.handle, bounds.ctypes.data, links.ctypes.data, prims.ctypes.data)
        return bounds, links, prims

    def trace_closest(self, rays, tmin=0.001, with_info=False, with_counts=False, linear=False):
        rays = _c(rays).reshape(-1, 6)
        n = rays.shape[0]
        prim = np.empty(n, np.uint32)
        t = np.empty(n, np.float32)
        info = np.empty((n, 8), np.float32) if with_info else None
        counts = np.zeros(6, np.uint64) if with_counts else None
        self.lib.orc_trace_closest(self.handle, rays.ctypes.data, n, tmin, prim.ctypes.data, t.ctypes.data,
                                   None if info is None else info.ctypes.data,
                                   None if counts is None else counts.ctypes.data, 1 if linear else 0)
        out = [prim, t]
        if with_info:
            out.append(info)
        if with_counts:
            out.append(counts)
        return tuple(out)

    def ray_color(self, rays, depth, include_emission=True, bsdf_pdf=None, seed=1):
        rays = _c(rays).reshape(-1, 6)
        out = np.empty((rays.shape[0], 3), np.float32)
        self.lib.orc_ray_color(self.handle, rays.ctypes.data, rays.shape[0], depth, 1 if include_emission else 0,
                               -1.0 if bsdf_pdf is None else float(bsdf_pdf), seed, out.ctypes.data)
        return out

    def render(self, seed=0, rows=None, row_step=1, threads=0, moments=False, counts=False):
        """Per-pixel mean (rows, width, 3), optional sums of squares and ray counters."""
        r0, r1 = (0, self.scene.height) if rows is None else rows
        nrows = len(range(r0, r1, row_step))
        w = self.scene.width
        mean = np.zeros((nrows, w, 3), np.float32)
        sq = np.zeros((nrows, w, 3), np.float64) if moments else None
        cnt = np.zeros(6, np.uint64) if counts else None
        self.lib.orc_render(self.handle, seed, r0, r1, row_step, threads, mean.ctypes.data,
                            None if sq is None else sq.ctypes.data, None if cnt is None else cnt.ctypes.data)
        return mean, sq, cnt

    def lights(self):
        n = len(self.scene.materials) + self.scene.triangle_count + self.scene.sphere_count
        out = np.zeros((max(n, 1), 4), np.float32)
        total = ctypes.c_float()
        k = self.lib.orc_lights(self.handle, out.ctypes.data, ctypes.byref(total))
        return out[:k], float(total.value)

    def sample_lights(self, n, seed=0):
        out = np.zeros((n, 10), np.float32)
        self.lib.orc_sample_lights(self.handle, seed, n, out.ctypes.data)
        return out

    def direct(self, point, normal, albedo, which, draws=1, seed=0):
        hit = _c(list(point) + list(normal))
        out = np.zeros(3, np.float32)
        alb = _c(albedo)
        self.lib.orc_direct(self.handle, hit.ctypes.data, alb.ctypes.data, which, seed, draws, out.ctypes.data)
        return out


class OracleEnvironment:
    """environment.rs EnvironmentMap restated (flat CDF, bilinear lookup, solid-angle pdf)."""

    def __init__(self, width, height, rgb, intensity=1.0, rotation=0.0):
        self.lib = _load()
        self.rgb = _c(rgb).reshape(-1, 3)
        self.width, self.height = width, height
        self.handle = self.lib.orc_env_create(width, height, self.rgb.ctypes.data, intensity, rotation)

    def __del__(self):
        try:
            self.lib.orc_env_destroy(self.handle)
        except Exception:
            pass

    def cdf(self):
        out = np.zeros(self.width * self.height, np.float32)
        self.lib.orc_env_cdf(self.handle, out.ctypes.data)
        return out

    def rotation(self):
        return self.lib.orc_env_rotation(self.handle)

    def lookup(self, dirs):
        dirs = _c(dirs).reshape(-1, 3)
        rgb = np.zeros((dirs.shape[0], 3), np.float32)
        pdf = np.zeros(dirs.shape[0], np.float32)
        self.lib.orc_env_lookup(self.handle, dirs.ctypes.data, dirs.shape[0], rgb.ctypes.data, pdf.ctypes.data)
        return rgb, pdf

    def sample(self, uniforms):
        u = _c(uniforms).reshape(-1, 3)
        out = np.zeros((u.shape[0], 8), np.float32)
        self.lib.orc_env_sample(self.handle, u.ctypes.data, u.shape[0], out.ctypes.data)
        return out

    def direction_to_uv(self, d):
        out = np.zeros(3, np.float32)
        dd = _c(d)
        ok = self.lib.orc_env_direction_to_uv(self.handle, dd.ctypes.data, out.ctypes.data)
        return tuple(out) if ok else None


def camera_basis(position, look_at, up, fov, aspect):
    lib = _load()
    out = np.zeros(12, np.float32)
    args = [_c(position), _c(look_at), _c(up)]
    ok = lib.orc_camera_basis(args[0].ctypes.data, args[1].ctypes.data, args[2].ctypes.data, fov, aspect,
                              out.ctypes.data)
    return out.reshape(4, 3) if ok else None


def scatter(in_dir, point, normal, front_face, kind, albedo=(1, 1, 1), roughness=0.0, ior=1.5, seed=0):
    lib = _load()
    hit = _c(list(point) + list(normal) + [1.0 if front_face else 0.0])
    mat = _c([kind] + list(albedo) + [roughness, ior])
    out = np.zeros(7, np.float32)
    d = _c(in_dir)
    ok = lib.orc_scatter(d.ctypes.data, hit.ctypes.data, mat.ctypes.data, seed, out.ctypes.data)
    return out if ok else None


def refract(d, n, ratio):
    lib = _load()
    out = np.zeros(3, np.float32)
    dd, nn = _c(d), _c(n)
    lib.orc_refract(dd.ctypes.data, nn.ctypes.data, ratio, out.ctypes.data)
    return out


def reflectance(cosine, ratio):
    return _load().orc_reflectance(cosine, ratio)


def power_heuristic(a, b):
    return _load().orc_power_heuristic(a, b)


def num_threads():
    return _load().orc_num_threads()


def aabb_intersects(mn, mx, origin, inv, tmin, tmax):
    lib = _load()
    args = [_c(mn), _c(mx), _c(origin), _c(inv)]
    return bool(lib.orc_aabb_intersects(args[0].ctypes.data, args[1].ctypes.data, args[2].ctypes.data,
                                        args[3].ctypes.data, tmin, tmax))


def display_rgba8(rgba, exposure_stops=0.0):
    """Linear-HDR float4 pixels -> display RGBA8 (color.rs:42-74, image_output.rs:57-88)."""
    lib = _load()
    px = _c(rgba).reshape(-1, 4)
    out = np.zeros((px.shape[0], 4), np.uint8)
    lib.orc_display_rgba8(px.ctypes.data, px.shape[0], exposure_stops, out.ctypes.data)
    return out
