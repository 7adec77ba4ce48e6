"""ctypes binding of the C ABI in include/toaster_cuda.h.

The shared library is built in-tree (``toaster_b200/lib/libtoaster_cuda.so``) by
``toaster_b200.build``. There is no fallback: importing a GPU entry point without the library
raises, and creating a context without an sm_100 device fails with the library's message.
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

from . import gpu_types as gt

LIB_DIR = Path(__file__).resolve().parent / "lib"
LIB_PATH = LIB_DIR / "libtoaster_cuda.so"

TC_OK = 0
TC_ERR_INVALID = -1
TC_ERR_CUDA = -2
TC_ERR_NO_DEVICE = -3
TC_ERR_STATE = -4
TC_ERR_DEVICE_STATUS = -5
TC_MISS = 0xFFFFFFFF
TC_PRIM_TRIANGLE_BIT = 0x80000000

# Exported symbols declared in include/toaster_cuda.h.
EXPORTED_SYMBOLS = (
    "tc_abi_version",
    "tc_last_error",
    "tc_create",
    "tc_destroy",
    "tc_set_stream",
    "tc_upload_scene",
    "tc_set_camera",
    "tc_render",
    "tc_readback",
    "tc_readback_sums",
    "tc_trace_closest",
    "tc_trace_closest_device_async",
    "tc_get_stats",
    "tc_build_bvh_host",
    "tc_record_sizes",
    "tc_umma_selftest",
    "tc_probe_cache_read",
    "tc_set_triangle_test",
    "tc_probe_last_error",
    "tc_guide_set_params",
    "tc_guide_get_params",
    "tc_guide_infer",
    "tc_guide_loss_grad",
    "tc_guide_adam_step",
    "tc_guide_train",
    "tc_render_no_alloc",
    "tc_guide_train_recorded",
    "tc_update_geometry",
    "tc_readback_rgba8",
    "tc_display_rgba8_async",
    "tc_render_batch",
    "tc_guide_recorded_samples",
    "tc_animation_create",
    "tc_animation_frame",
    "tc_animation_destroy",
    "tc_autotune",
    "tc_set_hierarchy_build",
    "tc_encode_jpeg",
    "tc_scene_load",
    "tc_loaded_scene_data",
    "tc_loaded_scene_display",
    "tc_loaded_scene_free",
)

GUIDE_PARAMS = 15584


class TcError(RuntimeError):
    """A tc_* call returned a nonzero status."""

    def __init__(self, code: int, message: str):
        super().__init__(f"toaster_cuda error {code}: {message}")
        self.code = code


class SceneChanges(ctypes.Structure):
    """tc_scene_changes: toaster_scene::SceneChanges (evaluation.rs:9-18)."""

    _fields_ = [("camera", ctypes.c_uint32), ("spheres", ctypes.c_uint32), ("triangles", ctypes.c_uint32),
                ("emissive_geometry", ctypes.c_uint32)]


class SceneData(ctypes.Structure):
    _fields_ = [
        ("params", ctypes.c_uint8 * 96),
        ("camera", ctypes.c_uint8 * 64),
        ("spheres", ctypes.c_void_p),
        ("sphere_count", ctypes.c_size_t),
        ("triangles", ctypes.c_void_p),
        ("triangle_count", ctypes.c_size_t),
        ("triangle_attributes", ctypes.c_void_p),
        ("triangle_attribute_count", ctypes.c_size_t),
        ("materials", ctypes.c_void_p),
        ("material_count", ctypes.c_size_t),
        ("lights", ctypes.c_void_p),
        ("light_count", ctypes.c_size_t),
        ("bvh_nodes", ctypes.c_void_p),
        ("bvh_node_count", ctypes.c_size_t),
        ("bvh_primitives", ctypes.c_void_p),
        ("bvh_primitive_count", ctypes.c_size_t),
        ("texture_pixels", ctypes.c_void_p),
        ("texture_pixel_count", ctypes.c_size_t),
        ("environment_pixels", ctypes.c_void_p),
        ("environment_pixel_count", ctypes.c_size_t),
    ]


class RenderOptions(ctypes.Structure):
    _fields_ = [
        ("block_size", ctypes.c_uint32),
        ("samples_per_item", ctypes.c_uint32),
        ("keep_moments", ctypes.c_uint32),
        ("guiding", ctypes.c_uint32),
        ("guide_record", ctypes.c_uint32),
        ("wave_paths", ctypes.c_uint32),
        ("short_stack", ctypes.c_uint32),
        ("refill_lanes", ctypes.c_uint32),
        ("guide_fraction", ctypes.c_float),
        ("schedule", ctypes.c_uint32),
        ("ray_sort", ctypes.c_uint32),
        ("phase_timing", ctypes.c_uint32),
    ]


SCHEDULES = {"auto": 0, "megakernel": 1, "wavefront": 2}


class TuneResult(ctypes.Structure):
    _fields_ = [("best", RenderOptions), ("best_kernel_ms", ctypes.c_float), ("best_mpaths_per_s", ctypes.c_float),
                ("candidates", ctypes.c_uint32), ("probe_samples", ctypes.c_uint32)]


class Stats(ctypes.Structure):
    _fields_ = [
        ("paths", ctypes.c_uint64),
        ("rays", ctypes.c_uint64),
        ("extension_rays", ctypes.c_uint64),
        ("shadow_rays", ctypes.c_uint64),
        ("kernel_ms", ctypes.c_float),
        ("total_ms", ctypes.c_float),
        ("bvh_depth", ctypes.c_uint32),
        ("status_flags", ctypes.c_uint32),
        ("kernel_launches", ctypes.c_uint32),
        ("trace_ms", ctypes.c_float),
        ("logic_ms", ctypes.c_float),
        ("shade_ms", ctypes.c_float),
        ("guide_ms", ctypes.c_float),
        ("wf_iterations", ctypes.c_uint32),
    ]


_LIB = None


def load_library(path: os.PathLike | None = None) -> ctypes.CDLL:
    """Loads (once) and returns the CUDA library; raises if it has not been built."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = Path(path) if path is not None else LIB_PATH
    if not p.exists():
        raise RuntimeError(f"{p} is missing: build it with `python -m toaster_b200.build` (no CPU fallback exists)")
    lib = ctypes.CDLL(str(p))
    vp, sz, u32, i32, f32 = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint32, ctypes.c_int, ctypes.c_float
    lib.tc_abi_version.restype = i32
    lib.tc_last_error.argtypes = [vp]
    lib.tc_last_error.restype = ctypes.c_char_p
    lib.tc_create.argtypes = [i32, ctypes.POINTER(vp)]
    lib.tc_destroy.argtypes = [vp]
    lib.tc_set_stream.argtypes = [vp, vp]
    lib.tc_upload_scene.argtypes = [vp, ctypes.POINTER(SceneData)]
    lib.tc_set_camera.argtypes = [vp, vp]
    lib.tc_render.argtypes = [vp, vp, ctypes.POINTER(RenderOptions)]
    lib.tc_readback.argtypes = [vp, vp, sz]
    lib.tc_readback_sums.argtypes = [vp, vp, vp, sz, ctypes.POINTER(u32)]
    lib.tc_trace_closest.argtypes = [vp, vp, sz, f32, vp, vp]
    lib.tc_trace_closest_device_async.argtypes = [vp, vp, sz, f32, vp, vp, vp]
    lib.tc_get_stats.argtypes = [vp, ctypes.POINTER(Stats)]
    lib.tc_build_bvh_host.argtypes = [vp, sz, vp, sz, vp, sz, vp, sz]
    lib.tc_build_bvh_host.restype = ctypes.c_long
    lib.tc_record_sizes.argtypes = [ctypes.POINTER(u32), sz]
    lib.tc_umma_selftest.argtypes = [vp, vp, vp, i32, i32, i32, i32]
    lib.tc_probe_cache_read.argtypes = [i32, sz, i32, ctypes.POINTER(ctypes.c_double)]
    lib.tc_probe_last_error.restype = ctypes.c_char_p
    lib.tc_guide_set_params.argtypes = [vp, vp, vp]
    lib.tc_guide_get_params.argtypes = [vp, vp]
    lib.tc_guide_infer.argtypes = [vp, vp, sz, vp]
    lib.tc_guide_loss_grad.argtypes = [vp, vp, sz, vp, vp]
    lib.tc_guide_adam_step.argtypes = [vp, f32]
    lib.tc_render_no_alloc.argtypes = [vp, vp, vp, sz, vp]
    lib.tc_guide_train_recorded.argtypes = [vp, u32, u32, f32, ctypes.c_uint64, vp, ctypes.POINTER(u32)]
    lib.tc_guide_train.argtypes = [vp, vp, sz, u32, u32, f32, ctypes.c_uint64, vp]
    lib.tc_update_geometry.argtypes = [vp, ctypes.POINTER(SceneData), ctypes.POINTER(SceneChanges)]
    lib.tc_readback_rgba8.argtypes = [vp, f32, vp, sz]
    lib.tc_display_rgba8_async.argtypes = [vp, f32, vp, sz, vp]
    lib.tc_render_batch.argtypes = [ctypes.POINTER(vp), vp, sz, ctypes.POINTER(RenderOptions)]
    lib.tc_guide_recorded_samples.argtypes = [vp, vp, sz, ctypes.POINTER(u32)]
    lib.tc_animation_create.argtypes = [vp, ctypes.POINTER(SceneData), vp, ctypes.POINTER(RenderOptions), f32, u32,
                                        ctypes.POINTER(vp)]
    lib.tc_animation_frame.argtypes = [vp, ctypes.POINTER(SceneData), u32, vp, sz]
    lib.tc_animation_destroy.argtypes = [vp]
    lib.tc_autotune.argtypes = [vp, vp, ctypes.POINTER(RenderOptions), u32, ctypes.POINTER(TuneResult)]
    lib.tc_set_hierarchy_build.argtypes = [vp, i32]
    lib.tc_set_triangle_test.argtypes = [vp, i32]
    lib.tc_encode_jpeg.argtypes = [vp, u32, f32, vp, sz, ctypes.POINTER(sz)]
    lib.tc_scene_load.argtypes = [ctypes.c_char_p, ctypes.POINTER(vp), ctypes.c_char_p, sz]
    lib.tc_loaded_scene_data.argtypes = [vp]
    lib.tc_loaded_scene_data.restype = ctypes.POINTER(SceneData)
    lib.tc_loaded_scene_display.argtypes = [vp, ctypes.POINTER(f32)]
    lib.tc_loaded_scene_free.argtypes = [vp]
    for name in EXPORTED_SYMBOLS:
        if not hasattr(lib, name):
            raise RuntimeError(f"{p} does not export {name}")
    if path is None:
        _LIB = lib
    return lib


def _ptr(a: np.ndarray | None):
    return None if a is None or a.size == 0 else a.ctypes.data


def check(lib, ctx, code: int) -> None:
    if code != TC_OK:
        msg = lib.tc_last_error(ctx)
        raise TcError(code, msg.decode() if msg else "")


def build_bvh_host(spheres: np.ndarray, triangles: np.ndarray):
    """Reference-layout hierarchy built by the library's host builder (no GPU needed)."""
    lib = load_library()
    spheres = np.ascontiguousarray(spheres, gt.SPHERE)
    triangles = np.ascontiguousarray(triangles, gt.TRIANGLE)
    n = len(spheres) + len(triangles)
    nodes = np.zeros(max(2 * n - 1, 1), gt.BVH_NODE)
    prims = np.zeros(max(n, 1), gt.PRIMITIVE_REF)
    count = lib.tc_build_bvh_host(_ptr(spheres), len(spheres), _ptr(triangles), len(triangles),
                                  nodes.ctypes.data, len(nodes), prims.ctypes.data, len(prims))
    if count < 0:
        raise TcError(int(count), lib.tc_last_error(None).decode())
    return nodes[:count].copy(), prims[:n].copy()


def umma_selftest(a: np.ndarray, b: np.ndarray, a_mn_major: bool = False, b_mn_major: bool = False) -> np.ndarray:
    """D = A @ B.T on the tensor cores for bf16 bit patterns a (128 x k) and b (n x k)."""
    lib = load_library()
    a = np.ascontiguousarray(a, np.uint16)
    b = np.ascontiguousarray(b, np.uint16)
    n, k = b.shape
    d = np.zeros((128, n), np.float32)
    check(lib, None, lib.tc_umma_selftest(a.ctypes.data, b.ctypes.data, d.ctypes.data, n, k, int(a_mn_major),
                                          int(b_mn_major)))
    return d


def probe_cache_read(device: int = 0, nbytes: int = 64 << 20, passes: int = 50) -> float:
    """Read bandwidth in GB/s of a device buffer of `nbytes` streamed by every SM with loads that
    bypass L1: L2 bandwidth for buffers smaller than L2, HBM for larger ones."""
    lib = load_library()
    out = ctypes.c_double(0.0)
    code = lib.tc_probe_cache_read(device, nbytes, passes, ctypes.byref(out))
    if code != 0:
        raise TcError(code, lib.tc_probe_last_error().decode())
    return out.value


class LoadedScene:
    """A scene file loaded and packed by the library (tc_scene_load); frees itself on close."""

    def __init__(self, path: os.PathLike):
        self._handle = None
        self._lib = load_library()
        handle = ctypes.c_void_p()
        err = ctypes.create_string_buffer(4096)
        code = self._lib.tc_scene_load(os.fsencode(path), ctypes.byref(handle), err, len(err))
        if code != TC_OK:
            raise TcError(code, err.value.decode(errors="replace"))
        self._handle = handle

    def data(self):
        """The packed records (a SceneData view valid until close())."""
        return self._lib.tc_loaded_scene_data(self._handle).contents

    def exposure_stops(self) -> float:
        out = ctypes.c_float()
        check(self._lib, None, self._lib.tc_loaded_scene_display(self._handle, ctypes.byref(out)))
        return float(out.value)

    def close(self) -> None:
        if getattr(self, "_handle", None):
            self._lib.tc_loaded_scene_free(self._handle)
            self._handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        self.close()


def record_sizes() -> list:
    lib = load_library()
    out = (ctypes.c_uint32 * 9)()
    check(lib, None, lib.tc_record_sizes(out, 9))
    return list(out)
