"""Host-side renderer API over the CUDA library: one ``GpuRenderer`` per context, one call per C-ABI
entry point, plus batched launches and animation graphs.

``progressive_batch`` and ``render_frame_seed`` keep the frame-seed and progressive batching rules
of crates/toaster-gpu/src/path_tracer.rs:892-923; the reference's public entry points built on
them (animation, video, progressive and benchmark renders) are in ``frames``. Images are
linear-HDR float4 (alpha = 1), row-major, y down.
"""

from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np

from . import gpu_types as gt
from . import native
from .scene import Scene, SceneGpuData, scene_to_gpu


class Animation:
    """Animated frames replayed through one captured CUDA graph (tc_animation_*).

    The renderer must hold the uploaded first frame; every frame passed to ``frame`` must keep its
    primitive counts. Frames are independent renders seeded by their frame index."""

    def __init__(self, renderer: "GpuRenderer", first: SceneGpuData, samples: Optional[int] = None,
                 max_bounces: Optional[int] = None, exposure_stops: float = 0.0, guiding: bool = False,
                 update_lights: bool = False, block_size: int = 0, wave_paths: int = 0, refill_lanes: int = 0,
                 rebuild: bool = False):
        self._r = renderer
        self._lib = renderer._lib
        self._h = None
        p = first.params.copy()
        if samples is not None:
            p["samples"] = samples
        if max_bounces is not None:
            p["max_bounces"] = max_bounces
        p["accumulated_samples"] = 0
        self.width, self.height = int(p["width"][0]), int(p["height"][0])
        opts = native.RenderOptions()
        opts.guiding = 1 if guiding else 0
        opts.block_size = block_size
        opts.wave_paths = wave_paths
        opts.refill_lanes = refill_lanes
        sd, keep = GpuRenderer._scene_struct(first)
        h = ctypes.c_void_p()
        renderer._check(self._lib.tc_animation_create(renderer._ctx, ctypes.byref(sd), p.ctypes.data, ctypes.byref(opts),
                                                      float(exposure_stops), int(update_lights) | (2 if rebuild else 0),
                                                      ctypes.byref(h)))
        self._h = h

    def frame(self, data: SceneGpuData, frame_index: int, out: Optional[np.ndarray] = None) -> np.ndarray:
        if out is None:
            out = np.empty((self.height, self.width, 4), np.uint8)
        sd, keep = GpuRenderer._scene_struct(data)
        self._r._check(self._lib.tc_animation_frame(self._h, ctypes.byref(sd), frame_index, out.ctypes.data, out.nbytes))
        self._r.width, self._r.height = self.width, self.height
        return out

    def close(self) -> None:
        if self._h:
            self._lib.tc_animation_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def render_batch(renderers, samples=None, frame_index: int = 0, accumulate: bool = False, block_size: int = 0,
                 samples_per_item: int = 0, short_stack: int = 0, refill_lanes: int = 0, guiding: bool = False,
                 guide_fraction: float = 0.0, wave_paths: int = 0, schedule: str = "auto") -> dict:
    """The uploaded scenes of several renderers (same device) in one call: frames too small to
    fill the GPU share one persistent launch; with ``schedule`` "auto" a frame of at least 2^20
    paths gets a wavefront call of its own ("megakernel": every frame in the shared launch,
    "wavefront": every frame in a call of its own).

    ``samples`` may be one count or one per renderer (one count for the shared launch's frames
    when ``guiding``).
    ``guiding``: every renderer needs guide parameters; each frame's queries go to its own
    network, in rounds of (batched path kernel, per-frame inference, batched resume). Returns the
    batch's stats (paths, rays, kernel and total milliseconds)."""
    if not renderers:
        raise ValueError("empty batch")
    lib = renderers[0]._lib
    n = len(renderers)
    spp = samples if isinstance(samples, (list, tuple)) else [samples] * n
    params = np.zeros(n, gt.RENDER_PARAMS)
    for i, r in enumerate(renderers):
        if r._params is None:
            raise RuntimeError("render before upload")
        p = r._params.copy()
        if spp[i] is not None:
            p["samples"] = spp[i]
        p["frame_index"] = frame_index
        p["accumulated_samples"] = r.accumulated if accumulate else 0
        params[i] = p[0] if p.shape else p
    ctxs = (ctypes.c_void_p * n)(*[r._ctx for r in renderers])
    opts = native.RenderOptions()
    opts.block_size = block_size
    opts.samples_per_item = samples_per_item
    opts.short_stack = short_stack
    opts.refill_lanes = refill_lanes
    opts.guiding = 1 if guiding else 0
    opts.guide_fraction = guide_fraction
    opts.wave_paths = wave_paths
    opts.schedule = native.SCHEDULES[schedule]
    native.check(lib, renderers[0]._ctx, lib.tc_render_batch(ctxs, params.ctypes.data, n, ctypes.byref(opts)))
    for i, r in enumerate(renderers):
        r.width, r.height = int(params[i]["width"]), int(params[i]["height"])
        r.accumulated = (r.accumulated if accumulate else 0) + int(params[i]["samples"])
    return renderers[0].stats()


def progressive_batch(requested_samples: int, accumulated_samples: int, target_samples: int) -> Optional[int]:
    """Next batch clamped to the remaining target, or None when complete (path_tracer.rs:900-923)."""
    if requested_samples <= 0:
        raise ValueError("sample batch must be greater than zero")
    if target_samples <= 0:
        raise ValueError("sample target must be greater than zero")
    if accumulated_samples > target_samples:
        raise ValueError("accumulated samples exceed the progressive target")
    if accumulated_samples == target_samples:
        return None
    return min(requested_samples, target_samples - accumulated_samples)


def render_frame_seed(frame: int, static_independent: bool) -> int:
    """Benchmark frames reuse seed 0; animated frames use their index (path_tracer.rs:892-897)."""
    return 0 if static_independent else frame


class GpuRenderer:
    """One CUDA context (device buffers + stream) holding one uploaded scene."""

    def __init__(self, device: int = 0):
        self._lib = native.load_library()
        ctx = ctypes.c_void_p()
        native.check(self._lib, None, self._lib.tc_create(device, ctypes.byref(ctx)))
        self._ctx = ctx
        self.width = 0
        self.height = 0
        self.accumulated = 0
        self._params = None

    def close(self) -> None:
        if self._ctx:
            self._lib.tc_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, code: int) -> None:
        native.check(self._lib, self._ctx, code)

    @staticmethod
    def _scene_struct(data: SceneGpuData):
        """tc_scene_data over the packed arrays; the arrays kept alive are returned beside it."""
        sd = native.SceneData()
        ctypes.memmove(sd.params, data.params.ctypes.data, 96)
        ctypes.memmove(sd.camera, data.camera.ctypes.data, 64)
        keep = []

        def arr(a, dtype):
            if a is None or len(a) == 0:
                return None, 0
            a = np.ascontiguousarray(a, dtype)
            keep.append(a)
            return a.ctypes.data, len(a)

        sd.spheres, sd.sphere_count = arr(data.spheres, gt.SPHERE)
        sd.triangles, sd.triangle_count = arr(data.triangles, gt.TRIANGLE)
        sd.triangle_attributes, sd.triangle_attribute_count = arr(data.triangle_attributes, gt.TRIANGLE_ATTRIBUTES)
        sd.materials, sd.material_count = arr(data.materials, gt.MATERIAL)
        sd.lights, sd.light_count = arr(data.lights, gt.LIGHT)
        sd.bvh_nodes, sd.bvh_node_count = arr(data.bvh_nodes, gt.BVH_NODE)
        sd.bvh_primitives, sd.bvh_primitive_count = arr(data.bvh_primitives, gt.PRIMITIVE_REF)
        sd.texture_pixels, sd.texture_pixel_count = arr(data.texture_pixels, np.uint32)
        if data.environment_pixels is not None:
            env = np.ascontiguousarray(data.environment_pixels, np.float32).reshape(-1, 4)
            keep.append(env)
            sd.environment_pixels, sd.environment_pixel_count = env.ctypes.data, env.shape[0]
        return sd, keep

    def upload(self, data: SceneGpuData) -> None:
        """Copies packed scene records to the device and builds hierarchy and sampling tables."""
        sd, keep = self._scene_struct(data)
        self._check(self._lib.tc_upload_scene(self._ctx, ctypes.byref(sd)))
        self._params = data.params.copy()
        self.accumulated = 0

    def upload_file(self, path) -> float:
        """Loads a scene file with the native loader (tc_scene_load) and uploads its records
        straight from the library's buffers; returns the scene's display exposure in stops."""
        with native.LoadedScene(path) as loaded:
            sd = loaded.data()
            self._check(self._lib.tc_upload_scene(self._ctx, ctypes.byref(sd)))
            self._params = np.frombuffer(bytes(sd.params), gt.RENDER_PARAMS, 1).copy()
            self.accumulated = 0
            return loaded.exposure_stops()

    def update_geometry(self, data: SceneGpuData, camera: bool = False, spheres: bool = True, triangles: bool = True,
                        emissive_geometry: bool = False) -> None:
        """Per-frame update: copies changed geometry and refits the hierarchy on the device."""
        sd, keep = self._scene_struct(data)
        ch = native.SceneChanges(int(camera), int(spheres), int(triangles), int(emissive_geometry))
        self._check(self._lib.tc_update_geometry(self._ctx, ctypes.byref(sd), ctypes.byref(ch)))

    def set_hierarchy_build(self, mode: str) -> None:
        """Where uploads build the hierarchy: "auto", "host" or "device"."""
        self._check(self._lib.tc_set_hierarchy_build(self._ctx, {"auto": 0, "host": 1, "device": 2}[mode]))

    def set_triangle_test(self, test: str) -> None:
        """Triangle test of later uploads: "moller_trumbore" (the reference's, bit-exact hits) or
        "watertight" (no ray slips between triangles sharing an edge; traced by trace_closest and
        wavefront renders)."""
        self._check(self._lib.tc_set_triangle_test(self._ctx, {"moller_trumbore": 0, "watertight": 1}[test]))

    def set_stream(self, stream: int) -> None:
        """Enqueue on a caller-owned cudaStream_t (0 = the context's own stream)."""
        self._check(self._lib.tc_set_stream(self._ctx, stream or None))

    def set_camera(self, camera: np.ndarray) -> None:
        cam = np.ascontiguousarray(camera, gt.CAMERA)
        self._check(self._lib.tc_set_camera(self._ctx, cam.ctypes.data))

    def render(self, samples: Optional[int] = None, max_bounces: Optional[int] = None, width: Optional[int] = None,
               height: Optional[int] = None, frame_index: int = 0, accumulate: bool = False,
               keep_moments: bool = False, block_size: int = 0, samples_per_item: int = 0, guiding: bool = False,
               guide_record: int = 0, wave_paths: int = 0, short_stack: int = 0, refill_lanes: int = 0,
               guide_fraction: float = 0.0, schedule: str = "auto", ray_sort: int = 0,
               phase_timing: bool = False) -> None:
        """Traces ``samples`` paths per pixel; ``accumulate`` adds them to the previous batches.
        ``guide_fraction``: probability of sampling the network's mixture at a guided diffuse
        vertex (0 = the library's default, 0.5). ``schedule`` (plain renders): "auto",
        "megakernel" or "wavefront". ``phase_timing`` (wavefront): device time of the trace,
        logic, shading and inference launches in ``stats()`` (trace_ms, logic_ms, ...).
        ``guide_record``: training samples of this batch into the sample pool, 1 (or True) after
        emptying it, 2 added to it."""
        if self._params is None:
            raise RuntimeError("render before upload")
        p = self._params.copy()
        if samples is not None:
            p["samples"] = samples
        if max_bounces is not None:
            p["max_bounces"] = max_bounces
        if width is not None:
            p["width"] = width
        if height is not None:
            p["height"] = height
        p["frame_index"] = frame_index
        p["accumulated_samples"] = self.accumulated if accumulate else 0
        opts = native.RenderOptions()
        opts.block_size = block_size
        opts.samples_per_item = samples_per_item
        opts.keep_moments = 1 if keep_moments else 0
        opts.guiding = 1 if guiding else 0
        opts.guide_record = int(guide_record)
        opts.wave_paths = wave_paths
        opts.short_stack = short_stack
        opts.refill_lanes = refill_lanes
        opts.guide_fraction = guide_fraction
        opts.schedule = native.SCHEDULES[schedule]
        opts.ray_sort = ray_sort
        opts.phase_timing = 1 if phase_timing else 0
        self._check(self._lib.tc_render(self._ctx, p.ctypes.data, ctypes.byref(opts)))
        self.width, self.height = int(p["width"][0]), int(p["height"][0])
        self.accumulated = (self.accumulated if accumulate else 0) + int(p["samples"][0])

    def autotune(self, samples: Optional[int] = None, width: Optional[int] = None, height: Optional[int] = None,
                 guiding: bool = False, probe_samples: int = 0) -> dict:
        """Fastest launch shape (block size, refill lanes, short stack, samples per item / wave
        width) for the uploaded scene, with its probe throughput. Replaces the accumulated image."""
        p = self._params.copy()
        if samples is not None:
            p["samples"] = samples
        if width is not None:
            p["width"] = width
        if height is not None:
            p["height"] = height
        base = native.RenderOptions()
        base.guiding = 1 if guiding else 0
        res = native.TuneResult()
        self._check(self._lib.tc_autotune(self._ctx, p.ctypes.data, ctypes.byref(base), probe_samples, ctypes.byref(res)))
        self.width, self.height = int(p["width"][0]), int(p["height"][0])
        self.accumulated = res.probe_samples
        b = res.best
        schedule = {v: k for k, v in native.SCHEDULES.items()}[b.schedule]
        return {"schedule": schedule, "block_size": b.block_size, "short_stack": b.short_stack,
                "samples_per_item": b.samples_per_item,
                "wave_paths": b.wave_paths, "refill_lanes": b.refill_lanes, "kernel_ms": res.best_kernel_ms,
                "mpaths_per_s": res.best_mpaths_per_s, "candidates": res.candidates,
                "probe_samples": res.probe_samples}

    def readback(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        """Linear-HDR float4 image (height, width, 4)."""
        if out is None:
            out = np.empty((self.height, self.width, 4), np.float32)
        self._check(self._lib.tc_readback(self._ctx, out.ctypes.data, out.size))
        return out

    def readback_rgba8(self, exposure_stops: float = 0.0, out: Optional[np.ndarray] = None) -> np.ndarray:
        """Display image (height, width, 4) uint8: exposure, ACES fitted, sRGB, converted on the device."""
        if out is None:
            out = np.empty((self.height, self.width, 4), np.uint8)
        self._check(self._lib.tc_readback_rgba8(self._ctx, float(exposure_stops), out.ctypes.data, out.nbytes))
        return out

    def encode_jpeg(self, quality: int = 90, exposure_stops: float = 0.0) -> bytes:
        """JPEG bytes of the accumulated image, display-converted and encoded on the device."""
        n = ctypes.c_size_t()
        cap = 4 * self.width * self.height + 65536  # above any baseline 4:2:0 frame of this size
        buf = (ctypes.c_uint8 * cap)()
        self._check(self._lib.tc_encode_jpeg(self._ctx, int(quality), float(exposure_stops), buf, cap,
                                             ctypes.byref(n)))
        return bytes(buf[: n.value])

    def display_rgba8_device(self, exposure_stops: float, d_out: int, nbytes: int, stream: int = 0) -> None:
        """Display conversion into caller-owned device memory, enqueued without synchronising."""
        self._check(self._lib.tc_display_rgba8_async(self._ctx, float(exposure_stops), d_out, nbytes, stream or None))

    def readback_sums(self, moments: bool = False):
        """FP64 per-pixel sums (and sums of squares when kept) plus the sample count."""
        n = self.height * self.width * 3
        s = np.empty((self.height, self.width, 3), np.float64)
        q = np.empty((self.height, self.width, 3), np.float64) if moments else None
        count = ctypes.c_uint32()
        self._check(self._lib.tc_readback_sums(self._ctx, s.ctypes.data, None if q is None else q.ctypes.data, n,
                                               ctypes.byref(count)))
        return s, q, int(count.value)

    def trace_closest(self, rays: np.ndarray, tmin: float = 0.001):
        """Closest hit per ray: (prim = kind << 31 | index or TC_MISS, t)."""
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 6)
        prim = np.empty(rays.shape[0], np.uint32)
        t = np.empty(rays.shape[0], np.float32)
        self._check(self._lib.tc_trace_closest(self._ctx, rays.ctypes.data, rays.shape[0], tmin, prim.ctypes.data,
                                               t.ctypes.data))
        return prim, t

    def trace_closest_device(self, rays_ptr: int, n: int, prim_ptr: int, t_ptr: int, tmin: float = 0.001,
                             stream: int = 0) -> None:
        """Enqueues the parity traversal on device buffers (no synchronisation)."""
        self._check(self._lib.tc_trace_closest_device_async(self._ctx, rays_ptr, n, tmin, prim_ptr, t_ptr,
                                                            stream or None))

    # ---------------------------------------------------------------- path-guiding network
    def guide_set_params(self, params: np.ndarray, bounds) -> None:
        """FP32 weights (TC_GUIDE_PARAMS) and encoding frame (cx, cy, cz, scale); resets Adam."""
        p = np.ascontiguousarray(params, np.float32).reshape(-1)
        if p.size != native.GUIDE_PARAMS:
            raise ValueError(f"expected {native.GUIDE_PARAMS} parameters, got {p.size}")
        b = np.ascontiguousarray(bounds, np.float32).reshape(4)
        self._check(self._lib.tc_guide_set_params(self._ctx, p.ctypes.data, b.ctypes.data))

    def guide_get_params(self) -> np.ndarray:
        out = np.empty(native.GUIDE_PARAMS, np.float32)
        self._check(self._lib.tc_guide_get_params(self._ctx, out.ctypes.data))
        return out

    def guide_infer(self, points: np.ndarray, normals: np.ndarray) -> np.ndarray:
        """Decoded mixtures (n, 40): 8 x (mu.xyz, kappa) then 8 weights."""
        q = np.ascontiguousarray(np.concatenate([points, normals], axis=1), np.float32)
        out = np.empty((q.shape[0], 40), np.float32)
        self._check(self._lib.tc_guide_infer(self._ctx, q.ctypes.data, q.shape[0], out.ctypes.data))
        return out

    def guide_loss_grad(self, samples: np.ndarray):
        """Mean weighted NLL and its gradient for samples (n, 10): position, normal, direction, weight."""
        s = np.ascontiguousarray(samples, np.float32).reshape(-1, 10)
        grad = np.empty(native.GUIDE_PARAMS, np.float32)
        loss = ctypes.c_float()
        self._check(self._lib.tc_guide_loss_grad(self._ctx, s.ctypes.data, s.shape[0], grad.ctypes.data,
                                                 ctypes.byref(loss)))
        return grad, float(loss.value)

    def guide_adam_step(self, lr: float = 1e-2) -> None:
        self._check(self._lib.tc_guide_adam_step(self._ctx, lr))

    def guide_train(self, samples: np.ndarray, steps: int, batch: int, lr: float = 1e-2, seed: int = 0) -> np.ndarray:
        s = np.ascontiguousarray(samples, np.float32).reshape(-1, 10)
        losses = np.empty(max(steps, 1), np.float32)
        self._check(self._lib.tc_guide_train(self._ctx, s.ctypes.data, s.shape[0], steps, batch, lr, seed,
                                             losses.ctypes.data))
        return losses[:steps]

    def guide_train_recorded(self, steps: int, batch: int, lr: float = 1e-2, seed: int = 0):
        """Adam steps on the sample pool (every render with guide_record since the last with 1)."""
        losses = np.empty(max(steps, 1), np.float32)
        n = ctypes.c_uint32()
        self._check(self._lib.tc_guide_train_recorded(self._ctx, steps, batch, lr, seed, losses.ctypes.data,
                                                      ctypes.byref(n)))
        return losses[:steps], int(n.value)

    def guide_recorded_samples(self) -> np.ndarray:
        """The sample pool: (n, 12) position + weight, normal, direction."""
        count = ctypes.c_uint32()
        self._check(self._lib.tc_guide_recorded_samples(self._ctx, None, 0, ctypes.byref(count)))
        out = np.empty((count.value, 12), np.float32)
        self._check(self._lib.tc_guide_recorded_samples(self._ctx, out.ctypes.data, out.size, ctypes.byref(count)))
        return out

    def stats(self) -> dict:
        s = native.Stats()
        self._check(self._lib.tc_get_stats(self._ctx, ctypes.byref(s)))
        return {f: getattr(s, f) for f, _ in native.Stats._fields_}


def render_hdr(scene: Scene, device: int = 0, frame_index: int = 0) -> np.ndarray:
    """Renders one frame of ``scene`` at its own settings and returns the linear-HDR image
    (height, width, 4) float32. The reference's file-based entry points are in ``frames``."""
    with GpuRenderer(device) as r:
        r.upload(scene_to_gpu(scene))
        r.render(frame_index=frame_index)
        return r.readback()
