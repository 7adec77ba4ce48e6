"""NumPy mirrors of toaster-gpu's ``#[repr(C)]`` scene records.

Byte layouts follow ``crates/toaster-gpu/src/gpu_types.rs`` (sizes pinned by its
``gpu_types_match_wgsl_layout_sizes`` test, gpu_types.rs:200-211) and are identical to the C
structs in ``include/toaster_cuda.h``.
"""

from __future__ import annotations

import numpy as np

RENDER_PARAMS = np.dtype(
    [
        ("width", "<u4"),
        ("height", "<u4"),
        ("samples", "<u4"),
        ("max_bounces", "<u4"),
        ("sphere_count", "<u4"),
        ("triangle_count", "<u4"),
        ("material_count", "<u4"),
        ("frame_index", "<u4"),
        ("background_kind", "<u4"),
        ("light_count", "<u4"),
        ("total_light_weight", "<f4"),
        ("_pad0", "<u4"),
        ("environment_width", "<u4"),
        ("environment_height", "<u4"),
        ("environment_intensity", "<f4"),
        ("environment_rotation_degrees", "<f4"),
        ("accumulated_samples", "<u4"),
        ("_pad1", "<u4", 3),
        ("bvh_node_count", "<u4"),
        ("bvh_primitive_count", "<u4"),
        ("_pad2", "<u4", 2),
    ]
)
CAMERA = np.dtype(
    [("origin", "<f4", 4), ("lower_left_corner", "<f4", 4), ("horizontal", "<f4", 4), ("vertical", "<f4", 4)]
)
SPHERE = np.dtype([("center_radius", "<f4", 4), ("material_index", "<u4"), ("_pad0", "<u4", 3)])
TRIANGLE = np.dtype(
    [("v0", "<f4", 4), ("v1", "<f4", 4), ("v2", "<f4", 4), ("material_index", "<u4"), ("_pad0", "<u4", 3)]
)
TRIANGLE_ATTRIBUTES = np.dtype(
    [
        ("n0", "<f4", 4),
        ("n1", "<f4", 4),
        ("n2", "<f4", 4),
        ("uv0", "<f4", 2),
        ("uv1", "<f4", 2),
        ("uv2", "<f4", 2),
        ("flags", "<u4"),
        ("_pad0", "<u4"),
    ]
)
MATERIAL = np.dtype(
    [
        ("kind", "<u4"),
        ("texture_offset", "<u4"),
        ("texture_width", "<u4"),
        ("texture_height", "<u4"),
        ("albedo", "<f4", 4),
        ("params", "<f4", 4),
    ]
)
LIGHT = np.dtype(
    [
        ("kind", "<u4"),
        ("material_index", "<u4"),
        ("_pad0", "<u4", 2),
        ("v0", "<f4", 4),
        ("v1", "<f4", 4),
        ("v2", "<f4", 4),
        ("center_radius", "<f4", 4),
        ("area_weight_cumulative", "<f4", 4),
    ]
)
BVH_NODE = np.dtype(
    [("min", "<f4", 4), ("max", "<f4", 4), ("first_or_right", "<u4"), ("primitive_count", "<u4"), ("_pad", "<u4", 2)]
)
PRIMITIVE_REF = np.dtype([("kind", "<u4"), ("index", "<u4")])

RECORD_SIZES = {
    "GpuRenderParams": (RENDER_PARAMS, 96),
    "GpuCamera": (CAMERA, 64),
    "GpuSphere": (SPHERE, 32),
    "GpuTriangle": (TRIANGLE, 64),
    "GpuTriangleAttributes": (TRIANGLE_ATTRIBUTES, 80),
    "GpuMaterial": (MATERIAL, 48),
    "GpuLight": (LIGHT, 96),
    "GpuBvhNode": (BVH_NODE, 48),
    "GpuPrimitiveRef": (PRIMITIVE_REF, 8),
}

# Material kind codes (gpu_types.rs:129) and background codes (scene_upload.rs:257-261).
DIFFUSE, METAL, DIELECTRIC, EMISSIVE = 0, 1, 2, 3
SKY, BLACK, ENVIRONMENT = 0, 1, 2
