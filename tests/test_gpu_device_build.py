"""The device median-split build (tc_set_hierarchy_build) against the oracle and the host build
(needs a B200).

Both builds produce the reference's tree, so closest hits through a device-built hierarchy must
equal the oracle's bit for bit, exactly as the host-built one does; a scene whose reference tree
has a degenerate leaf makes the device build fall back to the host build.
"""

import numpy as np
import pytest

import oracle
from toaster_b200 import configs
from toaster_b200.renderer import GpuRenderer
from toaster_b200.scene import Material, Scene, box_triangles, scene_to_gpu

pytestmark = pytest.mark.gpu
MISS = 0xFFFFFFFF


def hits(r, scene, rays, mode):
    r.set_hierarchy_build(mode)
    r.upload(scene_to_gpu(scene))
    return r.trace_closest(rays)


@pytest.mark.parametrize("make", [configs.plain_small, configs.mixed,
                                  lambda: configs.room_with_window(clutter=2048)], ids=["plain_small", "mixed", "room"])
def test_device_build_hits_equal_oracle(native_lib, make):
    scene = make()
    rays = configs.parity_rays(scene, 1 << 18, seed=9)
    op, ot = oracle.Oracle(scene).trace_closest(rays)
    with GpuRenderer(0) as r:
        gp, gt_ = hits(r, scene, rays, "device")
        assert r.stats()["bvh_depth"] > 1
    assert np.array_equal(gp, op)
    assert np.array_equal(gt_.view(np.uint32), ot.view(np.uint32))


def test_device_and_host_builds_trace_identically(native_lib):
    tris = configs.heightfield_triangles(configs.fbm_heights(128, seed=5))
    scene = Scene(camera_position=(0, 1.5, 5), camera_look_at=(0, 0, 0), materials=[Material.diffuse((0.5,) * 3)],
                  triangles=tris, triangle_materials=np.zeros(len(tris), np.uint32))
    rays = configs.parity_rays(scene, 1 << 18, seed=6)
    with GpuRenderer(0) as r:
        dp, dt = hits(r, scene, rays, "device")
        hp, ht = hits(r, scene, rays, "host")
    assert np.array_equal(dp, hp)
    assert np.array_equal(dt.view(np.uint32), ht.view(np.uint32))


def test_degenerate_leaf_falls_back_to_host_build(native_lib):
    # Six coincident spheres: the reference makes them one leaf of six (centroid extent 0).
    tris = box_triangles((2, 0, 0), (1, 1, 1))
    centers = np.array([(0, 2, 0)] * 6 + [(-2, 0, 0), (1.5, -1.5, 0.5)], np.float32)
    scene = Scene(camera_position=(0.5, 0.7, 4), camera_look_at=(0, 0, 0), materials=[Material.diffuse((0.5,) * 3)],
                  sphere_centers=centers, sphere_radii=np.array([0.3] * 6 + [0.5, 0.25], np.float32),
                  sphere_materials=np.zeros(8, np.uint32), triangles=tris,
                  triangle_materials=np.zeros(len(tris), np.uint32))
    rays = configs.parity_rays(scene, 1 << 14, seed=2)
    op, ot = oracle.Oracle(scene).trace_closest(rays)
    with GpuRenderer(0) as r:
        gp, gt_ = hits(r, scene, rays, "device")
    assert np.array_equal(gp, op)
    assert np.array_equal(gt_.view(np.uint32), ot.view(np.uint32))


def test_device_built_scene_renders_the_same_paths(native_lib):
    scene = configs.mixed(width=96, height=54, samples=8, max_bounces=6)
    with GpuRenderer(0) as r:
        out = []
        for mode in ("host", "device"):
            r.set_hierarchy_build(mode)
            r.upload(scene_to_gpu(scene))
            r.render(frame_index=3)
            out.append(r.readback_sums()[0])
    rel = np.abs(out[0] - out[1]) / np.maximum(np.abs(out[0]), 1e-6)
    assert np.mean(rel < 1e-9) > 0.999
