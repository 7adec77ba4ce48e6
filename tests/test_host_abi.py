"""Host-side checks that need no GPU: the C ABI library loads and exports what the header
declares, record layouts agree, and the library's host hierarchy build equals the oracle's."""

import re
from pathlib import Path

import numpy as np
import pytest

import oracle
from toaster_b200 import configs, gpu_types as gt, native
from toaster_b200.renderer import progressive_batch
from toaster_b200.scene import Material, Scene, box_triangles, load_scene, save_scene_json, scene_to_gpu

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    text = (ROOT / "include" / "toaster_cuda.h").read_text()
    return sorted(set(re.findall(r"^\s*(?:int|long|const \w+\s*\*)\s+(tc_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_function(native_lib):
    names = declared_functions()
    assert names, "no tc_* declarations found"
    for name in names:
        assert hasattr(native_lib, name), name
    assert set(names) == set(native.EXPORTED_SYMBOLS)
    assert native_lib.tc_abi_version() == 1


def test_record_sizes_match_reference_layouts(native_lib):
    sizes = native.record_sizes()
    expected = [gt.RECORD_SIZES[k][1] for k in ("GpuRenderParams", "GpuCamera", "GpuSphere", "GpuTriangle",
                                                   "GpuTriangleAttributes", "GpuMaterial", "GpuLight",
                                                   "GpuBvhNode", "GpuPrimitiveRef")]
    assert sizes == expected


def test_context_creation_fails_loudly_without_device(native_lib):
    import ctypes

    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    ctx = ctypes.c_void_p()
    code = native_lib.tc_create(0, ctypes.byref(ctx))
    assert code == -3  # TC_ERR_NO_DEVICE: there is no CPU fallback
    assert native_lib.tc_last_error(None)


def bvh_equal(scene):
    o = oracle.Oracle(scene)
    bounds, links, prims = o.bvh()
    d = scene_to_gpu(scene)
    nodes, refs = native.build_bvh_host(d.spheres, d.triangles)
    got_bounds = np.concatenate([nodes["min"], nodes["max"]], axis=1)
    assert np.array_equal(got_bounds.view(np.uint32), bounds.view(np.uint32))
    assert np.array_equal(nodes["first_or_right"], links[:, 0])
    assert np.array_equal(nodes["primitive_count"], links[:, 1])
    assert np.array_equal(refs["kind"], prims[:, 0]) and np.array_equal(refs["index"], prims[:, 1])


@pytest.mark.parametrize("make", [configs.plain_small, configs.mixed])
def test_host_bvh_build_is_bit_identical_to_oracle(native_lib, make):
    bvh_equal(make())


def test_host_bvh_handles_degenerate_and_tied_centroids(native_lib):
    # Coincident centroids (bvh.rs:119 degenerate leaf), equal keys on the split axis (stable
    # order) and negative zero / mixed signs in coordinates (total_cmp ordering).
    rng = np.random.default_rng(5)
    base = rng.uniform(-1, 1, (40, 3)).astype(np.float32)
    base[10:20] = base[10]  # ten identical spheres
    base[20:30, 0] = np.float32(0.25)  # ties along x
    base[30:35] = np.array([-0.0, 0.0, 0.0], np.float32)
    s = Scene(camera_position=(0, 0, 5), camera_look_at=(0, 0, 0), materials=[Material.diffuse((0.5, 0.5, 0.5))],
              sphere_centers=base, sphere_radii=np.full(40, 0.1, np.float32), sphere_materials=np.zeros(40, np.uint32),
              triangles=np.concatenate([box_triangles((0, 0, 0), (1, 1, 1)), box_triangles((0, 0, 0), (1, 1, 1))]),
              triangle_materials=np.zeros(24, np.uint32))
    bvh_equal(s)


def test_host_bvh_empty_input(native_lib):
    nodes, prims = native.build_bvh_host(np.zeros(0, gt.SPHERE), np.zeros(0, gt.TRIANGLE))
    assert len(nodes) == 0


def test_host_bvh_large_heightfield_matches_oracle(native_lib):
    tris = configs.heightfield_triangles(configs.fbm_heights(96))
    s = Scene(camera_position=(0, 2, 5), camera_look_at=(0, 0, 0), materials=[Material.diffuse((0.5, 0.5, 0.5))],
              triangles=tris, triangle_materials=np.zeros(len(tris), np.uint32))
    bvh_equal(s)


def test_progressive_batch_clamps_to_target():  # path_tracer.rs:900-923 and its tests
    assert progressive_batch(4, 0, 10) == 4
    assert progressive_batch(4, 8, 10) == 2
    assert progressive_batch(4, 10, 10) is None
    with pytest.raises(ValueError):
        progressive_batch(0, 0, 10)
    with pytest.raises(ValueError):
        progressive_batch(4, 11, 10)


def test_scene_json_round_trip(tmp_path):
    s = configs.plain_small()
    p = tmp_path / "scene.json"
    save_scene_json(s, p)
    t = load_scene(p)
    assert t.triangle_count == s.triangle_count and t.sphere_count == s.sphere_count
    assert np.array_equal(t.triangles, s.triangles)
    assert [m.kind for m in t.materials] == [m.kind for m in s.materials]
    a, b = scene_to_gpu(s), scene_to_gpu(t)
    assert np.array_equal(a.lights, b.lights) and np.array_equal(a.camera, b.camera)


def test_box_expands_to_twelve_triangles():  # loader.rs:1541-1568
    tris = box_triangles((0, 1, 0), (1, 2, 1))
    assert tris.shape == (12, 3, 3)
    assert tris[:, :, 1].min() == 0.0 and tris[:, :, 1].max() == 2.0


def test_light_packing_matches_oracle_cdf():  # scene_upload.rs:412-475 vs light.rs:57-113
    s = configs.mixed()
    d = scene_to_gpu(s)
    lights, total = oracle.Oracle(s).lights()
    assert len(d.lights) == len(lights) == 16
    assert np.array_equal(d.lights["area_weight_cumulative"][:, :3], lights[:, :3])
    assert np.float32(d.params["total_light_weight"][0]) == np.float32(total)


def test_camera_packing_matches_oracle():  # scene_upload.rs:352-368 vs camera.rs:54-91
    from oracle.binding import camera_basis

    s = configs.mixed()
    cam = scene_to_gpu(s).camera[0]
    ref = camera_basis(s.camera_position, s.camera_look_at, s.camera_up, s.fov_degrees, s.width / s.height)
    got = np.stack([cam["origin"][:3], cam["lower_left_corner"][:3], cam["horizontal"][:3], cam["vertical"][:3]])
    assert np.allclose(got, ref, rtol=0, atol=1e-6)


def test_host_display_conversion_of_the_baseline_matches_oracle():
    # The plain unbatched animation path converts on the host as the reference does; it must give
    # the oracle's bytes (color.rs:24-74) so latency comparisons compare equal work.
    from oracle import binding as ob
    from toaster_b200.batch_eval import host_display_rgba8

    rng = np.random.default_rng(3)
    hdr = np.concatenate([rng.exponential(0.5, (64, 96, 3)), np.ones((64, 96, 1))], -1).astype(np.float32)
    hdr[0, 0, :3] = [np.nan, np.inf, -1.0]
    for exposure in (0.0, 1.5, -2.0):
        ref = ob.display_rgba8(hdr.reshape(-1, 4), exposure).reshape(hdr.shape)
        got = host_display_rgba8(hdr, exposure)
        assert np.abs(ref.astype(int) - got.astype(int)).max() <= 1
        assert np.mean(ref == got) > 0.999


def test_ballistic_animation_is_deterministic_and_keeps_counts():
    a = configs.BallisticAnimation(frames=24, width=64, height=36)
    b = configs.BallisticAnimation(frames=24, width=64, height=36)
    s0, s23 = a.scene(0), a.scene(23)
    assert s0.sphere_count == s23.sphere_count == 64
    assert s0.triangle_count == s23.triangle_count == 2 + 64 * 12
    assert np.array_equal(a.scene(17).triangles, b.scene(17).triangles)
    assert not np.array_equal(s0.sphere_centers, s23.sphere_centers)
    assert np.all(s23.sphere_centers[:, 1] >= s23.sphere_radii - 1e-5)  # bodies stay above the ground


def test_uneven_batch_spans_sizes():
    scenes = configs.uneven_batch(count=4, seed=1)
    for s in scenes:
        assert 128 <= s.triangle_count <= 262144
        assert 320 <= s.width <= 1280 and s.width % 16 == 0 and s.height == s.width * 9 // 16


def test_mjpeg_part_framing():  # toaster-server routes.rs: formats_mjpeg_part
    from toaster_b200.stream import mjpeg_part, split_mjpeg

    part = mjpeg_part(bytes([0xFF, 0xD8, 0xFF, 0xD9]))
    assert part == b"--frame\r\nContent-Type: image/jpeg\r\nContent-Length: 4\r\n\r\n\xff\xd8\xff\xd9\r\n"
    frames = [bytes([0xFF, 0xD8, i, 0xFF, 0xD9]) for i in range(3)]
    assert split_mjpeg(b"".join(mjpeg_part(f) for f in frames)) == frames
