"""The reference's own known-answer tests, restated against the CPU oracle.

Each test cites the reference test it restates (paths relative to the toaster project). They
pin the oracle's arithmetic and sampling to the reference before the oracle is trusted as the
checker of the CUDA path.
"""

import math
import struct

import numpy as np
import pytest

import oracle
from oracle import binding as ob
from toaster_b200 import gpu_types as gt
from toaster_b200.scene import EnvironmentMap, Material, Scene, _read_hdr

MISS = 0xFFFFFFFF
TRI = 0x80000000


def tiny_scene(spheres=(), triangles=(), materials=None, background=gt.SKY, env=None, attrs=None,
               camera=((0, 0, 0), (0, 0, -1)), size=(1, 1), samples=1, max_bounces=1, fov=60.0):
    materials = materials or [Material.diffuse((1, 1, 1))]
    s = Scene(camera_position=camera[0], camera_look_at=camera[1], fov_degrees=fov, width=size[0], height=size[1],
              samples=samples, max_bounces=max_bounces, background=background, materials=materials,
              environment=env)
    if spheres:
        s.sphere_centers = np.array([c for c, r, m in spheres], np.float32)
        s.sphere_radii = np.array([r for c, r, m in spheres], np.float32)
        s.sphere_materials = np.array([m for c, r, m in spheres], np.uint32)
    if triangles:
        s.triangles = np.array([v for v, m in triangles], np.float32)
        s.triangle_materials = np.array([m for v, m in triangles], np.uint32)
    if attrs is not None:
        s.triangle_normals, s.triangle_uvs = attrs
    return s


def ray(o, d):
    return np.array([list(o) + list(d)], np.float32)


def norm(v):
    v = np.asarray(v, np.float32)
    return v * (np.float32(1) / np.sqrt(np.float32(np.dot(v, v))))


# ------------------------------------------------------------------ intersect.rs:354-639
def test_misses_sphere():  # intersect.rs:354-358
    o = oracle.Oracle(tiny_scene(spheres=[((0, 0, -1), 0.5, 0)]))
    prim, t = o.trace_closest(ray((0, 0, 0), (0, 1, 0)))
    assert prim[0] == MISS and np.isinf(t[0])


def test_hits_nearest_sphere_surface_and_preserves_material():  # intersect.rs:360-375
    mats = [Material.diffuse((1, 1, 1))] * 4
    o = oracle.Oracle(tiny_scene(spheres=[((0, 0, -2), 0.5, 3)], materials=mats))
    prim, t, info = o.trace_closest(ray((0, 0, 0), (0, 0, -1)), with_info=True)
    assert prim[0] == 0 and abs(t[0] - 1.5) < 1e-6
    assert tuple(info[0, :3]) == (0.0, 0.0, 1.0) and info[0, 3] == 1.0 and info[0, 4] == 3


def test_inside_ray_uses_far_root_and_orients_normal():  # intersect.rs:377-385
    o = oracle.Oracle(tiny_scene(spheres=[((0, 0, 0), 1.0, 0)]))
    prim, t, info = o.trace_closest(ray((0, 0, 0), (1, 0, 0)), with_info=True)
    assert abs(t[0] - 1.0) < 1e-6
    assert tuple(info[0, :3]) == (-1.0, 0.0, 0.0) and info[0, 3] == 0.0


def test_scene_returns_nearest_hit():  # intersect.rs:387-431
    mats = [Material.diffuse((1, 1, 1))] * 2
    o = oracle.Oracle(tiny_scene(spheres=[((0, 0, -4), 1.0, 0), ((0, 0, -2), 0.5, 1)], materials=mats))
    prim, t, info = o.trace_closest(ray((0, 0, 0), (0, 0, -1)), with_info=True)
    assert info[0, 4] == 1 and prim[0] == 1


TRIANGLE = [(-1.0, -1.0, -2.0), (1.0, -1.0, -2.0), (0.0, 1.0, -2.0)]


def test_triangle_hit_is_double_sided():  # intersect.rs:433-464
    mats = [Material.diffuse((1, 1, 1))] * 8
    o = oracle.Oracle(tiny_scene(triangles=[(TRIANGLE, 7)], materials=mats))
    prim, t, front = o.trace_closest(ray((0, 0, 0), (0, 0, -1)), with_info=True)
    assert prim[0] == TRI | 0 and abs(t[0] - 2.0) < 1e-6 and front[0, 3] == 1.0 and front[0, 4] == 7
    _, _, back = o.trace_closest(ray((0, 0, -3), (0, 0, 1)), with_info=True)
    assert back[0, 3] == 0.0
    assert np.array_equal(back[0, :3], -front[0, :3])


def test_triangle_misses_outside_its_edges():  # intersect.rs:466-480
    o = oracle.Oracle(tiny_scene(triangles=[([(0, 0, 0), (1, 0, 0), (0, 1, 0)], 0)]))
    prim, _ = o.trace_closest(ray((2, 2, 1), (0, 0, -1)))
    assert prim[0] == MISS


def test_bvh_matches_linear_intersection_for_mixed_scene():  # intersect.rs:482-552
    mats = [Material.diffuse((1, 1, 1))] * 3
    s = tiny_scene(spheres=[((-1.5, 0, -4), 0.75, 0), ((1.25, 0, -3), 0.5, 1)], triangles=[(TRIANGLE, 2)],
                   materials=mats)
    o = oracle.Oracle(s)
    rays = np.concatenate([
        ray((0, 0, 0), (0, 0, -1)),
        ray((0, 0, 0), norm((-0.4, 0.0, -1.0))),
        ray((0, 0, 0), norm((0.45, 0.0, -1.0))),
        ray((0, 0, -3), (0, 1, 0)),
        ray((5, 5, 0), (0, 0, -1)),
    ])
    p_bvh, t_bvh, i_bvh = o.trace_closest(rays, with_info=True)
    p_lin, t_lin, i_lin = o.trace_closest(rays, with_info=True, linear=True)
    assert np.array_equal(p_bvh == MISS, p_lin == MISS)
    hit = p_bvh != MISS
    assert np.all(np.abs(t_bvh[hit] - t_lin[hit]) < 1e-5)
    assert np.array_equal(i_bvh[hit, 3:5], i_lin[hit, 3:5])
    assert np.allclose(i_bvh[hit, :3], i_lin[hit, :3], atol=1e-5)


def test_triangle_interpolates_smooth_normal_and_texture_coordinates():  # intersect.rs:608-639
    normals = np.array([[(0, 0, 1)] * 3], np.float32)
    uvs = np.array([[(0.0, 0.0), (1.0, 0.0), (0.5, 1.0)]], np.float32)
    o = oracle.Oracle(tiny_scene(triangles=[(TRIANGLE, 0)], attrs=(normals, uvs)))
    _, _, info = o.trace_closest(ray((0, 0, 0), (0, 0, -1)), with_info=True)
    assert np.allclose(info[0, :3], (0, 0, 1), atol=1e-6)
    assert np.allclose(info[0, 5:7], (0.5, 0.5), atol=1e-6)


# ------------------------------------------------------------------ bvh.rs / flatten.rs / aabb.rs
def test_builds_empty_bvh():  # bvh.rs:172-178
    lib = ob._load()
    st = ob._Settings()
    st.width = st.height = st.samples = st.max_bounces = 1
    h = lib.orc_scene_create(None, 0, None, 0, None, None, 0, None, 0, None, None, 0, 0, 0.0, 0.0, 4)
    assert lib.orc_bvh_node_count(h) == 0 and lib.orc_bvh_prim_count(h) == 0
    lib.orc_scene_destroy(h)


def test_orders_primitives_into_leaves():  # bvh.rs:180-196
    spheres = [((x + 0.25, 0.5, 0.5), 0.25, 0) for x in (0.0, 4.0, 2.0, 6.0)]
    o = oracle.Oracle(tiny_scene(spheres=spheres), max_leaf=1)
    _, links, prims = o.bvh()
    assert len(prims) == 4 and sorted(prims[:, 1].tolist()) == [0, 1, 2, 3]
    assert links[0, 1] == 0  # root is interior


def test_coincident_centroids_create_leaf():  # bvh.rs:198-208
    spheres = [((0.25, 0.5, 0.5), 0.25, 0)] * 3
    o = oracle.Oracle(tiny_scene(spheres=spheres), max_leaf=1)
    _, links, _ = o.bvh()
    assert len(links) == 1 and links[0, 1] == 3


def test_flattens_left_child_next_and_right_child_by_index():  # flatten.rs:106-132
    o = oracle.Oracle(tiny_scene(spheres=[((0, 0, 0), 0.5, 0), ((3, 0, 0), 0.5, 0)]), max_leaf=1)
    _, links, _ = o.bvh()
    assert len(links) == 3
    assert links[0, 1] == 0 and links[0, 0] == 2
    assert links[1, 1] > 0 and links[2, 1] > 0


def test_aabb_intersects_from_outside_inside_and_parallel():  # aabb.rs:127-155
    inf = np.inf
    lo, hi = (-1, -1, -1), (1, 1, 1)
    assert ob.aabb_intersects(lo, hi, (0, 0, 3), (inf, inf, -1), 0.0, inf)
    assert ob.aabb_intersects(lo, hi, (0, 0, 0), (1, inf, inf), 0.0, inf)
    assert not ob.aabb_intersects(lo, hi, (2, 0, 0), (inf, inf, -1), 0.0, inf)


# ------------------------------------------------------------------ camera.rs / core light.rs
def test_center_ray_points_at_target():  # camera.rs:106-110
    b = ob.camera_basis((0, 0, 0), (0, 0, -1), (0, 1, 0), 60.0, 1.0)
    origin, ll, h, v = b
    d = norm(ll + 0.5 * h + 0.5 * v - origin)
    assert np.allclose(d, (0, 0, -1), atol=1e-6)


def test_camera_rejects_non_finite_aspect():  # camera.rs:112-116
    assert ob.camera_basis((0, 0, 0), (0, 0, -1), (0, 1, 0), 60.0, float("nan")) is None
    assert ob.camera_basis((0, 0, 0), (0, 0, -1), (0, 1, 0), 60.0, float("inf")) is None


def test_light_weight_combines_area_luminance_and_strength():  # core light.rs:135-147
    s = tiny_scene(triangles=[([(0, 0, 0), (2.5 * 2, 0, 0), (0, 1, 0)], 0)],
                   materials=[Material.emissive((0.4, 0.4, 0.4), 3.0)])
    lights, total = oracle.Oracle(s).lights()
    assert abs(lights[0, 0] - 2.5) < 1e-6 and abs(lights[0, 1] - 3.0) < 1e-6


# ------------------------------------------------------------------ integrator.rs:391-796
def sphere_scene(albedo=(1, 1, 1), background=gt.SKY, env=None, material=None):
    """integrator.rs:398-433 test_scene."""
    mat = material or Material.diffuse(albedo)
    return tiny_scene(spheres=[((0, 0, -2), 0.7, 0)], materials=[mat], background=background, env=env,
                      size=(5, 5), max_bounces=4)


def test_zero_depth_is_black():  # integrator.rs:527-537
    o = oracle.Oracle(sphere_scene())
    assert np.array_equal(o.ray_color(ray((0, 0, 0), (0, 1, 0)), depth=0), np.zeros((1, 3)))


def test_miss_returns_sky_gradient():  # integrator.rs:539-549
    o = oracle.Oracle(sphere_scene())
    c = o.ray_color(ray((0, 0, 0), (0, 1, 0)), depth=4)
    assert np.allclose(c[0], (0.35, 0.65, 1.0), atol=1e-6)


def test_miss_samples_environment_radiance():  # integrator.rs:551-562
    env = EnvironmentMap(1, 1, np.array([[[3.0, 2.0, 1.0]]], np.float32), 0.5, 0.0)
    o = oracle.Oracle(sphere_scene(background=gt.ENVIRONMENT, env=env))
    c = o.ray_color(ray((0, 0, 0), (1, 0, 0)), depth=1)
    assert tuple(c[0]) == (1.5, 1.0, 0.5)


def test_diffuse_hit_attenuates_returned_radiance_by_albedo():  # integrator.rs:564-573
    albedo = np.array([0.8, 0.4, 0.2], np.float32)
    white = oracle.Oracle(sphere_scene()).ray_color(ray((0, 0, 0), (0, 0, -1)), depth=2, seed=7)
    tinted = oracle.Oracle(sphere_scene(albedo)).ray_color(ray((0, 0, 0), (0, 0, -1)), depth=2, seed=7)
    assert np.allclose(tinted[0], white[0] * albedo, atol=1e-6)


def test_perfect_metal_reflects_and_below_surface_ray_is_absorbed():  # integrator.rs:575-601
    r = ob.scatter((1, -1, 0), (0, 0, 0), (0, 1, 0), True, gt.METAL, albedo=(0.8, 0.8, 0.8), roughness=0.0, seed=3)
    assert np.allclose(r[:3], norm((1, 1, 0)), atol=1e-6)
    assert ob.scatter((0, 1, 0), (0, 0, 0), (0, 1, 0), False, gt.METAL, roughness=0.0, seed=3) is None


def test_metal_scatter_clamps_roughness_defensively():  # integrator.rs:603-633
    a = ob.scatter((0, -1, 0), (0, 0, 0), (0, 1, 0), True, gt.METAL, roughness=1.0, seed=4)
    b = ob.scatter((0, -1, 0), (0, 0, 0), (0, 1, 0), True, gt.METAL, roughness=5.0, seed=4)
    assert np.allclose(a[:3], b[:3], atol=1e-6)


def test_dielectric_refraction_obeys_snells_law():  # integrator.rs:635-641
    d = (0.5, -math.sqrt(3.0) * 0.5, 0.0)
    r = ob.refract(d, (0, 1, 0), 1.0 / 1.5)
    assert abs(r[0] - 1.0 / 3.0) < 1e-6 and abs(np.linalg.norm(r) - 1.0) < 1e-6


def test_dielectric_uses_total_internal_reflection():  # integrator.rs:643-653
    incoming = (0.9, 0.4358899, 0.0)
    r = ob.scatter(incoming, (0, 0, 0), (0, -1, 0), False, gt.DIELECTRIC, ior=1.5, seed=5)
    u = norm(incoming)
    n = np.array([0, -1, 0], np.float32)
    expected = u - 2.0 * np.dot(u, n) * n
    assert np.allclose(r[:3], expected, atol=1e-6) and tuple(r[3:6]) == (1.0, 1.0, 1.0)


def test_schlick_reflectance_has_expected_endpoints():  # integrator.rs:655-659
    assert abs(ob.reflectance(0.0, 1.0 / 1.5) - 1.0) < 1e-6
    assert abs(ob.reflectance(1.0, 1.0 / 1.5) - 0.04) < 1e-6


def test_material_scatter_directions_are_finite_and_normalized():  # integrator.rs:661-680
    for seed, (kind, rough) in enumerate([(gt.DIFFUSE, 0.0), (gt.METAL, 0.2), (gt.DIELECTRIC, 0.0)]):
        r = ob.scatter((0, -1, 0), (0, 0, 0), (0, 1, 0), True, kind, roughness=rough, seed=seed)
        assert np.all(np.isfinite(r[:3])) and abs(np.linalg.norm(r[:3]) - 1.0) < 1e-5


def test_emissive_hit_returns_emitted_radiance_without_scattering():  # integrator.rs:682-691
    o = oracle.Oracle(sphere_scene(material=Material.emissive((1.0, 0.5, 0.25), 4.0)))
    c = o.ray_color(ray((0, 0, 0), (0, 0, -1)), depth=4, seed=9)
    assert np.allclose(c[0], (4.0, 2.0, 1.0), atol=1e-6)


def test_black_background_returns_no_radiance():  # integrator.rs:693-700
    o = oracle.Oracle(sphere_scene(background=gt.BLACK))
    assert np.array_equal(o.ray_color(ray((0, 0, 0), (0, 1, 0)), depth=4, seed=10)[0], np.zeros(3))


def direct_light_scene(blocked):  # integrator.rs:446-515
    tris = [([(-1.0, 2.0, -1.0), (1.0, 2.0, -1.0), (0.0, 2.0, 1.0)], 1)]
    if blocked:
        tris += [([(-3.0, 1.0, -3.0), (3.0, 1.0, 3.0), (3.0, 1.0, -3.0)], 0),
                 ([(-3.0, 1.0, -3.0), (-3.0, 1.0, 3.0), (3.0, 1.0, 3.0)], 0)]
    return tiny_scene(triangles=tris, materials=[Material.diffuse((1, 1, 1)), Material.emissive((1, 1, 1), 5.0)],
                      background=gt.BLACK, camera=((0, 0, 1), (0, 0, 0)), fov=45.0)


def test_direct_light_is_positive_when_visible():  # integrator.rs:702-717
    c = oracle.Oracle(direct_light_scene(False)).direct((0, 0, 0), (0, 1, 0), (0.5, 0.5, 0.5), 0, seed=11)
    assert np.all(c > 0)


def test_shadow_ray_removes_blocked_direct_light():  # integrator.rs:719-734
    c = oracle.Oracle(direct_light_scene(True)).direct((0, 0, 0), (0, 1, 0), (0.5, 0.5, 0.5), 0, seed=11)
    assert np.array_equal(c, np.zeros(3))


def test_direct_environment_sampling_contributes_when_visible():  # integrator.rs:736-752
    env = EnvironmentMap(1, 1, np.array([[[2.0, 2.0, 2.0]]], np.float32), 1.0, 0.0)
    # The reference clears the spheres; a far-away sphere behind the hit keeps the scene non-empty.
    s = tiny_scene(spheres=[((0, -50, 0), 0.1, 0)], background=gt.ENVIRONMENT, env=env)
    c = oracle.Oracle(s).direct((0, 0, 0), (0, 1, 0), (0.5, 0.5, 0.5), 1, draws=64, seed=12)
    assert np.all(c > 0)


def test_environment_miss_uses_bsdf_mis_weight():  # integrator.rs:754-780
    env_rgb = np.ones((1, 1, 3), np.float32)
    env = EnvironmentMap(1, 1, env_rgb, 1.0, 0.0)
    o = oracle.Oracle(sphere_scene(background=gt.ENVIRONMENT, env=env))
    bsdf_pdf = np.float32(1.0 / math.pi)
    env_pdf = oracle.OracleEnvironment(1, 1, env_rgb).lookup([(1, 0, 0)])[1][0]
    expected = ob.power_heuristic(bsdf_pdf, env_pdf)
    c = o.ray_color(ray((0, 0, 0), (1, 0, 0)), depth=1, bsdf_pdf=bsdf_pdf)
    assert np.allclose(c[0], (expected,) * 3, atol=1e-6)


def test_power_heuristic_is_normalized():  # integrator.rs:782-788
    assert abs(ob.power_heuristic(0.25, 0.75) + ob.power_heuristic(0.75, 0.25) - 1.0) < 1e-6
    assert ob.power_heuristic(0.0, 0.0) == 0.0


def test_renders_foreground_and_background():  # integrator.rs:790-796
    mean, _, _ = oracle.Oracle(sphere_scene((1.0, 0.0, 0.0))).render()
    assert mean.shape == (5, 5, 3)
    assert not np.array_equal(mean[2, 2], mean[0, 0])


# ------------------------------------------------------------------ light.rs:227-292
def light_scene():  # light.rs:179-225
    return tiny_scene(
        triangles=[([(0, 0, 0), (2, 0, 0), (0, 1, 0)], 0), ([(0, 0, 1), (1, 0, 1), (0, 1, 1)], 1)],
        materials=[Material.emissive((1.0, 0.5, 0.25), 4.0), Material.diffuse((1, 1, 1))],
        background=gt.BLACK, camera=((0, 0, 1), (0, 0, 0)), fov=45.0)


def test_collects_only_emissive_triangles():  # light.rs:227-232
    lights, _ = oracle.Oracle(light_scene()).lights()
    assert len(lights) == 1


def test_samples_uniform_triangle_with_area_pdf():  # light.rs:234-247
    draws = oracle.Oracle(light_scene()).sample_lights(100, seed=12)
    pos = draws[:, :3]
    assert np.all(pos[:, 0] >= 0) and np.all(pos[:, 1] >= 0)
    assert np.all(pos[:, 0] / 2 + pos[:, 1] <= 1 + 1e-6)
    assert np.allclose(draws[:, 9], 1.0, atol=1e-6)
    assert np.all(draws[:, 6:9] == np.array([4.0, 2.0, 1.0], np.float32))


def test_small_powerful_sphere_dominates_large_dim_triangle_distribution():  # light.rs:249-292
    s = light_scene()
    s.materials[0] = Material.emissive((1, 1, 1), 0.1)
    s.materials.append(Material.emissive((1, 1, 1), 20.0))
    s.triangles[0] = np.array([(0, 0, 0), (4, 0, 0), (0, 4, 0)], np.float32)
    s.sphere_centers = np.array([(0, 2, 0)], np.float32)
    s.sphere_radii = np.array([0.2], np.float32)
    s.sphere_materials = np.array([2], np.uint32)
    o = oracle.Oracle(s)
    lights, total = o.lights()
    assert len(lights) == 2
    dim, bright = lights[0], lights[1]
    assert abs(dim[0] - 8.0) < 1e-6 and abs(dim[1] - 0.8) < 1e-6
    assert abs(bright[1] - bright[0] * 20.0) < 1e-6 and bright[1] > dim[1] * 10
    assert abs(dim[2] - dim[1]) < 1e-6 and abs(bright[2] - total) < 1e-6
    expected = bright[1] / total
    draws = o.sample_lights(20000, seed=29)
    is_bright = np.abs(draws[:, 9] - expected / bright[0]) < 1e-6 * max(1.0, expected / bright[0])
    assert abs(is_bright.mean() - expected) < 0.01


# ------------------------------------------------------------------ environment.rs:295-466
def dir_at_u(u):
    a = (u - 0.5) * 2.0 * math.pi
    return (math.cos(a), 0.0, math.sin(a))


def test_environment_samples_directions_rotation_and_intensity():  # environment.rs:296-316
    px = np.array([[(1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 1)]], np.float32)
    e = oracle.OracleEnvironment(4, 1, px, 2.0, 0.0)
    rgb, _ = e.lookup([dir_at_u(0.625), dir_at_u(0.375)])
    assert np.allclose(rgb[0], (0, 0, 2), atol=1e-6) and np.allclose(rgb[1], (0, 2, 0), atol=1e-6)
    rot = oracle.OracleEnvironment(4, 1, px, 1.0, 90.0)
    assert np.allclose(rot.lookup([dir_at_u(0.375)])[0][0], (0, 0, 1), atol=1e-6)


def write_rgbe(path, pixels):
    """Flat (uncompressed) Radiance RGBE file."""
    h, w, _ = pixels.shape
    out = bytearray(b"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n" + f"-Y {h} +X {w}\n".encode())
    for y in range(h):
        for x in range(w):
            m = float(pixels[y, x].max())
            if m < 1e-32:
                out += bytes(4)
                continue
            mant, e = math.frexp(m)
            scale = mant * 256.0 / m
            out += bytes([int(c * scale) for c in pixels[y, x]] + [e + 128])
    path.write_bytes(bytes(out))


def test_loads_hdr_without_clamping_high_dynamic_range(tmp_path):  # environment.rs:318-337
    p = tmp_path / "env.hdr"
    write_rgbe(p, np.array([[[4.0, 2.0, 1.0]]], np.float32))
    env = _read_hdr(p)
    assert (env.width, env.height) == (1, 1)
    assert np.linalg.norm(env.pixels[0, 0] - (4, 2, 1)) < 0.05
    e = oracle.OracleEnvironment(1, 1, env.pixels, 0.5, -90.0)
    assert e.rotation() == 270.0
    assert np.linalg.norm(e.lookup([(1, 0, 0)])[0][0] - (2.0, 1.0, 0.5)) < 0.05


def entries(cdf):
    prev = np.concatenate([[0.0], cdf[:-1]]).astype(np.float32)
    return np.maximum(cdf - prev, 0.0)


def test_importance_distribution_favors_bright_texels_and_latitude():  # environment.rs:355-377
    px = np.ones((3, 2, 3), np.float32)
    px[0, 1] = 10.0
    cdf = oracle.OracleEnvironment(2, 3, px).cdf()
    p = entries(cdf)
    assert p[1] > p[0] * 9.9 and p[2] > p[0]
    assert abs(cdf[-1] - 1.0) < 1e-6 and abs(p.sum() - 1.0) < 1e-5


def test_importance_sample_and_direction_pdf_agree():  # environment.rs:379-408
    px = np.full((2, 4, 3), 0.1, np.float32)
    px[0, 2] = 8.0
    e = oracle.OracleEnvironment(4, 2, px, 2.0, 35.0)
    s = e.sample([(0.5, 0.37, 0.61)])[0]
    d = s[:3]
    assert s[7] == 1.0 and abs(np.linalg.norm(d) - 1.0) < 1e-6 and s[6] > 0
    rgb, pdf = e.lookup([d])
    assert abs(s[6] - pdf[0]) < 1e-5
    assert np.allclose(s[3:6], rgb[0], atol=1e-6)


def test_importance_sampling_frequencies_match_texel_probabilities():  # environment.rs:410-447
    px = np.array([[[1] * 3, [4] * 3, [2] * 3], [[3] * 3, [1] * 3, [5] * 3]], np.float32)
    e = oracle.OracleEnvironment(3, 2, px, 1.0, 27.0)
    expected = entries(e.cdf())
    n = 10000
    u = np.stack([(np.arange(n) + 0.5) / n, np.full(n, 0.5), np.full(n, 0.5)], 1)
    samples = e.sample(u)
    counts = np.zeros(6)
    for d in samples[:, :3]:
        uu, vv, _ = e.direction_to_uv(d)
        counts[int(math.floor(vv * 2)) * 3 + int(math.floor(uu * 3))] += 1
    assert np.all(np.abs(counts / n - expected) <= 2.0 / n + 1e-7)


def test_black_or_disabled_environment_has_no_importance_samples():  # environment.rs:449-457
    black = oracle.OracleEnvironment(2, 1, np.zeros((1, 2, 3), np.float32))
    disabled = oracle.OracleEnvironment(1, 1, np.ones((1, 1, 3), np.float32), 0.0)
    assert black.sample([(0.5, 0.5, 0.5)])[0, 7] == 0.0
    assert black.lookup([(1, 0, 0)])[1][0] == 0.0
    assert disabled.sample([(0.5, 0.5, 0.5)])[0, 7] == 0.0


def test_rejects_invalid_environment_dimensions_pixels_and_controls():  # environment.rs:459-466
    with pytest.raises(ValueError):
        EnvironmentMap(0, 1, np.zeros((0, 0, 3), np.float32))
    with pytest.raises(ValueError):
        EnvironmentMap(1, 1, -np.ones((1, 1, 3), np.float32))
    with pytest.raises(ValueError):
        EnvironmentMap(1, 1, np.ones((1, 1, 3), np.float32), -1.0)
    with pytest.raises(ValueError):
        EnvironmentMap(1, 1, np.ones((1, 1, 3), np.float32), 1.0, float("nan"))


# ------------------------------------------------------------------ gpu_types.rs:200-211
def test_gpu_types_match_wgsl_layout_sizes():
    for name, (dtype, size) in gt.RECORD_SIZES.items():
        assert dtype.itemsize == size, name


# ------------------------------------------------------------------ color.rs / image_output.rs
def test_converts_float_pixels_to_rgba_once():  # image_output.rs:96-103
    px = np.array([[-1.0, 0.5, 2.0, 1.0], [0.0, 0.25, 0.75, 0.0]], np.float32)
    assert ob.display_rgba8(px).reshape(-1).tolist() == [0, 206, 245, 255, 0, 165, 223, 0]


def test_display_conversion_handles_nonfinite_radiance():  # color.rs:104-113
    px = np.array([[np.nan, -np.inf, np.inf, 1.0]], np.float32)
    assert ob.display_rgba8(px)[0, :3].tolist() == [0, 0, 255]


def test_exposure_scales_by_powers_of_two():  # color.rs:88-93
    px = np.array([[0.125, 0.5, 2.0, 1.0]], np.float32)
    scale = lambda k: px * np.float32([k, k, k, 1.0])  # noqa: E731 - alpha is not exposed
    assert np.array_equal(ob.display_rgba8(px, 2.0), ob.display_rgba8(scale(4.0)))
    assert np.array_equal(ob.display_rgba8(px, -1.0), ob.display_rgba8(scale(0.5)))
