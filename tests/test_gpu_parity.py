"""CUDA path vs the CPU oracle on the same seeded inputs (needs a B200).

Closest hit: the primitive index must match bit-exactly and the hit distance within 4 ulp
(this implementation reproduces the reference's f32 arithmetic, so the distances are expected to
be identical; the 4-ulp bound is the stated tolerance). Images: per-pixel means must agree
within a 3-sigma band built from both renderers' per-pixel sample variances, with the fraction of
pixels outside it, the median block z-score and the image-mean difference held to bars calibrated
by running the oracle against itself (tests/calibrate_parity.py).
"""

import json
from pathlib import Path

import numpy as np
import pytest

import oracle
import parity_cases
import parity_stats
from toaster_b200 import configs, gpu_types as gt
from toaster_b200.native import TcError
from toaster_b200.scene import EnvironmentMap, Material, Scene, box_triangles, scene_to_gpu

pytestmark = pytest.mark.gpu
MISS = 0xFFFFFFFF


def ulp_distance(a, b):
    ai = a.view(np.int32).astype(np.int64)
    bi = b.view(np.int32).astype(np.int64)
    ai = np.where(ai < 0, np.int64(-(2**31)) - ai, ai)
    bi = np.where(bi < 0, np.int64(-(2**31)) - bi, bi)
    return np.abs(ai - bi)


def check_hits(renderer, scene, rays, tmin=0.001):
    renderer.upload(scene_to_gpu(scene))
    gp, gtt = renderer.trace_closest(rays, tmin)
    op, ot = oracle.Oracle(scene).trace_closest(rays, tmin)
    mismatch = np.nonzero(gp != op)[0]
    assert mismatch.size == 0, f"{mismatch.size} primitive mismatches, first rays {mismatch[:5]}: {gp[mismatch[:5]]} vs {op[mismatch[:5]]}"
    hit = op != MISS
    assert np.all(np.isinf(gtt[~hit]))
    assert np.max(ulp_distance(gtt[hit], ot[hit]), initial=0) <= 4
    return gp, gtt, op, ot


@pytest.mark.parametrize("make", [configs.plain_small, configs.mixed], ids=["plain_small", "mixed"])
def test_closest_hit_bit_exact_on_2_20_seeded_rays(renderer, make):
    scene = make()
    rays = configs.parity_rays(scene, 1 << 20, seed=0)
    gp, gtt, op, ot = check_hits(renderer, scene, rays)
    assert np.array_equal(gtt.view(np.uint32), ot.view(np.uint32))  # identical distances in practice
    assert 0.2 < np.mean(op != MISS) < 0.95


def test_closest_hit_edge_cases(renderer):
    # Axis-parallel rays (infinite 1/d), origins on box faces, rays aimed at shared box edges and
    # vertices, duplicated triangles (exact ties resolved by traversal order) and a stack of
    # coincident spheres (degenerate leaf).
    tris = np.concatenate([box_triangles((0, 0, 0), (1, 1, 1)), box_triangles((0, 0, 0), (1, 1, 1)),
                           box_triangles((2, 0.5, -1), (0.5, 2, 0.5))])
    centers = np.array([(0, 2, 0)] * 6 + [(-2, 0, 0), (1.5, -1.5, 0.5)], np.float32)
    radii = np.array([0.3] * 6 + [0.5, 0.25], np.float32)
    scene = Scene(camera_position=(0.5, 0.7, 4), camera_look_at=(0, 0, 0), materials=[Material.diffuse((0.5,) * 3)],
                  sphere_centers=centers, sphere_radii=radii, sphere_materials=np.zeros(8, np.uint32),
                  triangles=tris, triangle_materials=np.zeros(len(tris), np.uint32))
    rays = []
    for o in [(0, 0, 3), (0.5, 0.5, 3), (0.5, 0, 3), (3, 0.5, 0.5), (0, 3, 0), (-0.5, -0.5, -0.5), (0, 0, 0),
              (0.25, 0.25, 0.5), (2, 5, -1), (-2, 0, 5)]:
        for d in [(0, 0, -1), (0, 0, 1), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0)]:
            rays.append(list(o) + list(d))
    verts = np.unique(tris.reshape(-1, 3), axis=0)
    rng = np.random.default_rng(11)
    for v in verts:
        for _ in range(8):
            o = rng.uniform(-4, 4, 3).astype(np.float32)
            d = (v - o).astype(np.float32)
            d = d * (np.float32(1) / np.sqrt(np.float32(np.dot(d, d))))
            rays.append(list(o) + list(d))
    edge_mid = ((tris[:, 0] + tris[:, 1]) * np.float32(0.5)).astype(np.float32)
    for m in edge_mid:
        o = rng.uniform(-4, 4, 3).astype(np.float32)
        d = (m - o).astype(np.float32)
        d = d * (np.float32(1) / np.sqrt(np.float32(np.dot(d, d))))
        rays.append(list(o) + list(d))
    rays = np.array(rays, np.float32)
    for tmin in (0.001, 0.0):
        check_hits(renderer, scene, rays, tmin)


def test_closest_hit_heightfield_shared_edges(renderer):
    tris = configs.heightfield_triangles(configs.fbm_heights(192, seed=3))
    scene = Scene(camera_position=(0, 1.5, 5), camera_look_at=(0, 0, 0), materials=[Material.diffuse((0.5,) * 3)],
                  triangles=tris, triangle_materials=np.zeros(len(tris), np.uint32))
    rays = configs.parity_rays(scene, 1 << 18, seed=4)
    check_hits(renderer, scene, rays)


def constant_env(rgb, intensity=1.0):
    return EnvironmentMap(1, 1, np.array([[rgb]], np.float32), intensity, 0.0)


def render_image(renderer, scene, **kw):
    renderer.upload(scene_to_gpu(scene))
    renderer.render(**kw)
    return renderer.readback()


def test_environment_miss_radiance_known_answer(renderer):  # integrator.rs:551-562 on the GPU
    scene = Scene(camera_position=(0, 0, 0), camera_look_at=(1, 0, 0), width=16, height=8, samples=4, max_bounces=1,
                  background=gt.ENVIRONMENT, materials=[Material.diffuse((1, 1, 1))],
                  sphere_centers=np.array([(-50, 0, 0)], np.float32), sphere_radii=np.array([0.1], np.float32),
                  sphere_materials=np.zeros(1, np.uint32), environment=constant_env((3.0, 2.0, 1.0), 0.5))
    img = render_image(renderer, scene)
    assert np.array_equal(img[..., :3], np.broadcast_to(np.float32([1.5, 1.0, 0.5]), img[..., :3].shape))
    assert np.all(img[..., 3] == 1.0)


def test_emissive_and_black_known_answers(renderer):  # integrator.rs:682-700 on the GPU
    base = dict(camera_position=(0, 0, 0), camera_look_at=(0, 0, -1), width=8, height=8, samples=2, max_bounces=4,
                sphere_centers=np.array([(0, 0, -2)], np.float32), sphere_radii=np.array([50.0], np.float32),
                sphere_materials=np.zeros(1, np.uint32))
    emissive = Scene(background=gt.BLACK, materials=[Material.emissive((1.0, 0.5, 0.25), 4.0)], **base)
    img = render_image(renderer, emissive)
    assert np.allclose(img[..., :3], (4.0, 2.0, 1.0), atol=1e-6)
    black = Scene(background=gt.BLACK, materials=[Material.diffuse((0.7, 0.7, 0.7))], **base)
    assert np.array_equal(render_image(renderer, black)[..., :3], np.zeros((8, 8, 3), np.float32))
    zero_depth = Scene(background=gt.SKY, materials=[Material.emissive((1, 1, 1), 3.0)], **base)
    assert np.array_equal(render_image(renderer, zero_depth, max_bounces=0)[..., :3], np.zeros((8, 8, 3), np.float32))


CALIBRATION = Path(__file__).resolve().parent / "golden" / "parity_calibration.json"
# Bars over the oracle-against-itself calibration (worst of three independent seed pairs at the
# same sample counts): limit = factor x worst + slack. The slack covers the sampling noise of a
# statistic that three pairs cannot pin (binomial noise of a 1% fraction over ~7,000 z-scores is
# about 0.1%; the median of ~600 block z-scores moves by about 0.05).
BARS = {"outside_pixel": (1.5, 0.005), "outside_block": (1.5, 0.01), "median_z": (1.5, 0.15),
        "global_dz": (1.5, 2.0), "rel_mean": (1.5, 0.01)}


def statistical_parity(renderer, case_name, upload=None, scene=None):
    """GPU image vs the oracle's on one case of tests/parity_cases.py.

    Both renderers keep per-pixel sums of squared samples, and every z-score uses the variance of
    the difference of the two means (GPU variance / GPU samples + oracle variance / oracle
    samples), per pixel and channel and over 2x2-pixel luminance blocks (tests/parity_stats.py).
    The bars come from running the oracle against itself at the same sample counts
    (tests/calibrate_parity.py, tests/golden/parity_calibration.json). ``upload`` replaces the
    default upload of ``scene_to_gpu(scene)`` (the oracle always renders ``scene``).
    """
    case = parity_cases.BY_NAME[case_name]
    scene = scene if scene is not None else case.make()
    if upload is None:
        renderer.upload(scene_to_gpu(scene))
    else:
        upload()
    renderer.render(samples=case.gpu_spp, keep_moments=True, frame_index=17)
    s, q, n = renderer.readback_sums(moments=True)
    assert n == case.gpu_spp
    g_mean = s / n
    g_var = parity_stats.sample_variance(g_mean, q, n)
    cpu_scene = Scene(**{**scene.__dict__, "samples": case.cpu_spp})
    o_mean, o_sq, _ = oracle.Oracle(cpu_scene).render(seed=3, moments=True)
    o_var = parity_stats.sample_variance(o_mean, o_sq, case.cpu_spp)
    st = parity_stats.compare(g_mean, g_var, case.gpu_spp, o_mean, o_var, case.cpu_spp)
    print(json.dumps({"case": case_name, **st}))
    worst = json.loads(CALIBRATION.read_text())[case_name]["worst"]
    assert st["constant_mismatch"] == 0, st
    for key, (factor, slack) in BARS.items():
        limit = factor * worst[key] + slack
        if key == "rel_mean":
            # Heavy-tailed scenes (the sun room) move their image mean by more than three seed pairs
            # show; the relative bar is then at least three standard errors of this run's difference.
            limit = max(limit, 3.0 * st["rel_se"])
        assert abs(st[key]) <= limit, f"{case_name}: {key} = {st[key]:.4f} beyond {limit:.4f} ({st})"
    return st


@pytest.mark.parametrize("case_name", [c.name for c in parity_cases.CASES])
def test_image_statistical_parity(renderer, case_name):
    statistical_parity(renderer, case_name)


def test_progressive_accumulation_contract(renderer):
    s = configs.mixed(width=32, height=18, samples=8)
    renderer.upload(scene_to_gpu(s))
    for frame in range(4):
        renderer.render(samples=8, frame_index=frame, accumulate=frame > 0)
    assert renderer.accumulated == 32
    _, _, n = renderer.readback_sums()
    assert n == 32
    img = renderer.readback()
    assert np.all(np.isfinite(img)) and np.all(img[..., 3] == 1.0)
    # A batch that claims a different history is rejected (path_tracer.rs:900-923 contract).
    p = renderer._params.copy()
    p["accumulated_samples"] = 5
    with pytest.raises(TcError):
        renderer._check(renderer._lib.tc_render(renderer._ctx, p.ctypes.data, None))


def test_invalid_scene_is_rejected(renderer):
    s = configs.mixed(width=8, height=8, samples=1)
    d = scene_to_gpu(s)
    d.spheres["material_index"][0] = 10_000
    with pytest.raises(TcError, match="unknown material"):
        renderer.upload(d)


def to_bf16_bits(x):
    import torch

    return torch.from_numpy(np.ascontiguousarray(x, np.float32)).to(torch.bfloat16).view(torch.int16).numpy().view(np.uint16)


def from_bf16_bits(b):
    import torch

    return torch.from_numpy(b.view(np.int16)).view(torch.bfloat16).float().numpy()


@pytest.mark.parametrize("a_mn,b_mn", [(False, False), (True, False), (False, True), (True, True)])
@pytest.mark.parametrize("n,k", [(64, 80), (32, 64), (128, 16)])
def test_tcgen05_tile_matches_fp32_matmul(native_lib, a_mn, b_mn, n, k):
    from toaster_b200 import native

    rng = np.random.default_rng(n * 1000 + k)
    a = to_bf16_bits(rng.standard_normal((128, k)))
    b = to_bf16_bits(rng.standard_normal((n, k)))
    d = native.umma_selftest(a, b, a_mn, b_mn)
    ref = from_bf16_bits(a).astype(np.float64) @ from_bf16_bits(b).astype(np.float64).T
    assert np.allclose(d, ref, rtol=1e-3, atol=1e-3), np.abs(d - ref).max()


def test_closest_hit_large_mesh_2_20_rays(renderer):
    # Config 3 geometry: 1024 x 1024 fBm heightfield (2,093,058 triangles) + 512 spheres; the
    # hierarchy (2^20 - 1 nodes) lives in HBM.
    scene = configs.large_mesh()
    rays = configs.parity_rays(scene, 1 << 20, seed=9)
    gp, gtt, op, ot = check_hits(renderer, scene, rays)
    assert np.array_equal(gtt.view(np.uint32), ot.view(np.uint32))
    assert np.mean(op != MISS) > 0.3
