"""Seeded synthetic workloads standing in for the benchmark configurations.

The reference publishes no dataset for its GPU path beyond seven small fixture scenes; these
generators produce scenes of the stated shapes, sizes and value distributions instead (all
choices not fixed by the workload description are documented on each function):

  plain_small()   320x180, 4 spp, 4 bounces: 2,048 random triangles + ground sphere + area light
  mixed()         1280x720, 64 spp, 8 bounces: 2,048 triangles + 128 spheres, mixed materials,
                  1024x512 procedural HDR sky with a sun disc, 16 emissive triangles
  large_mesh()    1920x1080, 256 spp, 8 bounces: 1024x1024 fBm heightfield (~2.1 M triangles)
                  + 512 glass/metal spheres + the mixed-scene sky

Every scene is a ``toaster_b200.scene.Scene`` and can be written as reference JSON.
"""

from __future__ import annotations

import math

import numpy as np

from . import gpu_types as gt
from .scene import EnvironmentMap, Material, Scene, box_triangles, triangle_is_valid


def _unit_vectors(rng: np.random.Generator, n: int) -> np.ndarray:
    z = rng.uniform(-1.0, 1.0, n)
    phi = rng.uniform(0.0, 2.0 * math.pi, n)
    r = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    return np.stack([r * np.cos(phi), r * np.sin(phi), z], axis=1)


def random_triangles(n: int, seed: int = 0, lo: float = 0.05, hi: float = 0.2) -> np.ndarray:
    """``n`` triangles: centre uniform in [-1,1]^3, each vertex at centre + L*u with L uniform in
    [lo, hi] and u a uniform unit vector; degenerate ones (loader.rs:1584-1593) are redrawn."""
    rng = np.random.default_rng(seed)
    out = np.zeros((n, 3, 3), np.float32)
    filled = 0
    while filled < n:
        m = n - filled
        c = rng.uniform(-1.0, 1.0, (m, 1, 3))
        lengths = rng.uniform(lo, hi, (m, 3, 1))
        dirs = _unit_vectors(rng, 3 * m).reshape(m, 3, 3)
        cand = (c + lengths * dirs).astype(np.float32)
        for k in range(m):
            if triangle_is_valid(cand[k]):
                out[filled] = cand[k]
                filled += 1
                if filled == n:
                    break
    return out


def area_light_quad(y: float = 2.0, size: float = 0.5):
    """A downward-facing square emitter centred on the y axis (two triangles)."""
    h = size / 2.0
    a, b, c, d = (-h, y, -h), (h, y, -h), (h, y, h), (-h, y, h)
    return np.array([[a, b, c], [a, c, d]], np.float32)


def sky_environment(width: int = 1024, height: int = 512, sun_elevation_deg: float = 35.0,
                    sun_azimuth_deg: float = 60.0, sun_diameter_deg: float = 0.5, sun_radiance: float = 1e4,
                    supersample: int = 4) -> EnvironmentMap:
    """Procedural FP32 sky: radiance 0.2 at and below the horizon rising to 1.0 at the zenith
    (tinted (0.8, 0.9, 1.0)), plus a sun disc of the given angular diameter and radiance whose
    texel values are its anti-aliased coverage (``supersample``^2 samples per texel). Texel
    directions follow environment.rs:176-181 (u = x / W, v = y / H, rotation 0)."""
    ys = (np.arange(height) + 0.5) / height
    theta = np.pi * ys
    value = 0.2 + 0.8 * np.maximum(0.0, np.cos(theta))
    img = np.empty((height, width, 3), np.float64)
    img[...] = value[:, None, None] * np.array([0.8, 0.9, 1.0])[None, None, :]
    el, az = math.radians(sun_elevation_deg), math.radians(sun_azimuth_deg)
    sun = np.array([math.cos(el) * math.cos(az), math.sin(el), math.cos(el) * math.sin(az)])
    cos_r = math.cos(math.radians(sun_diameter_deg / 2.0))
    # Only texels near the sun can be covered; scan a small window around it.
    sun_theta = math.acos(sun[1])
    sun_phi = math.atan2(sun[2], sun[0])
    cy = int(sun_theta / math.pi * height)
    cx = int(((sun_phi / (2 * math.pi) + 0.5) % 1.0) * width)
    win = max(4, int(math.ceil(sun_diameter_deg / 360.0 * width)) + 4)
    offs = (np.arange(supersample) + 0.5) / supersample
    for y in range(max(0, cy - win), min(height, cy + win + 1)):
        for xx in range(cx - win, cx + win + 1):
            x = xx % width
            u = (x + offs[None, :]) / width
            v = (y + offs[:, None]) / height
            th = np.pi * v
            ph = 2 * np.pi * (u - 0.5)
            d = np.stack([np.sin(th) * np.cos(ph), np.cos(th) * np.ones_like(ph), np.sin(th) * np.sin(ph)], -1)
            cover = float(np.mean(d @ sun >= cos_r))
            if cover > 0:
                img[y, x] += sun_radiance * cover
    return EnvironmentMap(width, height, img.astype(np.float32), 1.0, 0.0)


def plain_small(seed: int = 0) -> Scene:
    """320x180, 4 spp, 4 bounces, black background. 2,048 random triangles (seed 0) with
    per-triangle Lambertian albedo uniform in [0.2, 0.8]^3, a ground sphere (radius 1000, centre
    y = -1001, albedo 0.5) and a 0.5 x 0.5 emitter at y = 2 (colour 1, strength 15). Camera at
    (0, 0.5, 4) looking at the origin with a 40-degree vertical FOV (the position is a choice)."""
    rng = np.random.default_rng(seed + 1000)
    tris = random_triangles(2048, seed)
    albedo = rng.uniform(0.2, 0.8, (2048, 3))
    mats = [Material.diffuse(a, f"tri{i}") for i, a in enumerate(albedo)]
    mats.append(Material.diffuse((0.5, 0.5, 0.5), "ground"))
    mats.append(Material.emissive((1.0, 1.0, 1.0), 15.0, "light"))
    light = area_light_quad()
    all_tris = np.concatenate([tris, light])
    tri_mat = np.concatenate([np.arange(2048), [2049, 2049]]).astype(np.uint32)
    return Scene(
        camera_position=(0.0, 0.5, 4.0), camera_look_at=(0.0, 0.0, 0.0), fov_degrees=40.0,
        width=320, height=180, samples=4, max_bounces=4, background=gt.BLACK, materials=mats,
        sphere_centers=np.array([[0.0, -1001.0, 0.0]], np.float32), sphere_radii=np.array([1000.0], np.float32),
        sphere_materials=np.array([2048], np.uint32), triangles=all_tris, triangle_materials=tri_mat,
    )


def _mixed_materials(rng: np.random.Generator, n: int, prefix: str):
    """50% diffuse (albedo U[0.2,0.8]^3), 30% metal (albedo U[0.5,0.95]^3, roughness U[0,0.5]),
    20% dielectric (IOR 1.5), drawn independently per primitive."""
    mats = []
    kind = rng.uniform(0.0, 1.0, n)
    for i in range(n):
        if kind[i] < 0.5:
            mats.append(Material.diffuse(rng.uniform(0.2, 0.8, 3), f"{prefix}{i}"))
        elif kind[i] < 0.8:
            mats.append(Material.metal(rng.uniform(0.5, 0.95, 3), rng.uniform(0.0, 0.5), f"{prefix}{i}"))
        else:
            mats.append(Material.dielectric(1.5, f"{prefix}{i}"))
    return mats


def mixed(seed: int = 0, width: int = 1280, height: int = 720, samples: int = 64, max_bounces: int = 8,
          environment: EnvironmentMap | None = None) -> Scene:
    """The mixed scene: the 2,048 seeded triangles of plain_small plus 128 spheres (centre
    uniform in [-1,1]^3, radius uniform in [0.05, 0.3]); materials 50/30/20 diffuse / metal /
    dielectric per primitive; 16 of the triangles (seeded choice) are emitters with colour
    U[0.5,1]^3 and strength U[5,25], sampled by power; the procedural 1024x512 sky with a
    0.5-degree sun of radiance 1e4 lights the scene (environment background)."""
    rng = np.random.default_rng(seed + 2000)
    tris = random_triangles(2048, seed)
    tri_mats = _mixed_materials(rng, 2048, "t")
    emitters = rng.choice(2048, 16, replace=False)
    for k in emitters:
        tri_mats[k] = Material.emissive(rng.uniform(0.5, 1.0, 3), rng.uniform(5.0, 25.0), f"t{k}")
    centers = rng.uniform(-1.0, 1.0, (128, 3)).astype(np.float32)
    radii = rng.uniform(0.05, 0.3, 128).astype(np.float32)
    sph_mats = _mixed_materials(rng, 128, "s")
    mats = tri_mats + sph_mats
    return Scene(
        camera_position=(0.0, 0.5, 4.0), camera_look_at=(0.0, 0.0, 0.0), fov_degrees=40.0,
        width=width, height=height, samples=samples, max_bounces=max_bounces, background=gt.ENVIRONMENT,
        materials=mats, sphere_centers=centers, sphere_radii=radii,
        sphere_materials=np.arange(2048, 2048 + 128, dtype=np.uint32), triangles=tris,
        triangle_materials=np.arange(2048, dtype=np.uint32),
        environment=environment if environment is not None else sky_environment(),
    )


def parity_rays(scene: Scene, n: int = 1 << 20, seed: int = 0) -> np.ndarray:
    """Seeded ray set for the closest-hit check: half jittered primary rays through the scene's
    camera, half random rays with origins uniform in [-2,2]^3 and uniform directions. Directions
    are normalised in f32. Returns (n, 6) float32 (origin.xyz, direction.xyz)."""
    from .scene import make_camera

    rng = np.random.default_rng(seed + 3000)
    cam = make_camera(scene.camera_position, scene.camera_look_at, scene.camera_up, scene.fov_degrees,
                      scene.width / scene.height)[0]
    half = n // 2
    u = rng.uniform(0.0, 1.0, half).astype(np.float32)
    v = rng.uniform(0.0, 1.0, half).astype(np.float32)
    o = cam["origin"][:3]
    d = (cam["lower_left_corner"][:3][None, :] + u[:, None] * cam["horizontal"][:3][None, :]
         + v[:, None] * cam["vertical"][:3][None, :] - o[None, :]).astype(np.float32)
    primary = np.concatenate([np.broadcast_to(o, (half, 3)), d], axis=1)
    m = n - half
    orig = rng.uniform(-2.0, 2.0, (m, 3)).astype(np.float32)
    dirs = _unit_vectors(rng, m).astype(np.float32)
    rand = np.concatenate([orig, dirs], axis=1)
    rays = np.concatenate([primary, rand]).astype(np.float32)
    dd = rays[:, 3:]
    inv = (np.float32(1.0) / np.sqrt((dd * dd).sum(axis=1, dtype=np.float32))).astype(np.float32)
    rays[:, 3:] = dd * inv[:, None]
    return np.ascontiguousarray(rays)


def fbm_heights(n: int, octaves: int = 6, seed: int = 7, amplitude: float = 0.2) -> np.ndarray:
    """(n, n) fractional Brownian motion of value noise: octave k has frequency 2^k over the
    unit square and weight 0.5^k; normalised to [-amplitude, amplitude]."""
    rng = np.random.default_rng(seed)
    xs = np.linspace(0.0, 1.0, n)
    total = np.zeros((n, n))
    for k in range(octaves):
        freq = 4 * (2 ** k)
        grid = rng.uniform(-1.0, 1.0, (freq + 2, freq + 2))
        gx = xs * freq
        i0 = np.floor(gx).astype(int)
        f = gx - i0
        f = f * f * (3 - 2 * f)
        a = grid[np.ix_(i0, i0)]
        b = grid[np.ix_(i0, i0 + 1)]
        c = grid[np.ix_(i0 + 1, i0)]
        d = grid[np.ix_(i0 + 1, i0 + 1)]
        fy, fx = f[:, None], f[None, :]
        total += (0.5 ** k) * ((a * (1 - fx) + b * fx) * (1 - fy) + (c * (1 - fx) + d * fx) * fy)
    total /= np.abs(total).max()
    return (amplitude * total).astype(np.float32)


def heightfield_triangles(heights: np.ndarray, extent: float = 4.0) -> np.ndarray:
    """Two triangles per grid cell over [-extent, extent]^2 (the cell split of the reference's
    benchmark terrain, scripts/generate_benchmark_scenes.py:71-80)."""
    n = heights.shape[0]
    xs = np.linspace(-extent, extent, n, dtype=np.float64)
    gx, gz = np.meshgrid(xs, xs)
    pos = np.stack([gx, heights.astype(np.float64), gz], -1).astype(np.float32)
    ll = pos[:-1, :-1].reshape(-1, 3)
    lr = pos[:-1, 1:].reshape(-1, 3)
    ul = pos[1:, :-1].reshape(-1, 3)
    ur = pos[1:, 1:].reshape(-1, 3)
    t1 = np.stack([ll, ul, lr], 1)
    t2 = np.stack([lr, ul, ur], 1)
    return np.ascontiguousarray(np.stack([t1, t2], 1).reshape(-1, 3, 3))


def large_mesh(seed: int = 7, grid: int = 1024, width: int = 1920, height: int = 1080, samples: int = 256,
               max_bounces: int = 8, environment: EnvironmentMap | None = None) -> Scene:
    """Heightfield terrain on a ``grid`` x ``grid`` vertex lattice (2*(grid-1)^2 triangles) with
    fBm heights (6 octaves, seed 7, amplitude 0.2) over [-4,4]^2, diffuse albedo 0.55; 512 spheres
    (radius U[0.05,0.25], half glass IOR 1.5, half metal roughness U[0,0.3]) resting on it; the
    mixed-scene sky."""
    rng = np.random.default_rng(seed + 4000)
    h = fbm_heights(grid, seed=seed)
    tris = heightfield_triangles(h)
    mats = [Material.diffuse((0.55, 0.55, 0.55), "terrain")]
    n_sph = 512
    radii = rng.uniform(0.05, 0.25, n_sph).astype(np.float32)
    xz = rng.uniform(-3.5, 3.5, (n_sph, 2))
    ix = np.clip(((xz + 4.0) / 8.0 * (grid - 1)).round().astype(int), 0, grid - 1)
    y = h[ix[:, 1], ix[:, 0]] + radii
    centers = np.stack([xz[:, 0], y, xz[:, 1]], 1).astype(np.float32)
    sph_mat = []
    for i in range(n_sph):
        if i % 2 == 0:
            mats.append(Material.dielectric(1.5, f"s{i}"))
        else:
            mats.append(Material.metal(rng.uniform(0.6, 0.95, 3), rng.uniform(0.0, 0.3), f"s{i}"))
        sph_mat.append(len(mats) - 1)
    return Scene(
        camera_position=(0.0, 1.6, 5.5), camera_look_at=(0.0, 0.0, 0.0), fov_degrees=45.0,
        width=width, height=height, samples=samples, max_bounces=max_bounces, background=gt.ENVIRONMENT,
        materials=mats, sphere_centers=centers, sphere_radii=radii, sphere_materials=np.array(sph_mat, np.uint32),
        triangles=tris, triangle_materials=np.zeros(tris.shape[0], np.uint32),
        environment=environment if environment is not None else sky_environment(),
    )


def _quad(a, b, c, d):
    """Two triangles of the quad a-b-c-d (counter-clockwise)."""
    return [[a, b, c], [a, c, d]]


def room_with_window(seed: int = 0, width: int = 1280, height: int = 720, samples: int = 16, max_bounces: int = 8,
                     clutter: int = 8192, environment: EnvironmentMap | None = None,
                     metal_fraction: float = 0.3) -> Scene:
    """Hard-lighting interior: a closed 4 x 3 x 4 room (x, z in [-2, 2], y in [0, 3]) whose only
    opening is a 0.4 x 0.4 window in the +z wall (x in [0.3, 0.7], y in [1.6, 2.0]); it is lit only
    by the mixed-scene sky and sun through that window. Walls 0.7, floor 0.5, ceiling 0.8 diffuse.
    ``clutter`` seeded triangles (centre uniform in [-1.8, 1.8] x [0.1, 2.5] x [-1.8, 1.6], edges as in
    random_triangles) are 70% diffuse (albedo U[0.2, 0.8]^3) and 30% metal (albedo U[0.5, 0.95]^3,
    roughness U[0, 0.5]); ``metal_fraction`` changes that split. The camera stands near the -z wall
    looking toward the window wall."""
    rng = np.random.default_rng(seed + 5000)
    x0, x1, y0, y1, z0, z1 = -2.0, 2.0, 0.0, 3.0, -2.0, 2.0
    wx0, wx1, wy0, wy1 = 0.3, 0.7, 1.6, 2.0
    shell = []
    shell += _quad((x0, y0, z0), (x1, y0, z0), (x1, y0, z1), (x0, y0, z1))  # floor
    shell += _quad((x0, y1, z0), (x0, y1, z1), (x1, y1, z1), (x1, y1, z0))  # ceiling
    shell += _quad((x0, y0, z0), (x0, y1, z0), (x1, y1, z0), (x1, y0, z0))  # -z wall
    shell += _quad((x0, y0, z0), (x0, y0, z1), (x0, y1, z1), (x0, y1, z0))  # -x wall
    shell += _quad((x1, y0, z0), (x1, y1, z0), (x1, y1, z1), (x1, y0, z1))  # +x wall
    # +z wall with the window cut out: below, above, left and right of the opening.
    shell += _quad((x0, y0, z1), (x1, y0, z1), (x1, wy0, z1), (x0, wy0, z1))
    shell += _quad((x0, wy1, z1), (x1, wy1, z1), (x1, y1, z1), (x0, y1, z1))
    shell += _quad((x0, wy0, z1), (wx0, wy0, z1), (wx0, wy1, z1), (x0, wy1, z1))
    shell += _quad((wx1, wy0, z1), (x1, wy0, z1), (x1, wy1, z1), (wx1, wy1, z1))
    shell = np.array(shell, np.float32)
    shell_mat = np.array([0, 0, 1, 1] + [2] * 14, np.uint32)  # floor, ceiling, walls
    mats = [Material.diffuse((0.5, 0.5, 0.5), "floor"), Material.diffuse((0.8, 0.8, 0.8), "ceiling"),
            Material.diffuse((0.7, 0.7, 0.7), "walls")]
    tris = random_triangles(clutter, seed + 1)
    lo = np.array([-1.8, 0.1, -1.8]); hi = np.array([1.8, 2.5, 1.6])
    centre = tris.mean(axis=1, keepdims=True)
    tris = (tris - centre + (lo + (centre + 1.0) / 2.0 * (hi - lo))).astype(np.float32)
    kinds = rng.uniform(0, 1, clutter)
    clutter_mat = []
    for i in range(clutter):
        if kinds[i] >= metal_fraction:
            mats.append(Material.diffuse(rng.uniform(0.2, 0.8, 3), f"c{i}"))
        else:
            mats.append(Material.metal(rng.uniform(0.5, 0.95, 3), rng.uniform(0.0, 0.5), f"c{i}"))
        clutter_mat.append(len(mats) - 1)
    return Scene(
        camera_position=(-1.0, 1.5, -1.8), camera_look_at=(0.5, 1.2, 1.0), fov_degrees=60.0,
        width=width, height=height, samples=samples, max_bounces=max_bounces, background=gt.ENVIRONMENT,
        materials=mats, triangles=np.concatenate([shell, tris]),
        triangle_materials=np.concatenate([shell_mat, np.array(clutter_mat, np.uint32)]),
        environment=environment if environment is not None else sky_environment(),
    )


def scene_bounds(scene: Scene):
    """(centre xyz, scale) mapping the scene's bounding box into [-1, 1] (guiding encoding frame)."""
    pts = [scene.triangles.reshape(-1, 3)] if scene.triangle_count else []
    if scene.sphere_count:
        r = scene.sphere_radii[:, None]
        pts += [scene.sphere_centers - r, scene.sphere_centers + r]
    allp = np.concatenate(pts).astype(np.float64)
    lo, hi = allp.min(0), allp.max(0)
    centre = (lo + hi) / 2
    half = max(float((hi - lo).max()) / 2, 1e-6)
    return (float(centre[0]), float(centre[1]), float(centre[2]), 1.0 / half)


class BallisticAnimation:
    """240 frames (24 fps, 10 s) of 64 spheres and 64 axis-aligned boxes thrown on seeded ballistic
    trajectories over a ground quad, bouncing with restitution 0.8. Four spheres are emitters
    (moving lights); materials are 50/30/20 diffuse / metal / dielectric otherwise. Lit by the mixed
    scene's sky. Positions are integrated in double precision with 8 sub-steps per frame and stored
    as f32 per frame, so frame k is a pure function of (seed, k)."""

    def __init__(self, seed: int = 0, width: int = 1280, height: int = 720, samples: int = 32, max_bounces: int = 8,
                 frames: int = 240, fps: float = 24.0, environment: EnvironmentMap | None = None):
        rng = np.random.default_rng(seed + 9000)
        self.frames, self.fps = frames, fps
        self.n_spheres, self.n_boxes = 64, 64
        n = self.n_spheres + self.n_boxes
        self.radius = np.concatenate([rng.uniform(0.1, 0.3, self.n_spheres), rng.uniform(0.1, 0.4, self.n_boxes) / 2])
        self.box_size = 2.0 * self.radius[self.n_spheres:]
        self.p0 = np.stack([rng.uniform(-3, 3, n), rng.uniform(0.5, 3.0, n), rng.uniform(-3, 3, n)], -1)
        self.v0 = np.stack([rng.uniform(-2, 2, n), rng.uniform(2, 6, n), rng.uniform(-2, 2, n)], -1)
        mats = [Material.diffuse((0.5, 0.5, 0.5), "ground")]
        kinds = rng.uniform(0, 1, n)
        self.mat = np.zeros(n, np.uint32)
        for i in range(n):
            if i < 4:
                mats.append(Material.emissive(rng.uniform(0.6, 1.0, 3), 20.0, f"e{i}"))
            elif kinds[i] < 0.5:
                mats.append(Material.diffuse(rng.uniform(0.2, 0.8, 3), f"d{i}"))
            elif kinds[i] < 0.8:
                mats.append(Material.metal(rng.uniform(0.5, 0.95, 3), rng.uniform(0.0, 0.5), f"m{i}"))
            else:
                mats.append(Material.dielectric(1.5, f"g{i}"))
            self.mat[i] = len(mats) - 1
        self.materials = mats
        self.width, self.height, self.samples, self.max_bounces = width, height, samples, max_bounces
        self.environment = environment if environment is not None else sky_environment()
        self._positions = self._simulate()

    def _simulate(self) -> np.ndarray:
        n = self.p0.shape[0]
        pos = np.empty((self.frames, n, 3), np.float64)
        p, v = self.p0.copy(), self.v0.copy()
        g = np.array([0.0, -9.81, 0.0])
        sub = 8
        dt = 1.0 / (self.fps * sub)
        for f in range(self.frames):
            pos[f] = p
            for _ in range(sub):
                v = v + g * dt
                p = p + v * dt
                low = p[:, 1] < self.radius
                p[low, 1] = self.radius[low]
                v[low, 1] = np.abs(v[low, 1]) * 0.8
        return pos

    def scene(self, frame: int) -> Scene:
        p = self._positions[frame].astype(np.float32)
        ns = self.n_spheres
        ground = np.array(_quad((-10, 0, -10), (-10, 0, 10), (10, 0, 10), (10, 0, -10)), np.float32)
        boxes = [box_triangles(p[ns + i], (self.box_size[i],) * 3) for i in range(self.n_boxes)]
        tris = np.concatenate([ground] + boxes).astype(np.float32)
        tri_mat = np.concatenate([np.zeros(2, np.uint32), np.repeat(self.mat[ns:], 12)])
        return Scene(camera_position=(0.0, 3.0, 10.0), camera_look_at=(0.0, 1.0, 0.0), fov_degrees=45.0,
                     width=self.width, height=self.height, samples=self.samples, max_bounces=self.max_bounces,
                     background=gt.ENVIRONMENT, materials=self.materials, sphere_centers=p[:ns],
                     sphere_radii=self.radius[:ns].astype(np.float32), sphere_materials=self.mat[:ns],
                     triangles=tris, triangle_materials=tri_mat, environment=self.environment)


def uneven_batch(seed: int = 0, count: int = 16, samples: int = 32, max_bounces: int = 8,
                 environment: EnvironmentMap | None = None, min_width: int = 320, max_width: int = 1280) -> list:
    """``count`` independent scenes for one batched launch: triangle counts log-uniform in
    [128, 262,144] (seeded random triangles as in random_triangles, scaled to a 4-unit cube, half
    diffuse, a quarter metal, a quarter dielectric, plus a ground sphere) and resolutions
    log-uniform between min_width and max_width (16:9, width a multiple of 16; 320x180 to
    1280x720 by default), lit by the mixed scene's sky."""
    rng = np.random.default_rng(seed + 7000)
    env = environment if environment is not None else sky_environment()
    out = []
    for i in range(count):
        n_tri = int(round(math.exp(rng.uniform(math.log(128), math.log(262144)))))
        width = int(round(math.exp(rng.uniform(math.log(min_width), math.log(max_width))) / 16)) * 16
        height = width * 9 // 16
        tris = random_triangles(n_tri, seed=seed * 100 + i) * np.float32(2.0)
        kinds = rng.uniform(0, 1, n_tri)
        mats = [Material.diffuse((0.5, 0.5, 0.5), "ground"), Material.diffuse((0.6, 0.5, 0.4), "d"),
                Material.metal((0.8, 0.8, 0.8), 0.2, "m"), Material.dielectric(1.5, "g")]
        tri_mat = np.where(kinds < 0.5, 1, np.where(kinds < 0.75, 2, 3)).astype(np.uint32)
        out.append(Scene(camera_position=(0.0, 1.0, 7.0), camera_look_at=(0.0, 0.0, 0.0), fov_degrees=45.0,
                         width=width, height=height, samples=samples, max_bounces=max_bounces,
                         background=gt.ENVIRONMENT, materials=mats,
                         sphere_centers=np.array([[0.0, -1002.0, 0.0]], np.float32),
                         sphere_radii=np.array([1000.0], np.float32), sphere_materials=np.zeros(1, np.uint32),
                         triangles=tris, triangle_materials=tri_mat, environment=env))
    return out
