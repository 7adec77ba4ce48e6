"""The regenerated benchmark suite (toaster_b200.bench_fixtures) (CPU).

Its scene and glTF files must equal the reference's own fixtures byte for byte where those are
present, and they load through the native loader with the geometry counts the reference's loader
test expects (crates/toaster-scene/src/loader.rs:1891-1916).
"""

import pytest
from conftest import reference_checkout

from toaster_b200.bench_fixtures import SCENES, write_suite
from toaster_b200.scene import load_scene_gpu

REFERENCE = reference_checkout()
COUNTS = [(128, 1, False), (2048, 1, False), (8192, 1, False), (2, 65, False), (2, 513, False), (2048, 129, False),
          (0, 4, True)]


def test_suite_loads_with_the_reference_counts(tmp_path):
    scenes = write_suite(tmp_path)
    for name, (tris, spheres, env) in zip(SCENES, COUNTS):
        data, _ = load_scene_gpu(scenes / name)
        p = data.params[0]
        assert (p["triangle_count"], p["sphere_count"], p["background_kind"] == 2) == (tris, spheres, env), name
        assert (p["width"], p["height"], p["samples"], p["max_bounces"]) == (320, 180, 4, 4)


@pytest.mark.skipif(not (REFERENCE / "scenes" / "benchmarks").is_dir(), reason="the reference's fixtures are not present")
def test_suite_files_equal_the_reference_fixtures(tmp_path):
    write_suite(tmp_path)
    for name in SCENES:
        assert (tmp_path / "scenes/benchmarks" / name).read_bytes() == (REFERENCE / "scenes/benchmarks" / name).read_bytes()
    for n in (8, 32, 64):
        rel = f"assets/benchmarks/terrain_grid_{n}.gltf"
        assert (tmp_path / rel).read_bytes() == (REFERENCE / rel).read_bytes()
