"""The algorithmic work figures bench.py reports its path rooflines against,
recomputed with the oracle (the reference's own traversal order and scene
query, code/Bvh/Bvh.cpp:353-444, code/Renderer.cpp:891-949).

* BVH-fetch bytes per ray of the batched-mesh workload's two scenes: every
  ray the reference estimator casts on the scene (camera, continuation and
  shadow rays; depth 8, 4 shadow rays, hero-4 spectral) is counted with the
  reference traversal: 48 B (two 24 B child boxes) per internal node
  processed plus 36 B (three vertices) per leaf triangle tested.  The ray
  distribution does not depend on the resolution (a finer grid samples the
  same field of view), so 64x64 at 4 paths per pixel stands for the
  workload's 512..1024 squares.
* Plane tests per ray of cornell: the reference tests all 18 planes for
  every ray.
"""
import os
import sys

import pytest

from conftest import GOLDEN, REPO, scene_path

sys.path.insert(0, REPO)


@pytest.mark.parametrize("glass", [False, True])
def test_bvh_bytes_per_ray_match_bench_constant(oracle_lib, glass):
    import bench
    from pcr_b200 import workloads
    O = oracle_lib
    sc = O.load_scene(workloads.mesh_scene(59, 21 + int(glass), glass=glass), GOLDEN)
    c = O.count_render_paths(sc, O.opts(64, depth=8, shadow=4, spectral=True, seed=3), 4, threads=os.cpu_count())
    per_ray = (48 * c["bvh_nodes"] + 36 * c["bvh_tris"]) / c["rays"]
    want = bench.BVH_BYTES_PER_RAY["ico59-glass" if glass else "ico59-diffuse"]
    assert abs(per_ray - want) <= 0.02 * want, (per_ray, want, c)
    assert c["plane_tests"] == c["rays"] * 6   # the five walls and the light


def test_cornell_tests_every_plane_per_ray(oracle_lib):
    O = oracle_lib
    sc = O.load_scene(scene_path("cornell"), GOLDEN)
    c = O.count_render_paths(sc, O.opts(32, depth=4, shadow=4, spectral=True, seed=3), 4, threads=os.cpu_count())
    assert c["rays"] > 32 * 32 * 4 and c["plane_tests"] == 18 * c["rays"] and c["bvh_nodes"] == 0
