"""Pins the CPU restatement oracle (oracle/pcr_oracle.c) before anything is
checked against it: the reference's own 17 golden PNGs (tests/render/run.sh
tuples, `-d 2 -s 4 -S 2 -w 120 --seed 12345`) must come out bit-exact, and
the BVH builder/traversal must reproduce the reference's node arrays and hit
answers committed in tests/golden/bvh_vectors.npz."""
import os

import numpy as np
import pytest

from conftest import BUNNY_SCENE, GOLDEN, have_bunny, scene_path

# (golden name, scene, renderer knobs) from the reference's render suite
GOLDENS = [
    ("cornell-rgb", "cornell", {}),
    ("cornell-spectral", "cornell", {"spectral": True}),
    ("cornell-spectral-hero1", "cornell", {"spectral": True, "hero": 1}),
    ("cornell-glass-rgb", "cornell-glass", {}),
    ("cornell-glass-spectral", "cornell-glass", {"spectral": True}),
    ("cornell-spheres-rgb", "cornell-spheres", {}),
    ("cornell-large-light-rgb", "cornell-large-light", {}),
    ("cornell-spec-rgb", "cornell-spec", {}),
    ("cornell-rgb-denoise", "cornell", {"denoise": True}),
    ("cornell-rgb-aces", "cornell", {"aces": True}),
    ("cornell-rgb-mis-russian-stratified", "cornell", {"mis": True, "russian": True, "stratified": True}),
    ("cornell-rgb-aa4", "cornell", {"aa": 4}),
    ("cornell-rgb-adaptive-aa8", "cornell", {"aa": 8, "adaptive": True}),
]


def _golden(name):
    from PIL import Image
    return np.asarray(Image.open(os.path.join(GOLDEN, "render", name + ".png")).convert("RGB"))


@pytest.mark.parametrize("name,scene,kw", GOLDENS, ids=[g[0] for g in GOLDENS])
def test_oracle_reproduces_golden(oracle_lib, name, scene, kw):
    O = oracle_lib
    sc = O.load_scene(scene_path(scene), GOLDEN)
    _, rgb = O.render(sc, O.opts(120, **kw))
    assert np.array_equal(rgb, _golden(name))


@pytest.fixture(scope="module")
def built_lut(oracle_lib):
    lut = np.zeros(3 * 16 ** 3 * 3, np.float32)
    oracle_lib.lib().oracle_lut_build(oracle_lib.fptr(lut))
    return lut


@pytest.mark.parametrize("name", ["cornell-spectral-lut", "cornell-spectral-lut-file"])
def test_oracle_lut_goldens(oracle_lib, built_lut, name):
    O = oracle_lib
    sc = O.load_scene(scene_path("cornell"), GOLDEN, lut=built_lut)
    _, rgb = O.render(sc, O.opts(120, spectral=True))
    assert np.array_equal(rgb, _golden(name))


def test_oracle_lut_matches_shipped_plut(built_lut):
    path = os.path.join(GOLDEN, "luts", "default-kres16.lut")
    raw = open(path, "rb").read()
    assert raw[:4] == b"PLUT"
    assert np.array_equal(np.frombuffer(raw[16:], np.float32).view(np.uint32), built_lut.view(np.uint32))


@pytest.mark.parametrize("name,kw", [("cornell-bunny-rgb", {}), ("cornell-bunny-spectral", {"spectral": True})])
def test_oracle_bunny_goldens(oracle_lib, name, kw):
    O = oracle_lib
    assert have_bunny(), "the Stanford bunny fixture (tests/golden/models) is missing"
    sc = O.load_scene(BUNNY_SCENE, GOLDEN)
    _, rgb = O.render(sc, O.opts(120, **kw))
    assert np.array_equal(rgb, _golden(name))


@pytest.mark.parametrize("name", ["soup200", "soup5k", "coplanar"])
def test_oracle_bvh_build_matches_reference_vectors(oracle_lib, name):
    v = np.load(os.path.join(GOLDEN, "bvh_vectors.npz"))
    boxes, ints, perm, _, _ = oracle_lib.bvh_build(v[f"{name}_tris"])
    assert np.array_equal(boxes, v[f"{name}_boxes"])
    assert np.array_equal(ints, v[f"{name}_ints"])
    assert np.array_equal(perm, v[f"{name}_perm"])


@pytest.mark.parametrize("name", ["soup200", "soup5k"])
def test_oracle_bvh_query_matches_reference_vectors(oracle_lib, name):
    v = np.load(os.path.join(GOLDEN, "bvh_vectors.npz"))
    _, _, _, arr, nodes = oracle_lib.bvh_build(v[f"{name}_tris"])
    hid, ht = oracle_lib.bvh_query(nodes, arr, v[f"{name}_rays"])
    assert np.array_equal(hid, v[f"{name}_hit"])
    assert np.array_equal(ht, v[f"{name}_t"])
