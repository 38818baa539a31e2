"""CPU tests of the product's host side: the C ABI library loads and exports
every symbol include/pcr_cuda.h declares, and the library's own scene
loader (JSONC, SPD, sigmoid fit, SAH BVH) produces arrays bit-identical to
the reference loader's (code/Scenes/SceneLoader.cpp:475-516), checked
against the compiled reference where it is present and against the CPU
restatement oracle everywhere."""
import os
import re

import numpy as np
import pytest

from conftest import BUNNY_SCENE, GOLDEN, REPO, have_bunny, scene_path

SCENES = ["cornell", "cornell-spec", "cornell-glass", "cornell-spheres", "closed-cornell-spec",
          "cornell-large-light", "bright-cornell-glass", "closed-cornell-glass", "cornell-frank"]


@pytest.fixture(scope="module")
def capi():
    from pcr_b200 import build, capi as c
    build.build()
    return c


def test_library_exports_every_declared_symbol(capi):
    header = open(os.path.join(REPO, "include", "pcr_cuda.h")).read()
    declared = set(re.findall(r"\b(pcr_[a-z0-9_]+)\s*\(", header))
    lib = capi.load_library()
    for name in declared:
        assert hasattr(lib, name), f"{name} declared in include/pcr_cuda.h but not exported"
    assert declared == set(capi.EXPORTS)


def _material_rows(hs):
    m = hs.materials().copy()
    mi = m.view(np.int32)
    # reorder to the oracle/reference export order: albedo3 emissive3 metallic
    # transparent ior cauchyB useTabA useTabE fits tabs
    return np.concatenate([m[:, :6], mi[:, 6:8].astype(np.float32), m[:, 10:12],
                           mi[:, 8:10].astype(np.float32), m[:, 12:]], 1)


@pytest.mark.parametrize("name", SCENES)
def test_host_loader_matches_oracle_loader(capi, oracle_lib, name):
    hs = capi.HostScene(scene_path(name), GOLDEN)
    osc = oracle_lib.load_scene(scene_path(name), GOLDEN)
    assert np.array_equal(_material_rows(hs).view(np.uint32), osc.material_table().view(np.uint32))
    p = hs.planes()
    q = osc.plane_table()
    assert np.array_equal(p[:, :13].view(np.uint32), q[:, :13].view(np.uint32))
    assert np.array_equal(p[:, 13].view(np.int32), q[:, 13].astype(np.int32))


@pytest.mark.parametrize("name", SCENES)
def test_host_loader_matches_reference_loader(capi, name):
    from oracle import ref
    if not ref.available():
        pytest.skip("reference harness not built")
    path = os.path.abspath(scene_path(name))
    hs = capi.HostScene(path, GOLDEN)
    rs = ref.load_scene(path, GOLDEN)
    assert np.array_equal(_material_rows(hs).view(np.uint32), rs.materials.view(np.uint32))
    assert np.array_equal(hs.planes()[:, :13].view(np.uint32), rs.planes[:, :13].view(np.uint32))


def test_host_loader_bunny_bvh_matches_reference(capi):
    from oracle import ref
    if not ref.available():
        pytest.skip("reference harness not built")
    assert have_bunny(), "the Stanford bunny fixture (tests/golden/models) is missing"
    hs = capi.HostScene(BUNNY_SCENE, GOLDEN)
    rs = ref.load_scene(BUNNY_SCENE, GOLDEN)
    assert np.array_equal(hs.triangles()[:, :21].view(np.uint32), rs.triangles[:, :21].view(np.uint32))
    b = hs.bvh()
    assert np.array_equal(b[:, :6].view(np.uint32), rs.bvh_boxes.view(np.uint32))
    assert np.array_equal(b[:, 6:].view(np.int32), rs.bvh_ints)


def test_fit_sigmoid_matches_oracle(capi, oracle_lib):
    rng = np.random.default_rng(5)
    rgb = np.concatenate([rng.uniform(0, 1, (64, 3)), [[0, 0, 0], [1, 1, 1], [0.63, 0.06, 0.05],
                                                       [2, -1, 0.5]]]).astype(np.float32)
    mine = capi.fit_sigmoid(rgb)
    ref = np.zeros_like(mine)
    for i in range(rgb.shape[0]):
        oracle_lib.lib().oracle_fit_sigmoid(oracle_lib.fptr(rgb[i].copy()), None, oracle_lib.fptr(ref[i]))
    assert np.array_equal(mine.view(np.uint32), ref.view(np.uint32))


def test_lut_build_and_lookup_match_oracle(capi, oracle_lib):
    lut = capi.lut_build()
    ol = np.zeros_like(lut)
    oracle_lib.lib().oracle_lut_build(oracle_lib.fptr(ol))
    assert np.array_equal(lut.view(np.uint32), ol.view(np.uint32))
    rng = np.random.default_rng(9)
    rgb = rng.uniform(0, 1, (256, 3)).astype(np.float32)
    mine = capi.fit_sigmoid(rgb, lut)
    ref = np.zeros_like(mine)
    for i in range(rgb.shape[0]):
        oracle_lib.lib().oracle_lut_lookup(oracle_lib.fptr(ol), oracle_lib.fptr(rgb[i].copy()), oracle_lib.fptr(ref[i]))
    assert np.array_equal(mine.view(np.uint32), ref.view(np.uint32))


@pytest.mark.parametrize("name", ["soup200", "soup5k", "coplanar"])
def test_product_bvh_build_matches_reference_vectors(capi, tmp_path, name):
    """Scene upload builds the BVH with the library's builder; check that
    builder through a mesh scene against the reference's node arrays."""
    v = np.load(os.path.join(GOLDEN, "bvh_vectors.npz"))
    tris = v[f"{name}_tris"]
    obj = tmp_path / "m.obj"
    with open(obj, "w") as f:
        for t in tris:
            for k in range(3):
                f.write("v %.9g %.9g %.9g\n" % tuple(t[k * 3:k * 3 + 3]))
        for i in range(len(tris)):
            f.write(f"f {3 * i + 1} {3 * i + 2} {3 * i + 3}\n")
    scene = tmp_path / "s.json"
    scene.write_text('{"schema": "1.0", "name": "m", "version": "1", "materials": {"w": {"albedo": [0.5,0.5,0.5]},'
                     ' "l": {"emissive": [1,1,1]}}, "primitives": [{"type": "mesh", "file": "m.obj", "material": "w"},'
                     ' {"type": "plane", "light": true, "origin": [0,2,0], "u": [1,0,0], "v": [0,0,1], "material": "l"}]}')
    hs = capi.HostScene(str(scene), str(tmp_path))
    b = hs.bvh()
    assert np.array_equal(b[:, :6].view(np.uint32), v[f"{name}_boxes"].view(np.uint32))
    assert np.array_equal(b[:, 6:].view(np.int32), v[f"{name}_ints"])
    assert np.array_equal(hs.triangle_ids(), v[f"{name}_perm"])


def test_loader_errors_are_reported(capi, tmp_path):
    bad = tmp_path / "bad.json"
    bad.write_text('{"schema": "2.0", "name": "x", "version": "1", "materials": {}, "primitives": []}')
    with pytest.raises(capi.PcrError) as e:
        capi.HostScene(str(bad))
    assert e.value.status == 5 and "schema major version 2" in str(e.value)
    nolight = tmp_path / "nolight.json"
    nolight.write_text('{"schema": "1.0", "name": "x", "version": "1", "materials": {"a": {"albedo": [1,1,1]}},'
                       ' "primitives": [{"type": "plane", "origin": [0,0,0], "u": [1,0,0], "v": [0,1,0], "material": "a"}]}')
    with pytest.raises(capi.PcrError) as e:
        capi.HostScene(str(nolight))
    assert "at least one primitive" in str(e.value)
    with pytest.raises(capi.PcrError):
        capi.HostScene(str(tmp_path / "missing.json"))


def test_parallel_host_bvh_build_matches_oracle_on_200k_triangles(capi):
    """Ranges above 65,536 triangles are binned by several threads and large
    sibling subtrees are built concurrently; the node arrays and the
    triangle order must equal the oracle's sequential restatement of the
    reference builder."""
    from oracle import oracle as O
    from pcr_b200 import workloads
    O.build()
    path = workloads.mesh_scene(100, 5)
    hs = capi.HostScene(path, GOLDEN)
    tl, ids = hs.triangles(), hs.triangle_ids()
    assert tl.shape[0] == 200_000
    tris = np.zeros((tl.shape[0], 9), np.float32)
    tris[ids] = tl[:, :9]
    boxes, ints, perm, _, _ = O.bvh_build(tris)
    b = hs.bvh()
    assert np.array_equal(b[:, :6].view(np.uint32), boxes.view(np.uint32))
    assert np.array_equal(b[:, 6:].view(np.int32), ints)
    assert np.array_equal(ids, perm)


def test_parallel_obj_reader_matches_oracle_reader(capi, tmp_path):
    """An OBJ over 1 MB is read by several threads in ranges of lines:
    relative (negative) indices, polygon fans, v//n and v/t/n tokens, signed
    and exponent number forms, and vertices interleaved with faces across
    range boundaries must give the triangles a sequential reader gives."""
    from oracle import oracle as O
    O.build()
    rng = np.random.default_rng(21)
    lines = []
    nv = nn = 0
    while len(lines) < 60000:
        k = int(rng.integers(3, 6))
        for _ in range(k):
            x = rng.uniform(-1, 1, 3)
            fmt = rng.integers(0, 3)
            if fmt == 0:
                lines.append("v %.9g %.9g %.9g" % tuple(x))
            elif fmt == 1:
                lines.append("v %+.6e %+.6e %+.6e" % tuple(x))
            else:
                lines.append("v  %.4f\t%.4f %.4f " % tuple(x))
            n = rng.normal(size=3)
            lines.append("vn %.7f %.7f %.7f" % tuple(n / np.linalg.norm(n)))
            nv += 1
            nn += 1
        form = rng.integers(0, 4)
        toks = []
        for j in range(k):
            vi = nv - k + j + 1
            ni = nn - k + j + 1
            if form == 0:
                toks.append(str(vi))
            elif form == 1:
                toks.append(f"{vi - nv - 1}//{ni - nn - 1}")   # relative
            elif form == 2:
                toks.append(f"{vi}/1/{ni}")
            else:
                toks.append(f"{vi}//{ni}")
        lines.append("f " + " ".join(toks))
        if rng.random() < 0.01:
            lines.append("# comment line")
    obj = tmp_path / "m.obj"
    obj.write_text("vt 0 0\n" + "\n".join(lines) + "\n")
    assert obj.stat().st_size > (1 << 20)
    scene = tmp_path / "s.json"
    scene.write_text('{"schema": "1.0", "name": "m", "version": "1", "materials": {"w": {"albedo": [0.5,0.5,0.5]},'
                     ' "l": {"emissive": [1,1,1]}}, "primitives": [{"type": "mesh", "file": "m.obj", "material": "w",'
                     ' "position": [0.1, -0.2, -3], "rotation": [10, 20, 30], "scale": 0.7},'
                     ' {"type": "plane", "light": true, "origin": [0,2,0], "u": [1,0,0], "v": [0,0,1], "material": "l"}]}')
    hs = capi.HostScene(str(scene), str(tmp_path))
    osc = O.load_scene(str(scene), str(tmp_path))
    mine = hs.triangles()   # both in BVH-leaf order
    ref = np.array([np.concatenate([np.asarray(t.v0), t.v1, t.v2, t.n0, t.n1, t.n2, t.flatN]).astype(np.float32)
                    for t in osc.triangles])
    assert mine.shape[0] == ref.shape[0] > 10000
    assert np.array_equal(mine[:, :21].view(np.uint32), ref.view(np.uint32))
    assert np.array_equal(mine[:, 21].view(np.int32), np.array([t.smooth for t in osc.triangles], np.int32))
    hs.close()


def test_obj_normal_index_out_of_range_is_an_error(capi, tmp_path):
    obj = tmp_path / "m.obj"
    obj.write_text("v 0 0 0\nv 1 0 0\nv 0 1 0\nvn 0 0 1\nf 1//1 2//1 3//2\n")
    scene = tmp_path / "s.json"
    scene.write_text('{"schema": "1.0", "name": "m", "version": "1", "materials": {"w": {"albedo": [0.5,0.5,0.5]},'
                     ' "l": {"emissive": [1,1,1]}}, "primitives": [{"type": "mesh", "file": "m.obj", "material": "w"},'
                     ' {"type": "plane", "light": true, "origin": [0,2,0], "u": [1,0,0], "v": [0,0,1], "material": "l"}]}')
    with pytest.raises(capi.PcrError) as e:
        capi.HostScene(str(scene), str(tmp_path))
    assert "normal index out of range" in str(e.value)


def test_parallel_obj_reader_reports_a_bad_index(capi, tmp_path):
    """A face that names a vertex defined only later in the file is an error
    for a sequential reader; the ranges-of-lines reader must report it too
    when the face and the vertex sit in different ranges of a >1 MB file."""
    lines = []
    for i in range(40000):
        lines.append("v %.6f %.6f %.6f" % (i * 1e-3, (i % 7) * 0.1, -1.0))
    for i in range(1, 13000):
        lines.append(f"f {3 * i - 2} {3 * i - 1} {3 * i}")
    lines.insert(5, "f 1 2 39999")            # vertex 39999 is defined later
    obj = tmp_path / "m.obj"
    obj.write_text("\n".join(lines) + "\n")
    assert obj.stat().st_size > (1 << 20)
    scene = tmp_path / "s.json"
    scene.write_text('{"schema": "1.0", "name": "m", "version": "1", "materials": {"w": {"albedo": [0.5,0.5,0.5]},'
                     ' "l": {"emissive": [1,1,1]}}, "primitives": [{"type": "mesh", "file": "m.obj", "material": "w"},'
                     ' {"type": "plane", "light": true, "origin": [0,2,0], "u": [1,0,0], "v": [0,0,1], "material": "l"}]}')
    with pytest.raises(capi.PcrError) as e:
        capi.HostScene(str(scene), str(tmp_path))
    assert "vertex index out of range" in str(e.value)
