"""The device BVH build (pcr_bvh_build, and scene loads through
pcr_scene_load_json) against the reference builder, Bvh::build
(code/Bvh/Bvh.cpp:122-325): node arrays bit for bit and the same triangle
order.  Pinned to the reference's own node arrays (bvh_vectors.npz), to the
oracle's restatement on edge cases, and to the host builder (itself equal to
the oracle) on the 69,620- and 1,003,520-triangle meshes."""
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from pcr_b200 import capi
    c = capi.Context()
    yield c
    c.close()


def _same(nodes, order, boxes, ints, perm):
    assert nodes.shape[0] == boxes.shape[0]
    assert np.array_equal(nodes[:, :6].view(np.uint32), boxes.view(np.uint32))
    assert np.array_equal(nodes[:, 6:].view(np.int32), ints)
    assert np.array_equal(order, perm)


def _oracle(tris9):
    from oracle import oracle as O
    O.build()
    boxes, ints, perm, _, _ = O.bvh_build(tris9)
    return boxes, ints, perm


@pytest.mark.parametrize("name", ["soup200", "soup5k", "coplanar"])
def test_device_build_matches_reference_vectors(ctx, name):
    v = np.load(os.path.join(GOLDEN, "bvh_vectors.npz"))
    nodes, order = ctx.build_bvh(v[f"{name}_tris"])
    _same(nodes, order, v[f"{name}_boxes"], v[f"{name}_ints"], v[f"{name}_perm"])


def _soup(n, seed, spread=2.0, size=0.05):
    rng = np.random.default_rng(seed)
    c = rng.uniform(-spread, spread, (n, 1, 3))
    return (c + rng.uniform(-size, size, (n, 3, 3))).reshape(n, 9).astype(np.float32)


def _cases():
    rng = np.random.default_rng(11)
    cases = {}
    for n in (1, 4, 5, 31, 32, 33, 34, 127, 128, 129, 1023, 1025, 20000):
        cases[f"soup{n}"] = _soup(n, n)
    # runs of identical triangles and clustered centroids (equal keys)
    base = _soup(40, 3)
    cases["duplicates"] = np.repeat(base, 60, axis=0)[rng.permutation(2400)]
    # every centroid equal: one leaf over all triangles
    cases["coincident"] = np.repeat(_soup(1, 5), 300, axis=0)
    # signed zeros: vertices on the plane z = +-0 and x = +-0
    z = _soup(3000, 7)
    z[:, 2::3] = np.where(rng.random((3000, 3)) < 0.5, np.float32(-0.0), np.float32(0.0))
    xz = rng.random((3000, 3)) < 0.3
    z[:, 0::3] = np.where(xz, np.where(rng.random((3000, 3)) < 0.5, np.float32(-0.0), np.float32(0.0)), z[:, 0::3])
    cases["signed_zero"] = z
    # one axis without extent
    f = _soup(5000, 9)
    f[:, 0::3] = np.float32(0.25)
    cases["flat_x"] = f
    # exponentially spaced positions: lopsided splits, deep trees
    k = np.arange(6000)
    e = _soup(6000, 13, spread=0.0, size=0.01)
    e[:, 1::3] += (2.0 ** (-(k % 60)) * 8.0)[:, None].astype(np.float32)
    cases["lopsided"] = e.astype(np.float32)
    return cases


CASES = _cases()


@pytest.mark.parametrize("name", sorted(CASES))
def test_device_build_matches_oracle(ctx, name):
    tris = CASES[name]
    nodes, order = ctx.build_bvh(tris)
    _same(nodes, order, *_oracle(tris))


def test_device_build_of_a_single_leaf_keeps_all_triangles(ctx):
    nodes, order = ctx.build_bvh(CASES["coincident"])
    assert nodes.shape[0] == 1 and nodes[0, 6:].view(np.int32)[2] == 300


@pytest.mark.parametrize("freq", [59, 224])
def test_device_build_matches_host_build_on_meshes(ctx, freq):
    """69,620 and 1,003,520 triangles: the level passes over many chunks,
    the small-node threads, and the preorder renumbering."""
    from pcr_b200 import capi, workloads
    path = workloads.mesh_scene(freq, 1)
    hs = capi.HostScene(path, GOLDEN)
    tl, ids = hs.triangles(), hs.triangle_ids()
    tris = np.zeros((tl.shape[0], 9), np.float32)
    tris[ids] = tl[:, :9]
    nodes, order = ctx.build_bvh(tris)
    b = hs.bvh()
    assert np.array_equal(nodes[:, :6].view(np.uint32), b[:, :6].view(np.uint32))
    assert np.array_equal(nodes[:, 6:].view(np.int32), b[:, 6:].view(np.int32))
    assert np.array_equal(order, ids)
    hs.close()


def test_scene_load_builds_on_the_device_with_the_same_hits(ctx):
    """pcr_scene_load_json builds the mesh BVH on the device; closest hits
    through it equal those of the host-built tree uploaded as it is."""
    from pcr_b200 import capi, workloads
    path = workloads.mesh_scene(59, 1)
    sid_dev = ctx.load_scene_json(path, GOLDEN)
    hs = capi.HostScene(path, GOLDEN)
    sid_host = ctx.upload_scene(hs.desc)
    rng = np.random.default_rng(3)
    o = rng.uniform(-0.9, 0.9, (200_000, 3)) + np.array([0.0, 0.0, -4.0])
    d = rng.normal(size=(200_000, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.concatenate([o, d], 1).astype(np.float32)
    a = ctx.trace_bvh(sid_dev, rays)
    b = ctx.trace_bvh(sid_host, rays)
    for x, y in zip(a, b):
        assert np.array_equal(np.asarray(x).view(np.uint32), np.asarray(y).view(np.uint32))
    assert (np.asarray(a[0]) >= 0).mean() > 0.05
    ctx.release_scene(sid_dev)
    ctx.release_scene(sid_host)
    hs.close()


def test_bvh_build_entry_point_errors(ctx):
    """pcr_bvh_build: too small an output array is an argument error, an
    empty input gives no nodes, and the context stays usable after both."""
    import ctypes as C

    from pcr_b200 import capi
    tris = np.zeros((100, 23), np.float32)
    tris[:, :9] = _soup(100, 3)
    nodes = np.zeros((4, 9), np.float32)
    order = np.zeros(100, np.int32)
    m = C.c_int32(0)
    st = ctx.L.pcr_bvh_build(ctx.h, capi._fp(tris), 100, capi._fp(nodes), 4, C.byref(m), capi._ip(order))
    assert st == 1 and b"too small" in ctx.L.pcr_last_error()
    st = ctx.L.pcr_bvh_build(ctx.h, None, 0, None, 0, C.byref(m), None)
    assert st == 0 and m.value == 0
    n2, o2 = ctx.build_bvh(_soup(100, 3))
    _same(n2, o2, *_oracle(_soup(100, 3)))
