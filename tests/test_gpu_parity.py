"""GPU parity tests: the sm_100a kernels, called through the C ABI, against
the CPU restatement oracle (pinned to the reference's goldens) and the
reference-generated fixtures.

Bars (from the reference's own oracle):
  * closest-hit material ids and t: bit-exact on plane/sphere scenes;
  * BVH hit triangle ids: bit-exact on 10M seeded rays over a 69,620-triangle
    mesh, except hits whose t values tie within 1e-6;
  * FP32 spectral / CIE / tone-map stage functions: 1e-5 relative (with an
    absolute floor of 1e-7 for values near zero);
  * rendered image: per-channel mean within 0.5 % of the converged CPU image,
    RMSE at a given spp within 3 sigma of the CPU estimator's RMSE at that spp.
"""
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from conftest import GOLDEN, scene_path

pytestmark = pytest.mark.gpu

PLANE_SCENES = ["cornell", "cornell-spec", "cornell-glass", "cornell-spheres", "closed-cornell-spec",
                "cornell-large-light", "bright-cornell-glass", "closed-cornell-glass", "cornell-frank"]


@pytest.fixture(scope="module")
def ctx():
    from pcr_b200 import capi
    c = capi.Context(device=0, queue_capacity=1 << 20)
    yield c
    c.close()


@pytest.fixture(scope="module")
def O():
    from oracle import oracle
    oracle.build()
    return oracle


def box_rays(n, seed):
    rng = np.random.default_rng(seed)
    o = np.stack([rng.uniform(-1.95, 1.95, n), rng.uniform(-1.95, 1.95, n), rng.uniform(-5.95, -0.05, n)], 1)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return np.concatenate([o, d], 1).astype(np.float32)


@pytest.mark.parametrize("name", PLANE_SCENES)
def test_trace_closest_bit_exact(ctx, O, name):
    sid = ctx.load_scene_json(scene_path(name), GOLDEN)
    osc = O.load_scene(scene_path(name), GOLDEN)
    rays = box_rays(200_000, sum(name.encode()))
    mat, prim, t = ctx.trace_closest(sid, rays)
    omat, ohn = O.scene_intersect(osc, rays)
    assert np.array_equal(mat, omat)
    # the oracle returns hit points; the hit point is origin + dir * t
    hit = rays[:, :3] + rays[:, 3:] * t[:, None]
    m = mat >= 0
    assert np.allclose(hit[m], ohn[m, :3], rtol=0, atol=2e-5)
    ctx.release_scene(sid)


def _shadow_rays(osc, n, seed):
    """Shadow segments as k_shade makes them: origins in the box, targets half
    on the scene's light planes, half anywhere in the box; direction
    Li * rsqrt(|Li|^2) and |Li|^2 in float32."""
    rng = np.random.default_rng(seed)
    o = box_rays(n, seed)[:, :3]
    lp = [L for L in osc.lights if L[0] == 0] if hasattr(osc, "lights") else []
    P = box_rays(n, seed + 1)[:, :3]
    if lp:
        k = rng.integers(0, len(lp), n)
        a, b = rng.uniform(size=n), rng.uniform(size=n)
        for j, L in enumerate(lp):
            pl = L[1]
            sel = (k == j) & (np.arange(n) < n // 2)
            P[sel] = (np.asarray(pl.origin, np.float32) + np.asarray(pl.u, np.float32) * a[sel, None]
                      + np.asarray(pl.v, np.float32) * b[sel, None])
    Li = (P - o).astype(np.float32)
    d2 = (Li[:, 0] * Li[:, 0] + Li[:, 1] * Li[:, 1] + Li[:, 2] * Li[:, 2]).astype(np.float32)
    ok = d2 > 1e-6
    d = Li[ok] / np.sqrt(d2[ok])[:, None]
    return np.concatenate([o[ok], d], 1).astype(np.float32), d2[ok]


def _oracle_blocked(O, osc, rays, d2):
    """code/Renderer.cpp:852-860 on the oracle: closest hit (reference
    arithmetic), blocked when non-emissive and |hit - o|^2 < lightDist2 - 1e-3."""
    mat, hn = O.scene_intersect(osc, rays)
    emis = np.array([max(m.emissive) > 0 for m in osc.materials] + [False])
    dd = (hn[:, :3] - rays[:, :3]).astype(np.float32)
    dist2 = ((dd[:, 0] * dd[:, 0] + dd[:, 1] * dd[:, 1]).astype(np.float32) + dd[:, 2] * dd[:, 2]).astype(np.float32)
    lim = d2.astype(np.float64) - 1e-3
    blocked = (mat >= 0) & ~emis[mat] & (lim > dist2.astype(np.float64))
    marginal = np.abs(lim - dist2) <= 1e-5 * np.maximum(d2, 1.0)
    return blocked, marginal


@pytest.mark.parametrize("name", PLANE_SCENES)
def test_shadow_test_matches_oracle(ctx, O, name):
    """k_shadow's early-exit query answers as the reference's closest-hit
    shadow test does, except where the hit lies at the light distance within
    rounding."""
    sid = ctx.load_scene_json(scene_path(name), GOLDEN)
    osc = O.load_scene(scene_path(name), GOLDEN)
    rays, d2 = _shadow_rays(osc, 200_000, sum(name.encode()) + 5)
    got = ctx.trace_shadow(sid, rays, d2).astype(bool)
    want, marginal = _oracle_blocked(O, osc, rays, d2)
    bad = (got != want) & ~marginal
    assert bad.sum() == 0, f"{bad.sum()} shadow decisions differ ({(got != want).sum()} incl. marginal)"
    assert want.mean() < 0.99
    if name == "cornell":   # two boxes: a fair share of segments is blocked
        assert want.mean() > 0.05
    ctx.release_scene(sid)


def test_shadow_test_matches_oracle_with_mesh_light(ctx, O):
    """The emissive-mesh scene (a 180-triangle icosphere whose mesh primitive
    is a light, beside the ceiling quad): emissive triangles sit in the BVH,
    so the shadow query takes the closest-hit route, where a hit on an
    emissive triangle never blocks.  A third of the segments end on the
    light triangles, a third on the quad, the rest anywhere in the box."""
    name = "cornell-mesh-light"
    sid = ctx.load_scene_json(scene_path(name), GOLDEN)
    osc = O.load_scene(scene_path(name), GOLDEN)
    tl = [t for kind, payload in osc.lights if kind == 1 for t in payload]
    assert len(tl) == 180
    n = 150_000
    rays, d2 = _shadow_rays(osc, n, 91)
    rng = np.random.default_rng(92)
    o = box_rays(n // 3, 93)[:, :3]
    k = rng.integers(0, len(tl), n // 3)
    a, b = rng.uniform(size=n // 3), rng.uniform(size=n // 3)
    flip = a + b > 1
    a[flip], b[flip] = 1 - a[flip], 1 - b[flip]
    v = np.array([[list(t.v0), list(t.v1), list(t.v2)] for t in tl], np.float32)[k]
    P = (v[:, 0] + (v[:, 1] - v[:, 0]) * a[:, None] + (v[:, 2] - v[:, 0]) * b[:, None]).astype(np.float32)
    Li = (P - o).astype(np.float32)
    dd = (Li[:, 0] * Li[:, 0] + Li[:, 1] * Li[:, 1] + Li[:, 2] * Li[:, 2]).astype(np.float32)
    ok = dd > 1e-6
    mr = np.concatenate([o[ok], Li[ok] / np.sqrt(dd[ok])[:, None]], 1).astype(np.float32)
    rays, d2 = np.concatenate([rays, mr]), np.concatenate([d2, dd[ok]])
    got = ctx.trace_shadow(sid, rays, d2).astype(bool)
    want, marginal = _oracle_blocked(O, osc, rays, d2)
    bad = (got != want) & ~marginal
    assert bad.sum() == 0, f"{bad.sum()} shadow decisions differ ({(got != want).sum()} incl. marginal)"
    # segments that end on the light mesh: some blocked (origins inside or
    # behind the boxes), most lit (a hit on the mesh's emissive near side
    # never blocks, code/Renderer.cpp:860)
    tail = want[-mr.shape[0]:]
    assert 0.05 < tail.mean() < 0.95
    ctx.release_scene(sid)


def _oracle_bvh_query(O, nodes, arr, rays, chunks=64):
    parts = np.array_split(np.arange(rays.shape[0]), chunks)
    with ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        res = list(ex.map(lambda ix: O.bvh_query(nodes, arr, rays[ix]), parts))
    return np.concatenate([r[0] for r in res]), np.concatenate([r[1] for r in res])


@pytest.fixture(scope="module")
def mesh(ctx, O):
    from pcr_b200 import capi, workloads
    path = workloads.mesh_scene(59, 1)
    hs = capi.HostScene(path, GOLDEN)
    tl = hs.triangles()
    ids = hs.triangle_ids()
    tris = np.zeros((tl.shape[0], 9), np.float32)
    tris[ids] = tl[:, :9]                       # file order
    boxes, ints, perm, arr, nodes = O.bvh_build(tris)
    sid = ctx.load_scene_json(path, GOLDEN)
    return {"sid": sid, "tris": tris, "arr": arr, "nodes": nodes, "boxes": boxes, "ints": ints, "hs": hs}


def test_mesh_bvh_matches_oracle_tree(mesh):
    b = mesh["hs"].bvh()
    assert np.array_equal(b[:, :6].view(np.uint32), mesh["boxes"].view(np.uint32))
    assert np.array_equal(b[:, 6:].view(np.int32), mesh["ints"])


def test_bvh_hit_ids_10m_rays(ctx, O, mesh):
    n = 10_000_000
    rng = np.random.default_rng(2024)
    o = np.stack([rng.uniform(-1.95, 1.95, n), rng.uniform(-1.95, 1.95, n), rng.uniform(-5.95, -0.05, n)], 1)
    # cosine-distributed about a random axis per ray
    axis = rng.normal(size=(n, 3))
    axis /= np.linalg.norm(axis, axis=1, keepdims=True)
    u1, u2 = rng.uniform(size=n), rng.uniform(size=n)
    r, phi = np.sqrt(u1), 2 * np.pi * u2
    helper = np.where(np.abs(axis[:, :1]) < 0.9, [[1.0, 0, 0]], [[0, 1.0, 0]])
    T = np.cross(axis, helper)
    T /= np.linalg.norm(T, axis=1, keepdims=True)
    B = np.cross(axis, T)
    d = T * (r * np.cos(phi))[:, None] + B * (r * np.sin(phi))[:, None] + axis * np.sqrt(1 - u1)[:, None]
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.concatenate([o, d], 1).astype(np.float32)
    del o, d, axis, T, B, helper
    gid, gt = ctx.trace_bvh(mesh["sid"], rays)
    oid, ot = _oracle_bvh_query(O, mesh["nodes"], mesh["arr"], rays)
    assert np.array_equal(gid >= 0, oid >= 0), "hit/miss disagreement"
    diff = gid != oid
    ties = np.abs(gt - ot) <= 1e-6
    bad = diff & ~ties
    assert bad.sum() == 0, f"{bad.sum()} id mismatches outside t-ties ({diff.sum()} total, {(gid >= 0).sum()} hits)"
    assert (gid >= 0).sum() > n // 20


def test_shadow_test_matches_oracle_on_mesh(ctx, O, mesh):
    """The early-exit shadow query through the 4-wide BVH (a blocking
    triangle ends the walk) against the oracle's closest-hit test."""
    from pcr_b200 import workloads
    path = workloads.mesh_scene(59, 1)
    osc = O.load_scene(path, GOLDEN)
    rays, d2 = _shadow_rays(osc, 100_000, 41)
    got = ctx.trace_shadow(mesh["sid"], rays, d2).astype(bool)
    want, marginal = _oracle_blocked(O, osc, rays, d2)
    bad = (got != want) & ~marginal
    assert bad.sum() == 0, f"{bad.sum()} shadow decisions differ ({(got != want).sum()} incl. marginal)"
    assert want.mean() > 0.05


def test_bvh_hit_ids_on_1m_triangle_mesh(ctx, O):
    """The serving-at-scale mesh: a seeded displaced icosphere of 1,003,520
    triangles.  The host-built tree equals the oracle's restatement of the
    reference builder node for node, and 2M seeded rays hit the same
    triangle ids through the 4-wide device BVH (t-ties within 1e-6 aside)."""
    from pcr_b200 import capi, workloads
    path = workloads.mesh_scene(224, 3)
    hs = capi.HostScene(path, GOLDEN)
    tl = hs.triangles()
    ids = hs.triangle_ids()
    tris = np.zeros((tl.shape[0], 9), np.float32)
    tris[ids] = tl[:, :9]
    assert tris.shape[0] == 1_003_520
    boxes, ints, perm, arr, nodes = O.bvh_build(tris)
    b = hs.bvh()
    assert np.array_equal(b[:, :6].view(np.uint32), boxes.view(np.uint32))
    assert np.array_equal(b[:, 6:].view(np.int32), ints)
    sid = ctx.load_scene_json(path, GOLDEN)
    rays = box_rays(2_000_000, 224)
    gid, gt = ctx.trace_bvh(sid, rays)
    oid, ot = _oracle_bvh_query(O, nodes, arr, rays)
    assert np.array_equal(gid >= 0, oid >= 0), "hit/miss disagreement"
    bad = (gid != oid) & ~(np.abs(gt - ot) <= 1e-6)
    assert bad.sum() == 0, f"{bad.sum()} id mismatches outside t-ties"
    assert (gid >= 0).mean() > 0.05
    ctx.release_scene(sid)
    hs.close()


def test_bvh_counts_match_reference_traversal_order_of_magnitude(ctx, O, mesh):
    rays = box_rays(65536, 3)
    _, _, cnt = ctx.trace_bvh(mesh["sid"], rays, counts=True)
    _, _, ocnt = O.bvh_query(mesh["nodes"], mesh["arr"], rays, counts=True)
    # the 4-wide tree visits fewer nodes than the binary one; leaf tests
    # stay within a small factor of the reference's
    assert cnt[:, 0].mean() < ocnt[:, 0].mean()
    assert 0.5 < cnt[:, 1].mean() / max(ocnt[:, 1].mean(), 1e-9) < 2.0


def _rel_ok(a, b, rel=1e-5, floor=1e-7):
    return np.all(np.abs(a - b) <= np.maximum(rel * np.abs(b), floor))


def test_stage_functions_match_oracle(ctx, O):
    from oracle.oracle import fptr
    lam = np.linspace(380.0, 720.0, 200001).astype(np.float32)
    L = O.lib()
    # sigmoid fits of the cornell materials (albedo and emissive)
    osc = O.load_scene(scene_path("cornell"), GOLDEN)
    for m in osc.materials:
        for fit in (np.asarray(m.afit, np.float32), np.asarray(m.efit, np.float32)):
            g = ctx.eval_stage(0, lam, fit)[:, 0]
            c = np.zeros_like(lam)
            L.oracle_eval_fit(fptr(fit), fptr(lam), lam.size, fptr(c))
            assert _rel_ok(g, c)
    # tabulated spectrum lerp (cornell-spec white paint)
    spec = O.load_scene(scene_path("cornell-spec"), GOLDEN)
    tab = np.asarray(spec.materials[0].tabA, np.float32)
    g = ctx.eval_stage(1, lam, tab)[:, 0]
    c = np.zeros_like(lam)
    L.oracle_eval_spectrum(fptr(tab), fptr(lam), lam.size, fptr(c))
    assert _rel_ok(g, c)
    # CIE colour-matching functions and singleLambdaXYZ
    g = ctx.eval_stage(2, lam)
    c = np.zeros((lam.size, 3), np.float32)
    L.oracle_eval_cmf(fptr(lam), lam.size, fptr(c))
    assert _rel_ok(g, c)
    rad = np.random.default_rng(1).uniform(0, 50, lam.size).astype(np.float32)
    g = ctx.eval_stage(3, np.stack([lam, rad], 1))
    L.oracle_single_lambda_xyz(fptr(lam), fptr(rad), lam.size, fptr(c))
    assert _rel_ok(g, c)
    # the form the hot path uses: raygen's interpolated colour-matching table
    # (the weight a path carries) times the radiance, 380..720 nm
    g = ctx.eval_stage(8, np.stack([lam, rad], 1))
    assert _rel_ok(g, c), "table-interpolated singleLambdaXYZ beyond 1e-5 relative"
    one = np.ones_like(lam)
    L.oracle_single_lambda_xyz(fptr(lam), fptr(one), lam.size, fptr(c))
    assert _rel_ok(ctx.eval_stage(8, np.stack([lam, one], 1)), c)
    # XYZ -> sRGB, Reinhard, ACES, quantisation
    xyz = np.random.default_rng(2).uniform(-0.2, 4.0, (100000, 3)).astype(np.float32)
    g = ctx.eval_stage(4, xyz)
    c = np.zeros_like(xyz)
    L.oracle_xyz_to_srgb(fptr(xyz), xyz.shape[0], fptr(c))
    assert np.allclose(g, c, rtol=1e-5, atol=1e-6)
    tm, q = O.tonemap(xyz, aces=False)
    assert _rel_ok(ctx.eval_stage(5, xyz), tm.reshape(-1, 3))
    tma, _ = O.tonemap(xyz, aces=True)
    assert _rel_ok(ctx.eval_stage(6, xyz), tma.reshape(-1, 3))
    assert np.array_equal(ctx.eval_stage(7, tm.reshape(-1, 3)).astype(np.uint8), q.reshape(-1, 3))


@pytest.fixture(scope="module")
def conv64():
    p = os.path.join(GOLDEN, "converged_cornell64.npz")
    if not os.path.exists(p):
        pytest.skip("converged fixture not generated")
    return np.load(p)


def test_render_mean_matches_converged_cpu(ctx, conv64):
    from pcr_b200 import capi
    sid = ctx.load_scene_json(scene_path("cornell"), GOLDEN)
    hdr, rgb, st = ctx.render(sid, capi.render_desc(64, depth=4, samples=16384, shadow=4, spectral=True, seed=5))
    cpu = conv64["image"].astype(np.float64)
    g = hdr.reshape(-1, 3).mean(0)
    c = cpu.reshape(-1, 3).mean(0)
    assert np.all(np.abs(g - c) / np.abs(c) < 0.005), (g, c)
    ctx.release_scene(sid)


@pytest.mark.parametrize("spp", [4, 16, 64])
def test_render_rmse_within_3_sigma_of_cpu(ctx, conv64, spp):
    from pcr_b200 import capi
    sid = ctx.load_scene_json(scene_path("cornell"), GOLDEN)
    k = list(conv64["rmse_spp"]).index(spp)
    cpu = conv64["rmse"][k]
    mu, sigma = cpu.mean(), cpu.std(ddof=1)
    r = []
    for s in range(4):
        hdr, _, _ = ctx.render(sid, capi.render_desc(64, depth=4, samples=spp, shadow=4, spectral=True, seed=77 + s))
        r.append(np.sqrt(np.mean((hdr.astype(np.float64) - conv64["image"]) ** 2)))
    assert abs(np.mean(r) - mu) <= 3 * sigma, (np.mean(r), mu, sigma)
    ctx.release_scene(sid)


def test_rgb_mode_and_knobs_against_oracle(ctx, O):
    """RGB mode plus MIS / Russian roulette / stratified / aa: image means
    against the oracle's estimator of the same configuration."""
    from pcr_b200 import capi
    for scene in ("cornell", "cornell-spheres", "cornell-glass"):
        sid = ctx.load_scene_json(scene_path(scene), GOLDEN)
        osc = O.load_scene(scene_path(scene), GOLDEN)
        for kw in ({"spectral": False}, {"spectral": False, "mis": True, "russian": True, "stratified": True},
                   {"spectral": True, "mis": True}):
            hdr, _, _ = ctx.render(sid, capi.render_desc(48, depth=3, samples=4096, shadow=2, seed=9, **kw))
            ref = O.render_paths(osc, O.opts(48, depth=3, shadow=2, seed=3, **kw), 256, threads=os.cpu_count())
            g, c = hdr.reshape(-1, 3).mean(0), ref.reshape(-1, 3).mean(0)
            assert np.all(np.abs(g - c) / np.abs(c) < 0.03), (scene, kw, g, c)
        ctx.release_scene(sid)


def test_batched_results_match_plain_and_alone(ctx):
    """Each render is the same alone (plain method), alone in the batched
    engine, and inside a mixed batch: the counter-based RNG ties every path
    to (seed, pixel, sample, bounce) and pixels accumulate in FP64."""
    from pcr_b200 import capi
    sids = [ctx.load_scene_json(scene_path(s), GOLDEN) for s in ("cornell", "cornell-glass", "cornell-spheres")]
    descs = [capi.render_desc(96, depth=4, samples=32, shadow=2, seed=11),
             capi.render_desc(64, 80, depth=5, samples=16, shadow=3, seed=12),
             capi.render_desc(40, depth=3, samples=64, shadow=1, spectral=False, seed=13)]
    alone = [ctx.render(s, d)[0] for s, d in zip(sids, descs)]
    rid = ctx.submit(sids[0], descs[0])
    ctx.run_until_idle()
    solo = ctx.fetch(rid)[0]
    ids = [ctx.submit(s, d) for s, d in zip(sids, descs)]
    ctx.run_until_idle()
    mixed = [ctx.fetch(i)[0] for i in ids]
    for a, m in zip(alone, mixed):
        assert np.allclose(a, m, rtol=1e-6, atol=1e-7)
    assert np.allclose(alone[0], solo, rtol=1e-6, atol=1e-7)
    for s in sids:
        ctx.release_scene(s)


def _aim(o, P):
    d = (P - o).astype(np.float64)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return np.concatenate([o, d], 1).astype(np.float32)


def test_rays_at_triangle_edges_match_oracle(ctx, O, mesh):
    """Rays aimed at triangle edges and vertices (barycentric u = 0, v = 0,
    u + v = 1, corners), where the approximate-reciprocal pre-filter of the
    triangle test is closest to its margins: hit / miss and t agree with the
    exact restatement, ids too except at t-ties (shared edges).

    A ray that grazes a box face can fail the reference's slab test by
    rounding.  The 4-wide tree does not test the binary boxes it collapsed,
    so on such rays the device may find a valid hit the reference's
    traversal skipped.  Measured: 2 of 400,000 edge rays, each 4-5e-6
    closer, with and without the pre-filters.  Such cases must stay rare,
    and the device's hit is never farther than the reference's."""
    rng = np.random.default_rng(77)
    tris = mesh["tris"].reshape(-1, 3, 3).astype(np.float32)
    n = 400_000
    k = rng.integers(0, tris.shape[0], n)
    v0, v1, v2 = tris[k, 0], tris[k, 1], tris[k, 2]
    r = rng.uniform(0, 1, n).astype(np.float32)
    kind = rng.integers(0, 6, n)
    u = np.select([kind == 0, kind == 1, kind == 2, kind == 3, kind == 4], [0 * r, r, r, 0 * r, 1 + 0 * r], 0 * r)
    v = np.select([kind == 0, kind == 1, kind == 2, kind == 3, kind == 4], [r, 0 * r, 1 - r, 0 * r, 0 * r], 1 + 0 * r)
    P = (v0 + (v1 - v0) * u[:, None] + (v2 - v0) * v[:, None]).astype(np.float32)
    o = np.stack([rng.uniform(-1.95, 1.95, n), rng.uniform(-1.95, 1.95, n), rng.uniform(-5.95, -0.05, n)], 1)
    rays = _aim(o.astype(np.float32), P)
    gid, gt = ctx.trace_bvh(mesh["sid"], rays)
    oid, ot = _oracle_bvh_query(O, mesh["nodes"], mesh["arr"], rays)
    assert np.array_equal(gid >= 0, oid >= 0), "hit/miss disagreement"
    hit = gid >= 0
    assert hit.mean() > 0.3
    same = gid == oid
    assert np.array_equal(gt[hit & same].view(np.uint32), ot[hit & same].view(np.uint32))
    bad = hit & ~same & (np.abs(gt - ot) > 1e-6)
    assert bad.sum() <= n // 50_000, f"{bad.sum()} id mismatches outside t-ties ({(~same & hit).sum()} at ties)"
    assert np.all(gt[bad] < ot[bad]), "the device returned a farther hit than the reference"


@pytest.mark.parametrize("name", ["cornell", "cornell-spheres"])
def test_rays_at_plane_quad_edges_match_oracle(ctx, O, name):
    """Rays aimed at the borders and corners of every plane quad (s or q
    exactly 0 or 1), where the plane test's pre-filters sit on their
    margins: same material and hit point as the exact restatement."""
    from pcr_b200 import capi
    hs = capi.HostScene(scene_path(name), GOLDEN)
    pl = hs.planes()
    rng = np.random.default_rng(5)
    n = 300_000
    k = rng.integers(0, pl.shape[0], n)
    org, pu, pv = pl[k, 0:3], pl[k, 3:6], pl[k, 6:9]
    r = rng.uniform(0, 1, n).astype(np.float32)
    kind = rng.integers(0, 5, n)
    s = np.select([kind == 0, kind == 1, kind == 2, kind == 3], [0 * r, 1 + 0 * r, r, r], (r > 0.5).astype(np.float32))
    q = np.select([kind == 0, kind == 1, kind == 2, kind == 3], [r, r, 0 * r, 1 + 0 * r], (r * 7 % 1 > 0.5).astype(np.float32))
    P = (org + pu * s[:, None] + pv * q[:, None]).astype(np.float32)
    rays = _aim(box_rays(n, 11)[:, :3], P)
    sid = ctx.load_scene_json(scene_path(name), GOLDEN)
    osc = O.load_scene(scene_path(name), GOLDEN)
    mat, prim, t = ctx.trace_closest(sid, rays)
    omat, ohn = O.scene_intersect(osc, rays)
    assert np.array_equal(mat, omat)
    hitp = rays[:, :3] + rays[:, 3:] * t[:, None]
    m = mat >= 0
    assert np.allclose(hitp[m], ohn[m, :3], rtol=0, atol=2e-5)
    ctx.release_scene(sid)
    hs.close()
