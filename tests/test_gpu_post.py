"""Device post-processing and adaptive sampling, and renders of the
synthetic mesh scene, through the C ABI.

* Bilateral denoise on the device against the oracle's restatement of
  Denoise::bilateralRGB (code/Denoise.cpp:14-86) applied to the same
  8-bit image.
* Adaptive aa rounds (code/Gpu/Opengl/OpenglRenderer.cpp:1288-1383): with
  fewer than 4 rounds nothing can converge, so the image equals the
  non-adaptive one; with many rounds converged pixels stop early (fewer
  paths) without moving the image mean; a batched adaptive render equals
  the same render alone.
* The displaced-icosphere mesh scene (diffuse and glass): per-channel image
  mean against the oracle's paths-per-pixel estimator at the same spp.
"""
import numpy as np
import pytest

from conftest import GOLDEN, scene_path

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from pcr_b200 import capi
    c = capi.Context(device=0, queue_capacity=1 << 18)
    yield c
    c.close()


@pytest.fixture(scope="module")
def O():
    from oracle import oracle
    oracle.build()
    return oracle


def test_denoise_on_device_matches_oracle_bilateral(ctx, O):
    from oracle.oracle import lib
    from pcr_b200 import capi
    sid = ctx.load_scene_json(scene_path("cornell-spheres"), GOLDEN)
    for w, h in ((96, 80), (33, 17)):
        plain = capi.render_desc(w, h, depth=3, samples=4, shadow=2, seed=17)
        den = capi.render_desc(w, h, depth=3, samples=4, shadow=2, seed=17, denoise=True)
        _, rgb, _ = ctx.render(sid, plain)
        _, rgb_d, _ = ctx.render(sid, den)
        want = np.ascontiguousarray(rgb.copy())
        import ctypes as C
        lib().oracle_bilateral(want.ctypes.data_as(C.POINTER(C.c_ubyte)), w, h)
        diff = np.abs(rgb_d.astype(int) - want.astype(int))
        # the weight's exponential is rounded once on both sides; a rare
        # last-bit difference may move a byte by one level
        assert diff.max() <= 1 and (diff > 0).mean() < 1e-3, (diff.max(), (diff > 0).mean())
        assert not np.array_equal(rgb_d, rgb)  # it did smooth
    ctx.release_scene(sid)


def test_adaptive_with_three_rounds_equals_plain_aa(ctx):
    from pcr_b200 import capi
    sid = ctx.load_scene_json(scene_path("cornell"), GOLDEN)
    a = ctx.render(sid, capi.render_desc(48, depth=3, samples=8, shadow=2, aa=3, seed=31))[0]
    b, _, st = ctx.render(sid, capi.render_desc(48, depth=3, samples=8, shadow=2, aa=3, adaptive=True, seed=31))
    assert st.paths == 48 * 48 * 8 * 3
    assert np.allclose(a, b, rtol=2e-5, atol=1e-6)
    ctx.release_scene(sid)


def test_adaptive_stops_converged_pixels_early(ctx):
    """aa = 5: a pixel either stops after round 4 (its output is then the
    mean of rounds 0-3, which the non-adaptive aa = 4 render gives) or runs
    round 4 too (the non-adaptive aa = 5 mean).  A path's random numbers
    depend on its pixel and sample number only, so those renders trace the
    same rounds.  The path count must match the per-pixel choice."""
    from pcr_b200 import capi
    sid = ctx.load_scene_json(scene_path("cornell-large-light"), GOLDEN)
    W, spp = 64, 16

    def desc(aa, adaptive):
        return capi.render_desc(W, depth=3, samples=spp, shadow=4, aa=aa, adaptive=adaptive, seed=41)
    m4 = ctx.render(sid, desc(4, False))[0].astype(np.float64)
    m5 = ctx.render(sid, desc(5, False))[0].astype(np.float64)
    ad, _, st = ctx.render(sid, desc(5, True))
    ad = ad.astype(np.float64)
    tol = 2e-5 * np.maximum(np.abs(ad), 1.0)
    is4 = np.all(np.abs(ad - m4) <= tol, axis=2)
    is5 = np.all(np.abs(ad - m5) <= tol, axis=2)
    assert np.all(is4 | is5), "an adaptive pixel is neither the 4-round nor the 5-round mean"
    stopped = is4 & ~is5
    assert stopped.sum() > 0 and (~is4).sum() > 0      # both outcomes occur
    n4 = int(stopped.sum())
    lo = (4 * n4 + 5 * (W * W - n4)) * spp
    # pixels whose round-4 mean equals the 4-round mean cannot be told apart
    amb = int((is4 & is5).sum())
    assert lo - amb * spp <= st.paths <= lo, (st.paths, lo, amb)
    ctx.release_scene(sid)


def test_adaptive_saves_paths_at_many_rounds(ctx):
    from pcr_b200 import capi
    sid = ctx.load_scene_json(scene_path("cornell-large-light"), GOLDEN)
    full, _, st_f = ctx.render(sid, capi.render_desc(64, depth=3, samples=16, shadow=4, aa=12, seed=41))
    ad, _, st_a = ctx.render(sid, capi.render_desc(64, depth=3, samples=16, shadow=4, aa=12, adaptive=True,
                                                    seed=41))
    assert st_f.paths == 64 * 64 * 16 * 12
    assert 64 * 64 * 16 * 4 <= st_a.paths < 0.8 * st_f.paths
    # stopping on a low sample variance misses rare bright paths: the image
    # is slightly darker, as with the reference's adaptive loop
    m_f, m_a = full.reshape(-1, 3).mean(0), ad.reshape(-1, 3).mean(0)
    assert np.all(np.abs(m_a - m_f) <= 0.1 * np.abs(m_f)), (m_a, m_f)
    ctx.release_scene(sid)


def test_adaptive_batched_equals_alone(ctx):
    from pcr_b200 import capi
    sids = [ctx.load_scene_json(scene_path(s), GOLDEN) for s in ("cornell-glass", "cornell")]
    da = capi.render_desc(40, 32, depth=4, samples=4, shadow=2, aa=8, adaptive=True, seed=51)
    db = capi.render_desc(56, depth=3, samples=8, shadow=1, seed=52)
    alone = ctx.render(sids[0], da)[0]
    ids = [ctx.submit(sids[1], db), ctx.submit(sids[0], da), ctx.submit(sids[1], db)]
    ctx.run_until_idle()
    mixed = [ctx.fetch(i)[0] for i in ids]
    assert np.allclose(alone, mixed[1], rtol=1e-6, atol=1e-7)
    assert np.allclose(mixed[0], mixed[2], rtol=1e-6, atol=1e-7)
    for s in sids:
        ctx.release_scene(s)


@pytest.mark.parametrize("glass", [False, True])
def test_mesh_scene_mean_matches_oracle(ctx, O, glass):
    """The seeded ~70k-triangle displaced icosphere in the Cornell box
    (diffuse, or dispersive glass with the 4-way hero fork), spectral."""
    import os
    from pcr_b200 import capi, workloads
    path = workloads.mesh_scene(59, 7, glass=glass)
    sid = ctx.load_scene_json(path, GOLDEN)
    osc = O.load_scene(path, GOLDEN)
    spp = 1024
    g = ctx.render(sid, capi.render_desc(24, depth=5, samples=spp, shadow=2, seed=61))[0].astype(np.float64)
    o = O.render_paths(osc, O.opts(24, depth=5, samples=1, shadow=2, spectral=True, seed=62), spp,
                       threads=os.cpu_count() or 4)
    mg, mo = g.reshape(-1, 3).mean(0), o.reshape(-1, 3).mean(0)
    # two independent 590k-path estimates of the same mean: a few percent
    # (glass caustics are the noisier estimate)
    tol = 0.04 if glass else 0.03
    assert np.all(np.abs(mg - mo) <= tol * np.abs(mo) + 1e-3), (mg, mo)
    ctx.release_scene(sid)


def test_sample_range_partials_sum_to_the_full_render(ctx):
    """A render split by sample range (the multi-GPU single render, here two
    ranges on one GPU): the partial HDR images add up to the full render and
    the device tone map of the sum gives its 8-bit image."""
    from pcr_b200 import capi
    from pcr_b200.replicas import sample_range
    sid = ctx.load_scene_json(scene_path("cornell-glass"), GOLDEN)
    for aa, stratified in ((1, False), (3, False), (1, True)):
        full = capi.render_desc(40, 36, depth=4, samples=9, shadow=2, aa=aa, stratified=stratified, seed=81)
        hdr, rgb, st = ctx.render(sid, full)
        acc = np.zeros_like(hdr, dtype=np.float64)
        paths = 0
        for rank in range(3):
            b, e = sample_range(9, rank, 3)
            part = capi.render_desc(40, 36, depth=4, samples=9, shadow=2, aa=aa, stratified=stratified, seed=81,
                                    sample_begin=b, sample_end=e)
            h, _, s = ctx.render(sid, part, want_rgb=False)
            acc += h
            paths += s.paths
        assert paths == st.paths
        assert np.allclose(acc, hdr, rtol=1e-5, atol=1e-6)
        rgb2 = ctx.tonemap(acc.astype(np.float32))
        d = np.abs(rgb2.astype(int) - rgb.astype(int))
        assert d.max() <= 1 and (d > 0).mean() < 1e-3
    with pytest.raises(capi.PcrError):
        ctx.render(sid, capi.render_desc(16, samples=4, sample_begin=3, sample_end=2))
    ctx.release_scene(sid)


def test_many_shadow_samples_grow_the_shadow_queue(ctx):
    """More than 8 shadow samples per hit (the reference takes any S): the
    shadow queue grows between iterations.  The estimate has the same
    expectation as with few samples, and the batched render equals the
    plain one."""
    from pcr_b200 import capi
    sid = ctx.load_scene_json(scene_path("cornell"), GOLDEN)
    few = ctx.render(sid, capi.render_desc(48, depth=3, samples=64, shadow=2, seed=91))[0]
    many_d = capi.render_desc(48, depth=3, samples=64, shadow=40, seed=91)
    many, _, st = ctx.render(sid, many_d)
    assert st.paths == 48 * 48 * 64
    mf, mm = few.reshape(-1, 3).mean(0), many.reshape(-1, 3).mean(0)
    assert np.all(np.abs(mm - mf) <= 0.03 * np.abs(mf)), (mm, mf)
    rid = ctx.submit(sid, many_d)
    ctx.run_until_idle()
    assert np.allclose(ctx.fetch(rid)[0], many, rtol=1e-6, atol=1e-7)
    with pytest.raises(capi.PcrError):
        ctx.render(sid, capi.render_desc(16, samples=1, shadow=65))
    ctx.release_scene(sid)


def test_spectral_terminate_keeps_the_mean_and_traces_fewer_rays(ctx):
    """spectral_terminate (the GPU backends' spectralFork = false): at a
    dispersive refraction a path keeps its hero wavelength alone, scaled by
    the number of hero wavelengths.  It estimates the same image as the
    4-way fork with fewer rays, and is inert where no glass disperses."""
    from pcr_b200 import capi
    sid = ctx.load_scene_json(scene_path("cornell-glass"), GOLDEN)
    means, rays = [], []
    for term in (False, True):
        ctx.reset_stats()
        img = ctx.render(sid, capi.render_desc(48, depth=6, samples=512, shadow=2, seed=17,
                                               terminate=term))[0].astype(np.float64)
        rays.append(ctx.stats()["rays"])
        means.append(img.reshape(-1, 3).mean(0))
    # ~1.2M paths per image: the two unbiased estimates agree to a few tenths
    # of a percent; 2 % leaves room for the noisier caustic
    assert np.all(np.abs(means[1] - means[0]) <= 0.02 * np.abs(means[0])), means
    assert rays[1] < rays[0], rays
    ctx.release_scene(sid)
    sid = ctx.load_scene_json(scene_path("cornell"), GOLDEN)
    a = ctx.render(sid, capi.render_desc(32, depth=4, samples=8, shadow=2, seed=3))
    b = ctx.render(sid, capi.render_desc(32, depth=4, samples=8, shadow=2, seed=3, terminate=True))
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    ctx.release_scene(sid)
