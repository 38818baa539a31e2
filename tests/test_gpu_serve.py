"""Served mode (continuous batching), the autotuner and the request router,
through the C ABI.

Serving admits renders on the engine's own thread as request slots and the
device-memory budget free up; a request that arrives while others are on the
GPU shares the path queue with them.  Each result must be the same as the
render alone (plain method): every path's random numbers are a hash of
(seed, pixel, sample, fork, bounce) and pixels accumulate in FP64, so only
the FP64 summation order differs (tolerance rtol 1e-6, atol 1e-7, the same
as the batched-invariance test).
"""
import threading
import time

import numpy as np
import pytest

from conftest import GOLDEN, scene_path

pytestmark = pytest.mark.gpu

RTOL, ATOL = 1e-6, 1e-7


def _requests():
    from pcr_b200 import capi
    rng = np.random.default_rng(77)
    out = []
    for k in range(14):
        w = int(rng.choice([48, 64, 96, 128, 160]))
        h = int(rng.choice([48, 64, 96, 128]))
        out.append((["cornell", "cornell-glass", "cornell-spheres"][k % 3],
                    capi.render_desc(w, h, depth=int(rng.integers(2, 7)), samples=int(rng.integers(1, 24)),
                                     shadow=int(rng.integers(1, 5)), spectral=bool(k % 4 != 3), seed=500 + k)))
    return out


def test_served_results_match_alone():
    """Requests arrive from another thread while earlier ones are in flight;
    a small memory budget makes later ones wait for admission.  Every
    result equals its plain render."""
    from pcr_b200 import capi
    reqs = _requests()
    biggest = max(d.width * d.height for _, d in reqs) * 3 * 13
    ctx = capi.Context(device=0, queue_capacity=1 << 17, memory_budget=3 * biggest)
    try:
        sids = {v: ctx.load_scene_json(scene_path(v), GOLDEN) for v in {v for v, _ in reqs}}
        alone = [ctx.render(sids[v], d)[0] for v, d in reqs]
        ctx.serve_start()
        ids = [None] * len(reqs)

        def producer():
            for k, (v, d) in enumerate(reqs):
                ids[k] = ctx.submit(sids[v], d)
                time.sleep(0.003)
        th = threading.Thread(target=producer)
        th.start()
        th.join()
        results, stats = [], []
        for rid in ids:
            ctx.wait(rid, 120_000)
            hdr, rgb, st = ctx.fetch(rid)
            results.append(hdr)
            stats.append(st)
        ctx.serve_stop()
        for (v, d), a, m in zip(reqs, alone, results):
            assert np.allclose(a, m, rtol=RTOL, atol=ATOL), (v, d.width, d.height)
        # the budget held some requests back: they waited for admission
        assert max(s.queue_ms for s in stats) > 0.0
        assert all(s.latency_ms >= s.queue_ms for s in stats)
        assert all(s.paths == d.width * d.height * d.samples for (_, d), s in zip(reqs, stats))
    finally:
        ctx.close()


def test_cancel_pending_request():
    """A request still waiting for admission can be cancelled; waiting on it
    then reports PCR_ERR_CANCELLED, and the others complete unchanged."""
    from pcr_b200 import capi
    ctx = capi.Context(device=0, queue_capacity=1 << 17, memory_budget=256 * 256 * 3 * 13)
    try:
        sid = ctx.load_scene_json(scene_path("cornell"), GOLDEN)
        d0 = capi.render_desc(256, depth=3, samples=8, shadow=2, seed=1)
        d1 = capi.render_desc(256, depth=3, samples=8, shadow=2, seed=2)
        ref1 = ctx.render(sid, d1)[0]
        r0 = ctx.submit(sid, d0)
        r1 = ctx.submit(sid, d1)
        r2 = ctx.submit(sid, d0)   # cannot be admitted while r0 holds the whole budget
        ctx.cancel(r2)
        with pytest.raises(capi.PcrError) as e:
            ctx.wait(r2, 60_000)
        assert e.value.status == 7
        with pytest.raises(capi.PcrError) as e:       # fetch reports it and releases it
            ctx.fetch(r2)
        assert e.value.status == 7
        with pytest.raises(capi.PcrError) as e:
            ctx.poll(r2)
        assert e.value.status == 4                    # gone
        ctx.wait(r0, 60_000)
        ctx.wait(r1, 60_000)
        ctx.fetch(r0, want_hdr=False, want_rgb=False)
        assert np.allclose(ctx.fetch(r1)[0], ref1, rtol=RTOL, atol=ATOL)
        with pytest.raises(capi.PcrError):
            ctx.cancel(r1 + 1000)
    finally:
        ctx.close()


def test_cancel_running_request_and_progress():
    """A request cancelled while it runs stops issuing paths and ends once
    the paths in flight retire: waiting on it reports PCR_ERR_CANCELLED, its
    fetch reports and releases it, its device memory goes back, and a request
    that shared the wavefront with it completes unchanged.  Progress rises
    from 0 while it runs; a finished request reports 1."""
    from pcr_b200 import capi
    ctx = capi.Context(device=0, queue_capacity=1 << 20)
    try:
        sid = ctx.load_scene_json(scene_path("cornell"), GOLDEN)
        small = capi.render_desc(96, depth=4, samples=16, shadow=2, spectral=True, seed=3)
        ref = ctx.render(sid, small)[0]
        big = ctx.submit(sid, capi.render_desc(1024, depth=8, samples=1024, shadow=4, spectral=True, seed=4))
        rid = ctx.submit(sid, small)
        assert ctx.progress(big) == 0.0
        seen = []
        for _ in range(2000):
            with pytest.raises(capi.PcrError) as e:
                ctx.wait(big, 5)                  # drives the engine on this thread for ~5 ms
            assert e.value.status == 6            # timed out: still running
            seen.append(ctx.progress(big))
            if seen[-1] > 0.01:
                break
        assert 0.01 < seen[-1] < 0.5 and seen == sorted(seen)
        ctx.cancel(big)
        with pytest.raises(capi.PcrError) as e:
            ctx.wait(big, 60_000)
        assert e.value.status == 7
        with pytest.raises(capi.PcrError) as e:
            ctx.fetch(big)
        assert e.value.status == 7
        ctx.wait(rid, 60_000)
        assert ctx.progress(rid) == 1.0
        assert np.allclose(ctx.fetch(rid)[0], ref, rtol=RTOL, atol=ATOL)
        # the engine is idle and usable: a render after the cancel is unchanged
        assert np.allclose(ctx.render(sid, small)[0], ref, rtol=RTOL, atol=ATOL)
    finally:
        ctx.close()


def test_concurrent_fetches_match_alone():
    """Results copied out from four threads at once (each fetch takes its own
    pinned staging buffer and copy stream) equal the renders made alone."""
    from concurrent.futures import ThreadPoolExecutor

    from pcr_b200 import capi
    ctx = capi.Context(device=0, queue_capacity=1 << 20)
    try:
        sid = ctx.load_scene_json(scene_path("cornell-spheres"), GOLDEN)
        descs = [capi.render_desc(64 + 32 * (k % 4), depth=3, samples=8, shadow=2, spectral=bool(k & 1), seed=300 + k)
                 for k in range(12)]
        alone = [ctx.render(sid, d) for d in descs]
        ids = [ctx.submit(sid, d) for d in descs]
        ctx.run_until_idle()
        with ThreadPoolExecutor(max_workers=4) as ex:
            got = list(ex.map(lambda i: ctx.fetch(i), ids))
        for (a_hdr, a_rgb, _), (g_hdr, g_rgb, _) in zip(alone, got):
            assert np.allclose(a_hdr, g_hdr, rtol=RTOL, atol=ATOL)
            assert np.abs(a_rgb.astype(int) - g_rgb.astype(int)).max() <= 1
    finally:
        ctx.close()


def test_autotune_picks_from_grid_and_keeps_results():
    """The autotuner times trial batches over queue capacity, block size,
    issue chunk and refill cadence; the chosen tuning is one of the grid's
    and renders are unchanged by it."""
    from pcr_b200 import capi
    ctx = capi.Context(device=0)
    try:
        sid = ctx.load_scene_json(scene_path("cornell-glass"), GOLDEN)
        descs = [capi.render_desc(64 + 16 * k, depth=4, samples=4, shadow=2, seed=900 + k) for k in range(4)]
        before = [ctx.render(sid, d)[0] for d in descs]
        chosen = ctx.autotune([sid] * len(descs), descs)
        assert chosen["queue_capacity"] in (1 << 19, 1 << 20, 1 << 21, 1 << 22, 1 << 23, 1 << 24)
        assert chosen["block_size"] in (64, 128, 256)
        assert chosen["chunk_paths"] in (1 << 14, 1 << 16)
        assert chosen["regen_every"] in (1, 2)
        st = ctx.stats()
        assert all(st[k] == chosen[k] for k in chosen)
        ids = [ctx.submit(sid, d) for d in descs]
        ctx.run_until_idle()
        for b, i in zip(before, ids):
            assert np.allclose(ctx.fetch(i)[0], b, rtol=RTOL, atol=ATOL)
    finally:
        ctx.close()


def test_router_spreads_requests_and_keeps_results():
    """Two contexts on one GPU stand in for two devices: the router replicates
    the scenes, sends each request to the context with fewer paths
    outstanding, and every image equals the same render on one context."""
    from pcr_b200 import capi
    a = capi.Context(device=0, queue_capacity=1 << 17)
    b = capi.Context(device=0, queue_capacity=1 << 17)
    try:
        router = capi.Router([a, b])
        names = ["cornell", "cornell-spheres"]
        rsid = {v: router.load_scene_json(scene_path(v), GOLDEN) for v in names}
        sid = {v: a.load_scene_json(scene_path(v), GOLDEN) for v in names}
        reqs = [(names[k % 2], capi.render_desc(32 + 8 * k, depth=3, samples=2 + k % 3, shadow=2, seed=700 + k))
                for k in range(10)]
        want = [a.render(sid[v], d)[0] for v, d in reqs]
        router.serve_start()
        tickets = [router.submit(rsid[v], d) for v, d in reqs]
        got = []
        for t, (_, d) in zip(tickets, reqs):
            router.wait(t, 120_000)
            got.append(router.fetch(t, d.width, d.height)[0])
        router.serve_stop()
        for w, g in zip(want, got):
            assert np.allclose(w, g, rtol=RTOL, atol=ATOL)
        outstanding, routed = router.load()
        assert outstanding == [0, 0]
        assert sum(routed) == len(reqs) and min(routed) >= 3
        with pytest.raises(capi.PcrError):
            router.fetch(tickets[0], 32, 32)     # a ticket is fetched once
        router.close()
    finally:
        a.close()
        b.close()


def test_pending_requests_are_admitted_by_priority():
    """A memory budget that holds one request at a time: after the first,
    pending requests are admitted lowest priority value first, in submit
    order among equals."""
    from pcr_b200 import capi
    ctx = capi.Context(device=0, queue_capacity=1 << 17, memory_budget=128 * 128 * 3 * 13)
    try:
        sid = ctx.load_scene_json(scene_path("cornell"), GOLDEN)

        def d(prio, seed):
            return capi.render_desc(128, depth=2, samples=2, shadow=1, seed=seed, priority=prio)
        ids = {"a": ctx.submit(sid, d(0, 1)), "b": ctx.submit(sid, d(5, 2)), "c": ctx.submit(sid, d(1, 3)),
               "e": ctx.submit(sid, d(1, 4)), "f": ctx.submit(sid, d(-2, 5))}
        ctx.run_until_idle()
        q = {k: ctx.fetch(i, want_hdr=False, want_rgb=False)[2].queue_ms for k, i in ids.items()}
        # nothing was admitted before run_until_idle: f (-2), a (0), c (1), e (1), b (5)
        assert q["f"] < q["a"] < q["c"] < q["e"] < q["b"], q
    finally:
        ctx.close()


def test_wait_times_out_and_serving_restarts():
    """A bounded wait on an unfinished request returns PCR_ERR_TIMEOUT and
    leaves it running; the serve loop can be stopped and started again and
    the request then completes unchanged."""
    from pcr_b200 import capi
    ctx = capi.Context(device=0, queue_capacity=1 << 17)
    try:
        sid = ctx.load_scene_json(scene_path("cornell-glass"), GOLDEN)
        d = capi.render_desc(384, depth=8, samples=48, shadow=4, seed=44)
        ref = ctx.render(sid, d)[0]
        rid = ctx.submit(sid, d)
        with pytest.raises(capi.PcrError) as e:
            ctx.wait(rid, 1)
        assert e.value.status == 6
        ctx.serve_start()
        ctx.serve_stop()
        ctx.serve_start()
        ctx.wait(rid, 120_000)
        ctx.serve_stop()
        assert np.allclose(ctx.fetch(rid)[0], ref, rtol=RTOL, atol=ATOL)
    finally:
        ctx.close()


def test_router_mesh_scene_built_once_matches_one_context():
    """A router scene load with triangles builds the BVH once, on the first
    context's device, and uploads the same tree to every context: renders
    of the mesh scene through the router equal the single-context render."""
    from pcr_b200 import capi, workloads
    a = capi.Context(device=0, queue_capacity=1 << 17)
    b = capi.Context(device=0, queue_capacity=1 << 17)
    try:
        path = workloads.mesh_scene(59, 1)
        router = capi.Router([a, b])
        rsid = router.load_scene_json(path, GOLDEN)
        sid = a.load_scene_json(path, GOLDEN)
        reqs = [capi.render_desc(40 + 8 * k, depth=3, samples=2, shadow=2, seed=900 + k) for k in range(4)]
        want = [a.render(sid, d)[0] for d in reqs]
        router.serve_start()
        tickets = [router.submit(rsid, d) for d in reqs]
        got = []
        for t, d in zip(tickets, reqs):
            router.wait(t, 120_000)
            got.append(router.fetch(t, d.width, d.height)[0])
        router.serve_stop()
        for w, g in zip(want, got):
            assert np.allclose(w, g, rtol=RTOL, atol=ATOL)
        assert min(router.load()[1]) >= 1   # both contexts rendered the mesh
        router.close()
    finally:
        a.close()
        b.close()
