#!/usr/bin/env python3
"""Benchmark of the B200 wavefront spectral path tracer.

Workload (a "step"): the uneven batch -- 64 renders drawn by seed from the 10
Cornell scene variants, square resolutions log-uniform in 128..1024, depth
2..8, paths per pixel log-uniform in 1..64, shadow rays 1..8, spectral
hero-4, FP32 -- rendered by the batched method (one persistent wavefront
over all 64 requests, graph-captured iterations).  Synthetic seeded data;
the cornell-bunny variant renders the reference's Stanford bunny (a
committed fixture).

Printed (rank 0, one JSON line):
  value        batched paths/s (device time, CUDA events on the engine stream,
               scene cache and requests resident; max over ranks for N > 1)
  e2e          same metric through the C ABI with host buffers: the engine serves
               on its own thread; each step submits the 64 renders from the
               host and copies every HDR + 8-bit image back into the caller's
               buffers as each finishes, host clock
  plain_value  the plain per-request method (one render per launch sequence)
  roofline     dominant wavefront kernel vs measured HBM bandwidth (all three
               in roofline.per_kernel); roofline.bvh_fetch: the mesh leg's
               reference-order BVH-fetch bytes vs measured HBM and L2;
               roofline.fp32_issue: Cornell's plane-test flops vs FP32 peak
  cpu_baseline the reference CPU renderer (oracle/_ref, built from the
               reference sources) on a bounded row sample of the same batch
  mesh_batch   batched mesh scenes (32 renders on the ~70k-triangle mesh)
  serve, serve_scale
               served streams with p50 / p99 latency (Poisson arrivals;
               the at-scale stream mixes heavy 2048^2 renders on a
               1M-triangle mesh with small ones)

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl cuda|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "paths/s, batched+served wavefront (64 uneven spectral renders); plain per-request alongside"
UNIT = "paths/s"
HBM_FALLBACK = 6650.0
# DRAM bytes (read + write) per unit of each wavefront kernel, measured with
# ncu (dram__bytes_read.sum + dram__bytes_write.sum over every launch of one
# 8-render step, divided by that step's rays / shadow rays; each launch
# replayed alone with a cold L2; the summary and command are kept in the
# profiles directory).  Traffic grows in proportion to the units, so a
# launch's traffic is this figure times its units.
NCU_DRAM_PER_UNIT = {"extend": 61.0, "shade": 548.7, "shadow": 83.2}
# Warp instructions per unit (smsp__inst_executed.sum over the same
# launches, divided by the same units), for the issue-rate roofline below.
NCU_INST_PER_UNIT = {"extend": 48.25, "shade": 69.57, "shadow": 43.90}
# Issue-rate side of the same kernels (ncu --set full, one launch each of an
# 8-render batch with the queue full): the share of issue slots used and the
# share of a warp's 32 lanes active per instruction.  The plane and triangle
# tests are dependent IEEE-exact FP32 chains, so these kernels are bound by
# issue and latency rather than by DRAM.
NCU_ISSUE = {"extend": {"issue_slots_busy": 0.638, "lanes_active": 16.2 / 32},
             "shade": {"issue_slots_busy": 0.382, "lanes_active": 23.2 / 32},
             "shadow": {"issue_slots_busy": 0.573, "lanes_active": 17.6 / 32, "l1_busy": 0.649}}
# Algorithmic BVH-fetch bytes per ray of the batched-mesh workload's two
# scenes: 2 x 24 B of child boxes per internal node processed plus 36 B per
# leaf triangle tested, counted by the reference's own traversal order
# (code/Bvh/Bvh.cpp:353-444, restated in the oracle) over every ray of the
# reference estimator on the same scene (camera, continuation and shadow
# rays alike; depth 8, 4 shadow rays, hero-4 spectral).  The figure does not
# depend on the device's tree layout.  tests/test_bvh_fetch_bytes.py
# recomputes it with the oracle and pins these values.
BVH_BYTES_PER_RAY = {"ico59-diffuse": 223.6, "ico59-glass": 1138.9}
# Algorithmic FP32 work of a plane test (3 dot products, 1 divide, 2
# projections onto the quad's edges); the reference tests every plane of the
# scene for every ray, light planes included (code/Renderer.cpp:891-949).
PLANE_TEST_FLOPS = 25


def args_():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="cuda", choices=["cuda", "reference"])
    p.add_argument("--renders", type=int, default=64)
    p.add_argument("--seed", type=int, default=2026)
    p.add_argument("--no-plain", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-profile", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-matched", action="store_true")
    p.add_argument("--queue", type=int, default=0, help="paths in flight (0: library default)")
    p.add_argument("--no-autotune", action="store_true",
                   help="skip the autotuner (queue size, block size, issue chunk, refill cadence)")
    p.add_argument("--serve-requests", type=int, default=2000, help="served stream length (2000: the serving config)")
    p.add_argument("--serve-rate", type=float, default=200.0)
    p.add_argument("--mesh-batch", type=int, default=32,
                   help="batched mesh scenes: renders per step (32 = the mesh configuration; 0: off)")
    p.add_argument("--serve-scale", type=int, default=100,
                   help="serving at scale: requests per stream (0: off; the 1M-triangle mesh is generated on first use)")
    return p.parse_args()


def peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK, "fallback"


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons.  The sampler is
    started before the warm-up (its start-up queries the driver, which must
    not fall inside the timed region) and runs through the timed region; the
    summary keeps the samples whose timestamps lie inside the timed window."""

    Q = ("timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.out = ""
        self.win = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.device), "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def stop(self, window):
        """window: (t0, t1) of the timed region, time.time() seconds."""
        self.win = window
        if self.proc:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        import datetime
        rows = []
        for line in (self.out or "").splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) == 8:
                try:
                    ts = datetime.datetime.strptime(parts[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                    rows.append([ts, float(parts[1]), float(parts[2]), parts[3]] + parts[4:])
                except ValueError:
                    pass
        if self.win:
            inside = [r for r in rows if self.win[0] - 0.05 <= r[0] <= self.win[1] + 0.05]
            rows = inside or rows
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[4 + k].lower() == "active"})
        return {"sm_mhz": float(np.median([r[1] for r in rows])), "sm_max_mhz": max(r[2] for r in rows),
                "samples": len(rows), "reasons": reasons}


def make_batch(n, seed):
    from pcr_b200 import workloads
    return workloads.batch_requests(n, seed=seed)


def scene_files():
    from pcr_b200 import workloads
    return {v: workloads.scene_path(v) for v in workloads.VARIANTS}, workloads.DEFAULT_DATA


# ------------------------------------------------------------------ reference arm
def cpu_sample_step(scenes, batch, rows):
    """One bounded sample of the batch on the reference CPU renderer: `rows`
    pixel rows of every request, spread evenly over its height (the centre
    row of each of `rows` equal bands, so the sample sees the image's
    average content, not only the ceiling and the light), at the request's
    own depth / paths per pixel / shadow rays (the reference's own
    castRaySpectral per path, samples = 1), all host threads.  Returns
    (paths, seconds)."""
    from oracle import ref
    paths, secs = 0, 0.0
    for r in batch:
        o = ref.opts(r["width"], r["height"], depth=r["depth"], samples=1, shadow=r["shadow"], spectral=True,
                     seed=r["seed"])
        picked = ref.spread_rows(r["height"], rows)
        _, s = ref.render_hdr_rows(scenes[r["variant"]], o, picked, spp=r["samples"], threads=0)
        paths += picked.size * r["width"] * r["samples"]
        secs += s
    return paths, secs


def reference_arm(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import ref
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libpcrref.so not built"}))
        return
    files, data = scene_files()
    scenes = {v: ref.load_scene(os.path.abspath(p), data) for v, p in files.items()}
    batch = make_batch(a.renders, a.seed)
    rows = os.cpu_count() or 8   # one row per host thread
    for _ in range(a.warmup):
        cpu_sample_step(scenes, batch, rows)
    tot_p, tot_s = 0, 0.0
    for _ in range(a.steps):
        p, s = cpu_sample_step(scenes, batch, rows)
        tot_p += p
        tot_s += s
    v = tot_p / tot_s
    cores = os.cpu_count()
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": 1e3 * tot_s / a.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded batch of the 10 Cornell variants)",
        "config": {"workload": f"batch{a.renders}-uneven", "sample": f"{rows} pixel rows spread evenly over each render"},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": f"{rows} rows spread evenly over each of the {a.renders} renders per step"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


# ------------------------------------------------------------------ matched image error
def matched_run(ctx, sids, stream, a, with_cpu, tune, sm_mhz):
    """The Cornell configuration at matched image error: cornell.json at
    256x256, depth 4, S = 4, hero-4 spectral, Reinhard.  The target error is
    the RMSE of the reference CPU renderer's branched s = 16 image against a
    4096-path converged image (both made by the reference itself,
    tests/golden/converged_cornell256.npz).  spp* is the smallest paths per
    pixel whose mean RMSE over 4 seeds reaches that target; the GPU then
    renders W*H*spp* paths per image, plain (one render per launch sequence)
    and batched (64 seeds in one wavefront).  The CPU time is the branched
    s = 16 render on a row sample, all host threads, scaled to the image."""
    import torch

    from pcr_b200 import capi
    fx = np.load(os.path.join(REPO, "tests", "golden", "converged_cornell256.npz"))
    conv, eps = fx["image"].astype(np.float64), float(fx["branched_rmse"])
    sid, W = sids["cornell"], 256

    def desc(spp, seed):
        return capi.render_desc(W, depth=4, samples=spp, shadow=4, spectral=True, seed=seed)

    def rmse(spp, seed):
        hdr, _, _ = ctx.render(sid, desc(spp, seed), want_rgb=False)
        return float(np.sqrt(np.mean((hdr.astype(np.float64) - conv) ** 2)))

    spp_star, err = None, None
    for spp in range(1, 65):
        err = float(np.mean([rmse(spp, 1 + k) for k in range(4)]))
        if err <= eps:
            spp_star = spp
            break
    if spp_star is None:
        return {"target_rmse": eps, "spp_star": None, "note": "target not reached by 64 paths per pixel"}
    paths = W * W * spp_star
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for k in range(3):
        ctx.render(sid, desc(spp_star, 100 + k), want_hdr=False, want_rgb=False)
    reps = 20
    torch.cuda.synchronize()
    e0.record(stream)
    for k in range(reps):
        ctx.render(sid, desc(spp_star, 200 + k), want_hdr=False, want_rgb=False)
    e1.record(stream)
    torch.cuda.synchronize()
    plain_s = e0.elapsed_time(e1) / 1e3 / reps
    nb = 64

    def batch(seed0):
        ids = [ctx.submit(sid, desc(spp_star, seed0 + k)) for k in range(nb)]
        ctx.run_until_idle()
        for i in ids:
            ctx.fetch(i, want_hdr=False, want_rgb=False)
    batch(300)
    torch.cuda.synchronize()
    e0.record(stream)
    batch(400)
    e1.record(stream)
    torch.cuda.synchronize()
    batched_s = e0.elapsed_time(e1) / 1e3 / nb
    fp32 = None
    if not a.no_profile:
        # FP32 roofline of the plane scene: the reference tests all 18 planes
        # for every ray (camera, continuation and shadow rays); a profiled
        # context times the two trace kernels over the same 64-image batch
        pctx = capi.Context(device=ctx.device, profile=True, **tune)
        psid = pctx.load_scene_json(os.path.join(REPO, "tests", "golden", "scenes", "cornell.json"),
                                    os.path.join(REPO, "tests", "golden"))
        ids = [pctx.submit(psid, desc(spp_star, 500 + k)) for k in range(nb)]
        pctx.run_until_idle()
        for i in ids:
            pctx.fetch(i, want_hdr=False, want_rgb=False)
        ps = pctx.stats()
        pctx.close()
        rays = ps["rays"] + ps["shadow_rays"]
        t = (ps["stage_ms"]["extend"] + ps["stage_ms"]["shadow"]) / 1e3
        mhz = sm_mhz or 1965.0
        peak = 148 * 128 * 2 * mhz * 1e6 / 1e12
        ach = rays * 18 * PLANE_TEST_FLOPS / t / 1e12
        fp32 = {"kernels": "k_extend + k_shadow", "rays": rays, "flops_per_ray": 18 * PLANE_TEST_FLOPS,
                "achieved": ach, "unit": "TFLOP/s", "peak": peak, "frac": ach / peak,
                "peak_basis": f"148 SMs x 128 FP32 lanes x 2 (FMA) x {mhz:.0f} MHz (sampled SM clock)",
                "flops": f"{PLANE_TEST_FLOPS} per plane test x 18 planes per ray, the reference's per-ray work",
                "rays_per_s_in_trace_kernels": rays / t}
    out = {"config": "cornell.json 256x256, depth 4, S=4, hero-4 spectral, Reinhard", "fp32_roofline": fp32,
           "target_rmse": eps, "target": "reference CPU branched s=16 image vs 4096-path converged image",
           "spp_star": spp_star, "gpu_rmse_at_spp_star": err, "paths_per_image": paths,
           "plain_ms_per_image": plain_s * 1e3, "plain_paths_s": paths / plain_s,
           "batched_ms_per_image": batched_s * 1e3, "batched_paths_s": paths / batched_s, "batched_images": nb}
    if with_cpu:
        try:
            from oracle import ref
            if ref.available():
                sc = ref.load_scene(os.path.join(REPO, "tests", "golden", "scenes", "cornell.json"),
                                    os.path.join(REPO, "tests", "golden"))
                # four bands spread over the image, one row per host thread in each
                band = min(W // 8, os.cpu_count() or 8)
                o = ref.opts(W, depth=4, samples=16, shadow=4, spectral=True, seed=1)
                secs = 0.0
                for b in range(4):
                    r0 = b * (W // 4) + (W // 8)
                    secs += ref.render_hdr(sc, o, mode=0, threads=0, rows=(r0, r0 + band))[1]
                t_img = secs * W / (4 * band)
                out.update({"cpu_branched_s_per_image": t_img, "cpu_cores": os.cpu_count(),
                            "cpu_sample": f"4 bands of {band} rows of the branched s=16 render, scaled to {W} rows",
                            "cpu_equiv_paths_s": paths / t_img,
                            "plain_over_cpu": t_img / plain_s, "batched_over_cpu": t_img / batched_s})
        except Exception as e:  # reported, not fatal
            out["cpu_error"] = str(e)
    return out


# ------------------------------------------------------------------ served stream
def serve_run(ctx, sids, files, data, a, n=None, rate=None, seed_off=17):
    """Requests arrive by a Poisson process at `rate` req/s (scene drawn from
    the 10 variants, 20 % the seeded ~70k-triangle mesh scene, glass or
    Lambertian by seed; square resolution log-uniform 64..1024, depth 2..8,
    paths per pixel 1..64, shadow rays 1..8).  The engine serves them on its
    own thread; a request is admitted as slots and the device-memory budget
    free up, and its paths share the queue with everything in flight.
    Latency is submit -> result on the host, per request."""
    from pcr_b200 import capi, workloads
    mesh = {False: ctx.load_scene_json(workloads.mesh_scene(59, 11, glass=False), data),
            True: ctx.load_scene_json(workloads.mesh_scene(59, 12, glass=True), data)}
    n = n or a.serve_requests
    rate = rate or a.serve_rate
    reqs = workloads.request_stream(n, rate, seed=a.seed + seed_off)
    ctx.serve_start()
    t0 = time.perf_counter()
    ids = []
    for r in reqs:
        now = time.perf_counter() - t0
        if r["arrival"] > now:
            time.sleep(r["arrival"] - now)
        sid = mesh[bool(r["seed"] & 1)] if r["variant"] == "mesh" else sids[r["variant"]]
        d = capi.render_desc(r["width"], r["height"], depth=r["depth"], samples=r["samples"], shadow=r["shadow"],
                             spectral=True, seed=r["seed"])
        ids.append((ctx.submit(sid, d), r))
    lat, paths, t_last = [], 0, 0.0
    for rid, r in ids:
        ctx.wait(rid, 600_000)
        _, _, st = ctx.fetch(rid, want_hdr=False, want_rgb=False)
        lat.append(st.latency_ms)
        paths += st.paths
        t_last = max(t_last, r["arrival"] * 1e3 + st.latency_ms)
    ctx.serve_stop()
    lat = np.asarray(lat)
    return {"requests": len(ids), "rate_req_s": rate, "p50_ms": float(np.percentile(lat, 50)),
            "p99_ms": float(np.percentile(lat, 99)), "max_ms": float(lat.max()),
            "paths_per_s": paths / (t_last / 1e3), "span_s": t_last / 1e3,
            "offered_paths_per_s": paths / max(reqs[-1]["arrival"], 1e-9),
            "mesh_fraction": 0.2, "resolution": "log-uniform 64..1024"}


def serve_scale_run(ctx, sids, data, a):
    """Serving at scale: 10 % heavy requests (2048x2048, depth 8, 64 paths
    per pixel, 4 shadow rays) over the seeded 1,003,520-triangle displaced
    icosphere, 90 % small ones (square 64..256, the served stream's scene
    mix: the 10 variants and 20 % the ~70k-triangle mesh).  A closed-loop
    pass (every request submitted at once) measures the saturation rate; the
    reported stream then arrives by a Poisson process at 80 % of it."""
    from pcr_b200 import capi, workloads
    mesh = {False: ctx.load_scene_json(workloads.mesh_scene(59, 11, glass=False), data),
            True: ctx.load_scene_json(workloads.mesh_scene(59, 12, glass=True), data)}
    path = workloads.mesh_scene(224, 1)
    t0 = time.perf_counter()
    big = ctx.load_scene_json(path, data)
    load_s = time.perf_counter() - t0
    heavy = {"variant": "mesh1m", "width": 2048, "height": 2048, "depth": 8, "samples": 64, "shadow": 4}

    def run(reqs):
        ctx.serve_start()
        t0 = time.perf_counter()
        ids = []
        for r in reqs:
            now = time.perf_counter() - t0
            if r["arrival"] > now:
                time.sleep(r["arrival"] - now)
            sid = (big if r["variant"] == "mesh1m" else
                   mesh[bool(r["seed"] & 1)] if r["variant"] == "mesh" else sids[r["variant"]])
            d = capi.render_desc(r["width"], r["height"], depth=r["depth"], samples=r["samples"],
                                 shadow=r["shadow"], spectral=True, seed=r["seed"])
            ids.append((ctx.submit(sid, d), r))
        lat, hv, paths, t_last = [], [], 0, 0.0
        for rid, r in ids:
            ctx.wait(rid, 600_000)
            _, _, st = ctx.fetch(rid, want_hdr=False, want_rgb=False)
            lat.append(st.latency_ms)
            hv.append(r["variant"] == "mesh1m")
            paths += st.paths
            t_last = max(t_last, r["arrival"] * 1e3 + st.latency_ms)
        ctx.serve_stop()
        return np.asarray(lat), np.asarray(hv), paths, t_last / 1e3

    n = a.serve_scale
    mix = dict(res=(64, 256), mesh_fraction=0.2, heavy_fraction=0.1, heavy=heavy)
    _, _, sat_paths, sat_span = run(workloads.request_stream(n, 1e9, seed=a.seed + 41, **mix))
    sat_rate = n / sat_span
    reqs = workloads.request_stream(n, 0.8 * sat_rate, seed=a.seed + 43, **mix)
    lat, hv, paths, span = run(reqs)

    def pct(x, q):
        return float(np.percentile(x, q)) if x.size else None
    return {"requests": n, "heavy": int(hv.sum()), "saturation_req_s": sat_rate,
            "saturation_paths_per_s": sat_paths / sat_span, "rate_req_s": 0.8 * sat_rate,
            "p50_ms": pct(lat, 50), "p99_ms": pct(lat, 99), "max_ms": float(lat.max()),
            "small_p50_ms": pct(lat[~hv], 50), "small_p99_ms": pct(lat[~hv], 99),
            "heavy_p50_ms": pct(lat[hv], 50), "heavy_p99_ms": pct(lat[hv], 99),
            "paths_per_s": paths / span, "span_s": span, "mesh_1m_load_s": load_s,
            "mix": "10 % 2048x2048 d8 s64 S4 on 1,003,520 triangles; 90 % 64..256 squares"}


def mesh_batch_run(ctx, stream, data, a, tune, hbm_peak, l2_peak):
    """Batched mesh scenes: the Cornell box with the seeded ~70k-triangle
    displaced icosphere, glass or Lambertian by seed (50/50); `n` renders
    per step, square resolution log-uniform 512..1024, depth 8, 32 paths per
    pixel, 4 shadow rays.  Device-timed like the main batched value (one
    warm-up step, then up to 3 steps).

    BVH-fetch roofline: a profiled context renders each scene's share of the
    batch alone; its rays (path vertices + shadow rays) times the scene's
    algorithmic bytes per ray (BVH_BYTES_PER_RAY) over the CUDA-event time
    of the two trace kernels (k_extend + k_shadow) is the achieved BVH-fetch
    bandwidth, against the measured HBM copy bandwidth and the measured L2
    L2 read bandwidth (the mesh's nodes and triangles, ~8 MB, stay in L2)."""
    import torch

    from pcr_b200 import capi, workloads
    files = {g: workloads.mesh_scene(59, 21 + int(g), glass=g) for g in (False, True)}
    sids = {g: ctx.load_scene_json(files[g], data) for g in (False, True)}
    rng = np.random.default_rng(a.seed + 53)
    batch = []
    for _ in range(a.mesh_batch):
        side = int(round(np.exp(rng.uniform(np.log(512), np.log(1024)))))
        batch.append((bool(rng.integers(0, 2)), capi.render_desc(side, depth=8, samples=32, shadow=4,
                                                                 spectral=True, seed=int(rng.integers(1, 2**31)))))
    paths = sum(d.width * d.height * d.samples for _, d in batch)
    steps = max(1, min(a.steps, 3))

    def step():
        ids = [ctx.submit(sids[g], d) for g, d in batch]
        ctx.run_until_idle()
        for i in ids:
            ctx.fetch(i, want_hdr=False, want_rgb=False)
    step()
    ctx.reset_stats()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(steps):
        step()
    ev1.record(stream)
    torch.cuda.synchronize()
    sec = ev0.elapsed_time(ev1) / 1e3
    st = ctx.stats()
    for v in sids.values():
        ctx.release_scene(v)
    out = {"renders": a.mesh_batch, "paths_per_step": paths, "paths_per_s": paths * steps / sec,
           "rays_per_s": (st["rays"] + st["shadow_rays"]) / sec, "ms_per_step": sec * 1e3 / steps, "steps": steps,
           "triangles": 69620, "config": "512..1024 squares, depth 8, 32 paths per pixel, S 4, glass / Lambertian 50/50"}
    if a.no_profile:
        return out
    roof = {}
    for g in (False, True):
        name = "ico59-glass" if g else "ico59-diffuse"
        pctx = capi.Context(device=ctx.device, profile=True, **tune)
        psid = pctx.load_scene_json(files[g], data)
        ids = [pctx.submit(psid, d) for gg, d in batch if gg == g]
        pctx.run_until_idle()
        for i in ids:
            pctx.fetch(i, want_hdr=False, want_rgb=False)
        ps = pctx.stats()
        pctx.close()
        rays = ps["rays"] + ps["shadow_rays"]
        t = (ps["stage_ms"]["extend"] + ps["stage_ms"]["shadow"]) / 1e3
        gbs = rays * BVH_BYTES_PER_RAY[name] / t / 1e9
        roof[name] = {"renders": len(ids), "rays": rays, "bytes_per_ray": BVH_BYTES_PER_RAY[name],
                      "trace_ms": t * 1e3, "achieved": gbs, "unit": "GB/s", "frac_hbm": gbs / hbm_peak,
                      "frac_l2": gbs / l2_peak if l2_peak else None,
                      "rays_per_s_in_trace_kernels": rays / t}
    tot_b = sum(v["rays"] * v["bytes_per_ray"] for v in roof.values())
    tot_t = sum(v["trace_ms"] for v in roof.values()) / 1e3
    out["bvh_fetch"] = {"kernels": "k_extend + k_shadow", "achieved": tot_b / tot_t / 1e9, "unit": "GB/s",
                        "peak_hbm": hbm_peak, "frac_hbm": tot_b / tot_t / 1e9 / hbm_peak, "peak_l2": l2_peak,
                        "frac_l2": tot_b / tot_t / 1e9 / l2_peak if l2_peak else None, "per_scene": roof,
                        "bytes": "2 x 24 B per internal node processed + 36 B per leaf triangle tested, "
                                 "reference traversal order, per ray of the reference estimator"}
    return out


# ------------------------------------------------------------------ CUDA arm
def main():
    a = args_()
    if a.impl == "reference":
        reference_arm(a)
        return
    from pcr_b200.replicas import Replicas
    rep = Replicas("nccl")
    world, rank, local = rep.world, rep.rank, rep.local
    import torch

    from pcr_b200 import capi
    torch.cuda.set_device(local)
    ctx = capi.Context(device=local, queue_capacity=a.queue)
    stream = torch.cuda.ExternalStream(ctx.stream())
    files, data = scene_files()
    sids = {v: ctx.load_scene_json(p, data) for v, p in files.items()}
    batch = make_batch(a.renders, rep.seed(a.seed))
    descs = [capi.render_desc(r["width"], r["height"], depth=r["depth"], samples=r["samples"], shadow=r["shadow"],
                              spectral=True, seed=r["seed"]) for r in batch]
    step_paths = sum(r["width"] * r["height"] * r["samples"] for r in batch)
    autotune = None
    if not a.no_autotune and not a.queue:
        # the library's autotuner times a grid of tunings on a sample of the
        # batch (every 4th render) and keeps the fastest for the run
        sub = list(range(0, len(batch), 4))
        t0 = time.perf_counter()
        chosen = ctx.autotune([sids[batch[k]["variant"]] for k in sub], [descs[k] for k in sub])
        autotune = {"chosen": chosen, "sample_renders": len(sub), "seconds": time.perf_counter() - t0}

    def batched_step(want_images=False):
        ids = [ctx.submit(sids[r["variant"]], d) for r, d in zip(batch, descs)]
        ctx.run_until_idle()
        for i in ids:
            ctx.fetch(i, want_hdr=want_images, want_rgb=want_images)

    barrier, max_over_ranks, sum_over_ranks = rep.barrier, rep.max, rep.sum

    clk = Clocks(local).start()
    for _ in range(a.warmup):
        batched_step()
    ctx.reset_stats()
    # ---- device-timed batched region
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t_w0 = time.time()
    ev0.record(stream)
    for _ in range(a.steps):
        batched_step()
    ev1.record(stream)
    torch.cuda.synchronize()
    t_w1 = time.time()
    clk.stop((t_w0, t_w1))
    barrier()
    ms = max_over_ranks(ev0.elapsed_time(ev1))
    st = ctx.stats()
    launches = sum(st["stage_launches"].values()) + a.steps * a.renders
    total_paths = sum_over_ranks(step_paths * a.steps)
    value = total_paths / (ms / 1e3)
    rays = sum_over_ranks(st["rays"] + st["shadow_rays"]) / (ms / 1e3)

    # ---- e2e: host buffers in and out through the C ABI, host clock.  The
    # engine serves on its own thread; each step submits the 64 renders from
    # the host and copies every finished HDR + 8-bit image back as soon as it
    # is ready, while the rest still render (continuous batching).
    e2e = None
    if not a.no_e2e:
        # the caller's host image buffers, allocated once
        outs = [(np.zeros((r["height"], r["width"], 3), np.float32), np.zeros((r["height"], r["width"], 3), np.uint8))
                for r in batch]

        def served_step():
            ids = {ctx.submit(sids[r["variant"]], d): k for k, (r, d) in enumerate(zip(batch, descs))}
            left = set(ids)
            while left:
                ready = [i for i in left if ctx.poll(i)]
                for i in ready:
                    ctx.fetch(i, hdr_out=outs[ids[i]][0], rgb_out=outs[ids[i]][1])
                    left.discard(i)
                if left and not ready:
                    time.sleep(0.0005)
        ctx.serve_start()
        served_step()   # warm-up of the served path
        barrier()
        t0 = time.perf_counter()
        for _ in range(a.steps):
            served_step()
        barrier()
        e2e_s = max_over_ranks(time.perf_counter() - t0)
        ctx.serve_stop()
        e2e = total_paths / e2e_s
    d2h = sum(r["width"] * r["height"] * 15 for r in batch)
    h2d = a.renders * 96

    # ---- plain method on the same batch (one render per launch sequence)
    plain = None
    if not a.no_plain:
        barrier()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        for r, d in zip(batch, descs):
            ctx.render(sids[r["variant"]], d, want_hdr=False, want_rgb=False)
        p1.record(stream)
        torch.cuda.synchronize()
        pms = max_over_ranks(p0.elapsed_time(p1))
        plain = sum_over_ranks(step_paths) / (pms / 1e3)

    # ---- per-stage events (profiled pass) for the roofline
    roofline = None
    if not a.no_profile:
        tune = {k: st[k] for k in ("queue_capacity", "block_size", "chunk_paths", "regen_every")}
        pctx = capi.Context(device=local, profile=True, **tune)
        psids = {v: pctx.load_scene_json(p, data) for v, p in files.items()}
        ids = [pctx.submit(psids[r["variant"]], d) for r, d in zip(batch, descs)]
        pctx.run_until_idle()
        for i in ids:
            pctx.fetch(i, want_hdr=False, want_rgb=False)
        ps = pctx.stats()
        pctx.close()
        peak, kind = peaks()
        # algorithmic bytes per unit (queue records, 16-byte words):
        #   extend: ray in (origin, dir, id: 48 B) + hit out (16 B)
        #   shadow: shadow record in (48 B)
        #   shade : spectral path in (o, d, tp, id, XYZ weights: 112 B) + hit in (16 B)
        #           + path out (112 B) + shadow out (48 B each)
        bytes_stage = {"extend": 64.0 * ps["rays"], "shadow": 48.0 * ps["shadow_rays"],
                       "shade": 240.0 * ps["rays"] + 48.0 * ps["shadow_rays"]}
        dom = max(bytes_stage, key=lambda k: ps["stage_ms"][k])
        t_ms = ps["stage_ms"][dom]
        n_l = max(1, ps["stage_launches"][dom])
        achieved = bytes_stage[dom] / (t_ms / 1e3) / 1e9
        units = ps["shadow_rays"] if dom == "shadow" else ps["rays"]
        traffic = NCU_DRAM_PER_UNIT[dom] * units / n_l if dom in NCU_DRAM_PER_UNIT else None
        # every wavefront kernel against the same bound, for the full picture
        per_kernel = {}
        for k in bytes_stage:
            if ps["stage_ms"][k] <= 0:
                continue
            nk = max(1, ps["stage_launches"][k])
            gbs = bytes_stage[k] / (ps["stage_ms"][k] / 1e3) / 1e9
            uk = ps["shadow_rays"] if k == "shadow" else ps["rays"]
            per_kernel[f"k_{k}"] = {"ms": ps["stage_ms"][k], "achieved_gbs": gbs, "frac_hbm": gbs / peak,
                                    "ncu_traffic_per_launch": NCU_DRAM_PER_UNIT[k] * uk / nk,
                                    "algorithmic_bytes_per_launch": bytes_stage[k] / nk}
        roofline = {"bound": "hbm", "kernel": f"k_{dom}", "achieved": achieved, "peak": peak, "unit": "GB/s",
                    "frac": achieved / peak, "peak_kind": kind, "traffic": traffic,
                    "traffic_note": "ncu DRAM bytes per unit (8-render capture) x units per launch",
                    "bytes_per_launch": bytes_stage[dom] / n_l, "ms_per_launch": t_ms / n_l,
                    "issue": dict(NCU_ISSUE.get(dom, {}), note="ncu, one launch per kernel of an 8-render batch"),
                    "stage_ms": ps["stage_ms"], "stage_share": {k: v / max(1e-9, sum(ps["stage_ms"].values()))
                                                                for k, v in ps["stage_ms"].items()},
                    "per_kernel": per_kernel}
        # The bound that applies: instruction issue.  The same kernel's warp
        # instructions (ncu per unit x units) over its CUDA-event time,
        # against one warp instruction per cycle per scheduler (4 per SM) at
        # the SM clock sampled during the timed region.
        if dom in NCU_INST_PER_UNIT:
            mhz = clk.summary().get("sm_mhz") or 1965.0
            sms = torch.cuda.get_device_properties(local).multi_processor_count
            ach = NCU_INST_PER_UNIT[dom] * units / (t_ms / 1e3)
            pk = sms * 4 * mhz * 1e6
            roofline["issue_roofline"] = {"achieved": ach, "peak": pk, "unit": "warp instructions/s",
                                          "frac": ach / pk, "warp_inst_per_unit": NCU_INST_PER_UNIT[dom],
                                          "sm_mhz": mhz, "sms": sms}

    # ---- served stream: Poisson arrivals, continuous batching, p50/p99
    serve = None
    if a.serve_requests > 0:
        serve = serve_run(ctx, sids, files, data, a)
        # the configured 200 req/s exceeds what one GPU serves, so latency
        # there is mostly backlog; a second stream arrives at 80 % of the
        # measured service rate (requests served per second above)
        cap = serve["requests"] / serve["span_s"]
        serve["at_80pct_capacity"] = serve_run(ctx, sids, files, data, a, n=min(400, a.serve_requests),
                                               rate=0.8 * cap, seed_off=29)

    serve_scale = serve_scale_run(ctx, sids, data, a) if a.serve_scale > 0 else None
    tune = {k: st[k] for k in ("queue_capacity", "block_size", "chunk_paths", "regen_every")}
    hbm_peak, hbm_kind = peaks()
    # measured L2 read bandwidth (the library's probe: a 32 MiB buffer read
    # 400 times with L1-bypassing loads), best of 3
    l2_peak = max(ctx.l2_bandwidth(32 << 20, 400) for _ in range(3)) if not a.no_profile else None
    mesh_batch = mesh_batch_run(ctx, stream, data, a, tune, hbm_peak, l2_peak) if a.mesh_batch > 0 else None

    # ---- Cornell configuration at matched image error
    matched = None
    if not a.no_matched:
        matched = matched_run(ctx, sids, stream, a, with_cpu=(not a.no_cpu and rank == 0 and world == 1), tune=tune,
                              sm_mhz=clk.summary().get("sm_mhz"))

    # ---- CPU baseline (rank 0, N = 1): reference renderer on a row sample
    cpu = None
    if not a.no_cpu and rank == 0 and world == 1:
        try:
            from oracle import ref
            if ref.available():
                rscenes = {v: ref.load_scene(os.path.abspath(p), data) for v, p in files.items()}
                rows = os.cpu_count() or 8   # one row per host thread
                pp, ss = cpu_sample_step(rscenes, batch, rows)
                cpu = {"value": pp / ss, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                       "sample": f"{rows} pixel rows spread evenly over each of the {a.renders} renders "
                                 f"({pp} paths, {ss:.1f} s)"}
        except Exception as e:  # reported, not fatal
            cpu = {"value": None, "error": str(e)}

    if roofline is not None:
        # the path's own rooflines (bounds of the work the reference defines):
        # BVH-fetch bytes on the mesh scenes, FP32 plane tests on cornell
        roofline["bvh_fetch"] = (mesh_batch or {}).get("bvh_fetch")
        roofline["fp32_issue"] = (matched or {}).get("fp32_roofline")
        roofline["l2_peak_gbs"] = l2_peak
    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32",
            "data": "synthetic: seeded 64-render batch of the 10 Cornell variants (cornell-bunny with the "
                    "reference's Stanford bunny, a committed fixture)",
            "config": {"workload": f"batch{a.renders}-uneven", "renders": a.renders, "paths_per_step": step_paths,
                       "parallelism": f"replicas x{world} (own seeded batch per GPU, no collective)",
                       "resolution": "square, log-uniform 128..1024", "depth": "2..8", "paths_per_pixel": "1..64",
                       "shadow_rays": "1..8", "spectral": "hero-4",
                       "l2": "path/shadow queues (2-40 GB at the tuned 1M-16M paths in flight) > 126 MB L2 (no flush needed)"},
            "rays_per_s": rays,
            "work": {"paths": step_paths * a.steps, "rays": st["rays"], "shadow_rays": st["shadow_rays"],
                     "iterations": st.get("iterations")},
            "plain_value": plain, "batched_over_plain": (value / plain) if plain else None,
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "roofline": roofline, "cpu_baseline": cpu, "clocks": clk.summary(), "gpu_launches": launches,
            "serve": serve, "serve_scale": serve_scale, "mesh_batch": mesh_batch, "matched_rmse": matched,
            "tuning": {k: st[k] for k in ("queue_capacity", "block_size", "chunk_paths", "regen_every")},
            "autotune": autotune,
        }
        print(json.dumps(out))
    ctx.close()
    rep.close()


if __name__ == "__main__":
    main()
