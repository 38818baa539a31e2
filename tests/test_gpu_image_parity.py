"""Image parity of every scene against the reference CPU renderer.

The fixtures under tests/golden/converged were made by the reference
renderer itself (oracle/_ref, built from the reference sources; script
tests/golden/make_converged.py): for each scene variant, the Stanford bunny
scene, the emissive-mesh scene and the two ~70k-triangle mesh scenes of the
batched-mesh workload, in spectral (hero-4) and RGB mode, a 64x64 image of
depth 4 and 4 shadow rays averaged over 16384 paths per pixel (8192 on the
mesh scenes) in FP64, and the RMSE of the reference's own paths-per-pixel
estimator against that image at 4 and 16 paths per pixel over 16 seeds.

Gates (the reference's CPU renderer as the oracle):
  * each channel of the GPU image's mean within 0.5 % of the converged CPU
    image's, the GPU image traced with as many paths per pixel;
  * the GPU's RMSE against the converged CPU image at 4 and 16 paths per
    pixel (mean of 4 seeds) within 3 sigma of the CPU estimator's RMSE at
    the same paths per pixel (sigma from the 16 CPU seeds).
The headline configuration's size (cornell, 256x256) is gated the same way
against converged_cornell256.npz.

Both renderers run the same estimator (the GPU backends' paths-per-pixel
meaning of `samples`: one continuation and S shadow rays per diffuse vertex,
the 4-way hero fork at dispersive glass), so the expectations are equal and
so are the error distributions; only the random streams differ.  All
renders of a test go through the batched method in one submission.
"""
import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN, scene_path

pytestmark = pytest.mark.gpu

CONVERGED = os.path.join(GOLDEN, "converged")
CASES = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(CONVERGED, "*-*.npz"))
               if not os.path.basename(p).startswith("cornell-256"))
SEEDS = 4


def _scene_file(name):
    from pcr_b200 import workloads
    if name == "ico59-diffuse":
        return workloads.mesh_scene(59, 21, glass=False)
    if name == "ico59-glass":
        return workloads.mesh_scene(59, 22, glass=True)
    return scene_path(name)


def _split(case):
    name, mode = case.rsplit("-", 1)
    return name, mode == "spectral"


@pytest.fixture(scope="module")
def renders():
    """Every case's renders, submitted together to one context: the
    converged-size image and SEEDS images at each RMSE paths-per-pixel."""
    from pcr_b200 import capi
    ctx = capi.Context(device=0, queue_capacity=1 << 21)
    sids, jobs = {}, []
    for case in CASES:
        name, spectral = _split(case)
        if name not in sids:
            sids[name] = ctx.load_scene_json(_scene_file(name), GOLDEN)
        fx = np.load(os.path.join(CONVERGED, case + ".npz"))
        w, spp = int(fx["width"]), int(fx["spp"])
        seed = 1 + 97 * len(jobs)
        d = capi.render_desc(w, depth=int(fx["depth"]), samples=spp, shadow=int(fx["shadow"]), spectral=spectral,
                             seed=seed)
        jobs.append((case, "mean", 0, ctx.submit(sids[name], d)))
        for spp_k in fx["rmse_spp"]:
            for s in range(SEEDS):
                d = capi.render_desc(w, depth=int(fx["depth"]), samples=int(spp_k), shadow=int(fx["shadow"]),
                                     spectral=spectral, seed=seed + 1 + s + 10 * int(spp_k))
                jobs.append((case, "rmse", int(spp_k), ctx.submit(sids[name], d)))
    # the headline configuration's size: cornell 256x256, spectral
    fx = np.load(os.path.join(CONVERGED, "cornell-256-spectral.npz"))
    c256 = sids.get("cornell") or ctx.load_scene_json(scene_path("cornell"), GOLDEN)
    jobs.append(("cornell-256-spectral", "mean", 0,
                 ctx.submit(c256, capi.render_desc(256, depth=4, samples=int(fx["spp"]), shadow=4, spectral=True,
                                                   seed=31337))))
    for spp_k in fx["rmse_spp"]:
        for s in range(SEEDS):
            jobs.append(("cornell-256-spectral", "rmse", int(spp_k),
                         ctx.submit(c256, capi.render_desc(256, depth=4, samples=int(spp_k), shadow=4,
                                                           spectral=True, seed=4242 + s + 10 * int(spp_k)))))
    ctx.run_until_idle()
    out = {}
    for case, kind, spp_k, rid in jobs:
        hdr = ctx.fetch(rid, want_rgb=False)[0].astype(np.float64)
        out.setdefault((case, kind, spp_k), []).append(hdr)
    ctx.close()
    return out


def _converged_image(case):
    if case == "cornell-256-spectral":
        return np.load(os.path.join(GOLDEN, "converged_cornell256.npz"))["image"].astype(np.float64)
    return np.load(os.path.join(CONVERGED, case + ".npz"))["image"].astype(np.float64)


def test_every_scene_has_fixtures():
    from pcr_b200 import workloads
    names = {_split(c)[0] for c in CASES}
    assert set(workloads.VARIANTS) | {"cornell-mesh-light", "ico59-diffuse", "ico59-glass"} <= names
    assert all(f"{n}-{m}" in CASES for n in names for m in ("spectral", "rgb"))


@pytest.mark.parametrize("case", CASES + ["cornell-256-spectral"])
def test_image_mean_within_half_percent_of_cpu(renders, case):
    g = renders[(case, "mean", 0)][0].reshape(-1, 3).mean(0)
    c = _converged_image(case).reshape(-1, 3).mean(0)
    rel = np.abs(g - c) / np.abs(c)
    assert np.all(rel < 0.005), f"{case}: gpu {g} cpu {c} rel {rel}"


@pytest.mark.parametrize("case", CASES + ["cornell-256-spectral"])
def test_image_rmse_within_3_sigma_of_cpu(renders, case):
    conv = _converged_image(case)
    fx = np.load(os.path.join(CONVERGED, case + ".npz"))
    for k, spp in enumerate(fx["rmse_spp"]):
        cpu = fx["rmse"][k]
        mu, sigma = cpu.mean(), cpu.std(ddof=1)
        gpu = [np.sqrt(np.mean((img - conv) ** 2)) for img in renders[(case, "rmse", int(spp))]]
        assert abs(np.mean(gpu) - mu) <= 3 * sigma, f"{case} spp {spp}: gpu {np.mean(gpu)} cpu {mu} +- {sigma}"
