"""The reference-facing surface on the GPU: the `pcr-render` CLI (same flags
as code/Cli/Main.cpp) writes a PNG whose name pattern and tEXt keys match the
reference renderer's (code/Renderer.cpp:393-447) and whose pixels are the
library's tone-mapped output for the same request."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, REPO, scene_path

pytestmark = pytest.mark.gpu

CLI = os.path.join(REPO, "pcr_b200", "lib", "pcr-render")


def test_cli_png_matches_library_and_reference_format(tmp_path):
    from PIL import Image

    from pcr_b200 import build, capi
    build.build()
    args = [CLI, "--scenes-dir", os.path.join(GOLDEN, "scenes"), "--scene", "cornell", "-w", "64", "--height", "48",
            "-d", "3", "-s", "8", "-S", "2", "--spectral", "--seed", "77", "-o", str(tmp_path)]
    out = subprocess.run(args, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    assert "Render took" in out.stdout and "Wrote" in out.stdout
    files = os.listdir(tmp_path)
    assert len(files) == 1
    name = files[0]
    assert re.match(r"cornell-1\.1\.0-\d{8}-\d{6}-[A-Z]+-d3-s8-S2-w64-h48-spectral-t\d+\.png$", name), name
    img = Image.open(tmp_path / name)
    golden = Image.open(os.path.join(GOLDEN, "render", "cornell-spectral.png"))
    assert list(img.text.keys()) == list(golden.text.keys())
    assert img.text["Spectral"] == "1" and img.text["Depth"] == "3" and img.text["Tonemap"] == "Reinhard"
    rgb = np.asarray(img.convert("RGB"))
    ctx = capi.Context()
    sid = ctx.load_scene_json(scene_path("cornell"), GOLDEN)
    _, lib_rgb, _ = ctx.render(sid, capi.render_desc(64, 48, depth=3, samples=8, shadow=2, spectral=True, seed=77))
    ctx.close()
    assert np.array_equal(rgb, lib_rgb)


def test_cli_rejects_unknown_scene():
    out = subprocess.run([CLI, "--scenes-dir", os.path.join(GOLDEN, "scenes"), "--scene", "nope"],
                         capture_output=True, text=True, timeout=60)
    assert out.returncode == 1 and "Unknown scene" in out.stderr


def test_cli_denoise_adaptive_aces_match_library(tmp_path):
    """--denoise, --aa-samples with --adaptive and --aces go through the same
    device paths as the library call with those knobs."""
    from PIL import Image

    from pcr_b200 import capi
    args = [CLI, "--scenes-dir", os.path.join(GOLDEN, "scenes"), "--scene", "cornell-spheres", "-w", "40",
            "--height", "32", "-d", "3", "-s", "4", "-S", "2", "--spectral", "--seed", "5", "--denoise", "--aa",
            "--aa-samples", "6", "--adaptive", "--aces", "-o", str(tmp_path)]
    out = subprocess.run(args, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    files = os.listdir(tmp_path)
    assert len(files) == 1 and "-aces-" in files[0]
    img = Image.open(tmp_path / files[0])
    assert img.text["Adaptive"] == "1" and img.text["Denoise"] == "1"
    rgb = np.asarray(img.convert("RGB"))
    ctx = capi.Context()
    sid = ctx.load_scene_json(scene_path("cornell-spheres"), GOLDEN)
    _, lib_rgb, _ = ctx.render(sid, capi.render_desc(40, 32, depth=3, samples=4, shadow=2, spectral=True, seed=5,
                                                     denoise=True, aa=6, adaptive=True, aces=True))
    ctx.close()
    assert np.array_equal(rgb, lib_rgb)


@pytest.mark.parametrize("terminate", [False, True])
def test_cli_spectral_terminate_matches_library(tmp_path, terminate):
    """--spectral-terminate sets CudaRenderer::spectralFork = false, which
    reaches the device as spectral_terminate; the default forks."""
    from PIL import Image
    from pcr_b200 import capi
    args = [CLI, "--scenes-dir", os.path.join(GOLDEN, "scenes"), "--scene", "cornell-glass", "-w", "40",
            "--height", "40", "-d", "5", "-s", "16", "-S", "2", "--spectral", "--seed", "9", "-o", str(tmp_path)]
    if terminate:
        args.append("--spectral-terminate")
    out = subprocess.run(args, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    files = os.listdir(tmp_path)
    rgb = np.asarray(Image.open(tmp_path / files[0]).convert("RGB"))
    ctx = capi.Context()
    sid = ctx.load_scene_json(scene_path("cornell-glass"), GOLDEN)
    lib = [ctx.render(sid, capi.render_desc(40, 40, depth=5, samples=16, shadow=2, spectral=True, seed=9,
                                            terminate=t))[1] for t in (False, True)]
    ctx.close()
    assert np.array_equal(rgb, lib[int(terminate)])
    assert not np.array_equal(lib[0], lib[1])


def test_renderer_progress_and_cancel(tmp_path):
    """pcr::CudaRenderer polls cancelRequested and fills progressRows between
    blocks of iterations, as the reference renderers poll between pixels or
    tiles (code/Renderer.cpp:170-181, code/Gpu/Opengl/OpenglRenderer.cpp:
    2170-2175).  A 1024x1024 render of 1024 paths per pixel, cancelled from
    another thread once its progress moves, returns within a fraction of a
    second of the cancel and writes no PNG; the next render completes with
    progressRows = height."""
    from pcr_b200 import build
    build.build()
    exe = str(tmp_path / "renderer_cancel")
    lib = os.path.join(REPO, "pcr_b200", "lib")
    cmd = ["g++", "-std=c++17", "-O2", "-o", exe, os.path.join(REPO, "tests", "cpp", "renderer_cancel.cpp"),
           os.path.join(REPO, "pcr_b200", "csrc", "cuda_renderer.cpp"), "-I", os.path.join(REPO, "include"),
           "-I", os.path.join(REPO, "pcr_b200", "csrc"), "-I", "/usr/local/cuda/include", "-L", lib, "-lpcr_b200",
           "-Wl,-rpath," + lib, "-lz", "-lpthread"]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-3000:]
    out = subprocess.run([exe, scene_path("cornell"), GOLDEN, str(tmp_path / "png")], capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stderr[-3000:]
    line = [x for x in out.stdout.splitlines() if x.startswith("rows_at_cancel=")][-1]
    r = dict(kv.split("=") for kv in line.split())
    assert int(r["rows_at_cancel"]) > 0, line          # progress moved while it ran
    assert r["big_written"] == "0", line               # cancelled: no PNG
    assert float(r["cancel_to_return"]) < 1.0, line    # the paths in flight retire, no more are issued
    assert "GPU render cancelled." in out.stdout
    assert r["small_written"] == "1" and int(r["small_rows"]) == 48, line
