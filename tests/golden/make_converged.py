"""Generates the converged-image fixtures with the reference CPU renderer
itself (oracle/_ref/libpcrref.so, built from the reference sources):

  converged_cornell64.npz   cornell, 64x64, spectral hero-4, depth 4, S=4,
                            16384 paths per pixel centre, FP64 mean, plus the
                            RMSE of the reference's own paths-per-pixel
                            estimator at spp 4/16/64 over 16 seeds each.
  converged_cornell256.npz  the 256x256 image of the headline configuration
                            (4096 paths per pixel), the reference's branched
                            s=16 render of that configuration and its RMSE
                            (the matched-RMSE target), with the CPU time.
  converged/<scene>-<mode>.npz
                            every scene variant, the reference's bunny, the
                            emissive-mesh scene and the two ~70k-triangle
                            mesh scenes of the batched-mesh workload, each in
                            spectral (hero-4) and RGB mode: 64x64, depth 4,
                            S = 4, paths through the pixel centre, FP64 mean
                            of 16384 paths per pixel (8192 for the mesh
                            scenes), plus the RMSE of the reference's own
                            paths-per-pixel estimator against that image at
                            4 and 16 paths per pixel over 16 seeds each.
                            cornell-256-spectral.npz holds the same
                            statistics at 256x256 (the headline
                            configuration's size) around the image of
                            converged_cornell256.npz.

    python tests/golden/make_converged.py [64|256|scenes|all]
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import ref  # noqa: E402


def scene():
    return ref.load_scene(os.path.join(HERE, "scenes", "cornell.json"), HERE)


def rmse(a, b):
    return float(np.sqrt(np.mean((a - b) ** 2)))


def make64():
    s = scene()
    o = ref.opts(64, depth=4, samples=1, shadow=4, spectral=True, seed=99)
    t = time.time()
    conv, _ = ref.render_hdr(s, o, mode=1, spp=16384, threads=0)
    print("converged 64:", time.time() - t, "s", flush=True)
    stats = {}
    for spp in (4, 16, 64):
        r = []
        for k in range(16):
            img, _ = ref.render_hdr(s, ref.opts(64, depth=4, samples=1, shadow=4, spectral=True, seed=1000 + k),
                                    mode=1, spp=spp, threads=0)
            r.append(rmse(img, conv))
        stats[spp] = r
        print("spp", spp, np.mean(r), np.std(r), flush=True)
    np.savez_compressed(os.path.join(HERE, "converged_cornell64.npz"), image=conv.astype(np.float32),
                        spp=16384, rmse_spp=np.array(sorted(stats)),
                        rmse=np.array([stats[k] for k in sorted(stats)]))


def make256():
    s = scene()
    o = ref.opts(256, depth=4, samples=1, shadow=4, spectral=True, seed=7)
    t = time.time()
    conv, secs_c = ref.render_hdr(s, o, mode=1, spp=4096, threads=0)
    print("converged 256:", time.time() - t, "s", flush=True)
    ob = ref.opts(256, depth=4, samples=16, shadow=4, spectral=True, seed=11)
    branched, secs_b = ref.render_hdr(s, ob, mode=0, threads=0)
    eps = rmse(branched, conv)
    print("branched s=16 rmse", eps, "cpu s", secs_b, flush=True)
    np.savez_compressed(os.path.join(HERE, "converged_cornell256.npz"), image=conv.astype(np.float32), spp=4096,
                        branched=branched.astype(np.float32), branched_rmse=eps, branched_seconds=secs_b,
                        threads=os.cpu_count())


# (name, scene JSON, converged paths per pixel)
def scene_list():
    from pcr_b200 import workloads
    out = [(v, os.path.join(HERE, "scenes", v + ".json"), 16384) for v in workloads.VARIANTS]
    out.append(("cornell-mesh-light", os.path.join(HERE, "scenes", "cornell-mesh-light.json"), 16384))
    # the batched-mesh workload's two scenes (seeded displaced icospheres)
    out.append(("ico59-diffuse", workloads.mesh_scene(59, 21, glass=False), 8192))
    out.append(("ico59-glass", workloads.mesh_scene(59, 22, glass=True), 8192))
    return out


RMSE_SPP = (4, 16)


def stats(s, width, spectral, conv, seeds=16):
    out = []
    for spp in RMSE_SPP:
        r = []
        for k in range(seeds):
            img, _ = ref.render_hdr(s, ref.opts(width, depth=4, samples=1, shadow=4, spectral=spectral,
                                                seed=1000 + k), mode=1, spp=spp, threads=0)
            r.append(rmse(img, conv))
        out.append(r)
    return np.array(out)


def make_scenes(only=None):
    os.makedirs(os.path.join(HERE, "converged"), exist_ok=True)
    for name, path, n in scene_list():
        if only and name not in only:
            continue
        s = ref.load_scene(os.path.abspath(path), HERE)
        for spectral in (True, False):
            mode = "spectral" if spectral else "rgb"
            t = time.time()
            conv, _ = ref.render_hdr(s, ref.opts(64, depth=4, samples=1, shadow=4, spectral=spectral, seed=99),
                                     mode=1, spp=n, threads=0)
            r = stats(s, 64, spectral, conv)
            np.savez_compressed(os.path.join(HERE, "converged", f"{name}-{mode}.npz"), image=conv.astype(np.float32),
                                spp=n, width=64, depth=4, shadow=4, spectral=spectral,
                                rmse_spp=np.array(RMSE_SPP), rmse=r)
            print(name, mode, f"{time.time() - t:.1f} s", conv.reshape(-1, 3).mean(0), r.mean(1), flush=True)
    if not only or "cornell-256" in only:
        s = scene()
        conv = np.load(os.path.join(HERE, "converged_cornell256.npz"))["image"].astype(np.float64)
        r = stats(s, 256, True, conv)
        np.savez_compressed(os.path.join(HERE, "converged", "cornell-256-spectral.npz"), spp=4096, width=256,
                            depth=4, shadow=4, spectral=True, rmse_spp=np.array(RMSE_SPP), rmse=r)
        print("cornell 256", r.mean(1), flush=True)


if __name__ == "__main__":
    what = sys.argv[1] if len(sys.argv) > 1 else "all"
    if what in ("64", "all"):
        make64()
    if what in ("256", "all"):
        make256()
    if what in ("scenes", "all"):
        make_scenes(sys.argv[2:] or None)
