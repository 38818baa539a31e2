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

    python tests/golden/make_converged.py [64|256|all]
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


if __name__ == "__main__":
    what = sys.argv[1] if len(sys.argv) > 1 else "all"
    if what in ("64", "all"):
        make64()
    if what in ("256", "all"):
        make256()
