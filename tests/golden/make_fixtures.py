"""Regenerates the committed test fixtures from the reference project.

Run in a container that has the reference tree (default /root/reference):

    python tests/golden/make_fixtures.py [REFERENCE_ROOT]

It copies, unmodified:
  * Scenes/*.json          -> tests/golden/scenes/   (workload definitions)
  * spd/cornell/*.spd      -> tests/golden/spd/cornell/
  * tests/render/golden/*  -> tests/golden/render/   (the 17 golden PNGs)
and writes tests/golden/bvh_vectors.npz: seeded triangle soups with the
reference's own Bvh::build node arrays and Bvh::intersect answers (via the
compiled reference, oracle/_ref/libpcrref.so).  The GPU box has no reference
tree, so these files are what the parity tests read there.
"""
import os
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)


def soup(seed: int, n: int) -> np.ndarray:
    """n small random triangles in a 2x2x2 cube centred at z = -5."""
    rng = np.random.default_rng(seed)
    a = rng.uniform(-1, 1, (n, 3)).astype(np.float32)
    a[:, 2] -= 5
    b = a + 0.05 * rng.uniform(-1, 1, (n, 3)).astype(np.float32)
    c = a + 0.05 * rng.uniform(-1, 1, (n, 3)).astype(np.float32)
    return np.concatenate([a, b, c], 1).astype(np.float32)


def soup_rays(seed: int, n: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    o = np.zeros((n, 3), np.float32)
    o[:, :2] = rng.uniform(-1, 1, (n, 2))
    d = np.stack([rng.uniform(-1, 1, n) * 0.2, rng.uniform(-1, 1, n) * 0.2, -np.ones(n)], 1)
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    return np.concatenate([o, d], 1).astype(np.float32)


def main(ref_root: str) -> None:
    for sub, pat, dst in (("Scenes", ".json", "scenes"), ("spd/cornell", ".spd", "spd/cornell"),
                          ("tests/render/golden", ".png", "render")):
        src = os.path.join(ref_root, sub)
        out = os.path.join(HERE, dst)
        os.makedirs(out, exist_ok=True)
        for f in sorted(os.listdir(src)):
            if f.endswith(pat):
                shutil.copyfile(os.path.join(src, f), os.path.join(out, f))
    from oracle import ref
    if not ref.available():
        raise SystemExit("build oracle/_ref first: make -C oracle ref")
    arrays = {}
    for name, seed, n in (("soup200", 0xC0FFEE, 200), ("soup5k", 7, 5000)):
        tris = soup(seed, n)
        boxes, ints, perm = ref.bvh_build(tris)
        rays = soup_rays(seed + 1, 4096)
        hid, ht, _ = ref.bvh_intersect(tris, rays, threads=1)
        arrays.update({f"{name}_tris": tris, f"{name}_boxes": boxes, f"{name}_ints": ints,
                       f"{name}_perm": perm, f"{name}_rays": rays, f"{name}_hit": hid,
                       f"{name}_t": ht})
    # 100 coplanar triangles (reference tests/unit/bvh.cpp:71-89 shape)
    cop = np.asarray([[i * 0.01, 0, -5, i * 0.01 + 0.005, 0, -5, i * 0.01, 0.01, -5]
                      for i in range(100)], np.float32)
    boxes, ints, perm = ref.bvh_build(cop)
    arrays.update({"coplanar_tris": cop, "coplanar_boxes": boxes, "coplanar_ints": ints,
                   "coplanar_perm": perm})
    np.savez_compressed(os.path.join(HERE, "bvh_vectors.npz"), **arrays)
    print("fixtures written under", HERE)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
