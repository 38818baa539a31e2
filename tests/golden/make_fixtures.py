"""Regenerates the committed test fixtures from the reference project.

Run where the reference tree is present, naming it by argument or by the
PCR_REFERENCE_ROOT environment variable (the reference project's top level,
holding code/, Scenes/, models/):

    python tests/golden/make_fixtures.py [REFERENCE_ROOT]

It copies, unmodified:
  * Scenes/*.json          -> tests/golden/scenes/   (workload definitions)
  * spd/cornell/*.spd      -> tests/golden/spd/cornell/
  * models/*.obj           -> tests/golden/models/   (the Stanford bunny that
                              cornell-bunny.json loads as ../models/...)
  * luts/*.lut             -> tests/golden/luts/     (the shipped PLUT table)
  * tests/render/golden/*  -> tests/golden/render/   (the 17 golden PNGs)
writes an emissive-mesh scene of its own (scenes/cornell-mesh-light.json
with models/ico-light.obj: the Cornell box lit by its ceiling quad and by a
180-triangle icosphere whose mesh primitive carries "light": true, the
reference loader's TriangleSet light, code/Scenes/SceneLoader.cpp:449-460),
and writes tests/golden/bvh_vectors.npz: seeded triangle soups with the
reference's own Bvh::build node arrays and Bvh::intersect answers (via the
compiled reference, oracle/_ref/libpcrref.so).  The GPU box has no reference
tree, so these files are what the parity tests read there.
"""
import json
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


def mesh_light_scene() -> None:
    """cornell.json plus an emissive icosphere (frequency 3, 180 triangles,
    radius 0.3, no displacement, outward winding so every triangle's flat
    normal faces away from its centre) hanging below the ceiling near the
    left wall.  Two lights: the ceiling quad (a plane light) and the mesh (a
    triangle-set light), so light picking, the cumulative-area triangle
    pick and emissive triangles in the BVH all run."""
    from pcr_b200 import workloads
    tris = workloads.displaced_icosphere(3, 0, radius=0.3, amplitude=0.0)
    os.makedirs(os.path.join(HERE, "models"), exist_ok=True)
    workloads.write_obj(os.path.join(HERE, "models", "ico-light.obj"), tris)
    sc = workloads.read_scene_json(os.path.join(HERE, "scenes", "cornell.json"))
    sc["name"] = "cornell-mesh-light"
    sc["version"] = "1.0.0"
    sc["materials"]["coollight"] = {"emissive": [9.0, 11.0, 16.0]}
    light = [p for p in sc["primitives"] if p.get("light")]
    rest = [p for p in sc["primitives"] if not p.get("light")]
    sc["primitives"] = rest + [{"type": "mesh", "file": "../models/ico-light.obj", "position": [-1.1, 1.2, -3.2],
                                "material": "coollight", "light": True}] + light
    with open(os.path.join(HERE, "scenes", "cornell-mesh-light.json"), "w") as f:
        json.dump(sc, f, indent=1)
        f.write("\n")


def main(ref_root: str) -> None:
    for sub, pat, dst in (("Scenes", ".json", "scenes"), ("spd/cornell", ".spd", "spd/cornell"),
                          ("models", ".obj", "models"), ("luts", ".lut", "luts"),
                          ("tests/render/golden", ".png", "render")):
        src = os.path.join(ref_root, sub)
        out = os.path.join(HERE, dst)
        os.makedirs(out, exist_ok=True)
        for f in sorted(os.listdir(src)):
            if f.endswith(pat):
                shutil.copyfile(os.path.join(src, f), os.path.join(out, f))
    from oracle import ref
    if not ref.available():
        raise SystemExit("build oracle/_ref first: make -C oracle ref REF=<reference>/code")
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
    mesh_light_scene()
    print("fixtures written under", HERE)


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PCR_REFERENCE_ROOT", "")
    if not root:
        raise SystemExit("name the reference tree: make_fixtures.py REFERENCE_ROOT (or set PCR_REFERENCE_ROOT)")
    main(root)
