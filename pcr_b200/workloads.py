"""Seeded synthetic workloads for the batched and served methods.

* displaced_icosphere(freq, seed): a geodesic icosphere (20*freq^2
  triangles; freq 59 -> 69,620, freq 224 -> 1,003,520) with radial
  displacement from 4-octave value noise of amplitude 0.15 r.
* mesh_scene(...): that mesh inside the Cornell box, written as an OBJ plus a
  scene JSON so the library, the reference CPU renderer and the oracle all
  load the same file.
* batch_requests(...): the uneven batch (scene variant, resolution, depth,
  paths per pixel, shadow rays) drawn by seed.
* request_stream(...): Poisson arrivals for the served method.

The Stanford bunny OBJ is a test fixture of this repository
(tests/golden/models); where a workload draws the cornell-bunny variant and
that file is absent, a displaced icosphere of the bunny's triangle count
stands in for it (same pose and material).
"""
from __future__ import annotations

import hashlib
import json
import math
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
DEFAULT_SCENES = os.path.join(REPO, "tests", "golden", "scenes")
DEFAULT_DATA = os.path.join(REPO, "tests", "golden")
VARIANTS = ["cornell", "cornell-spec", "cornell-glass", "cornell-spheres", "closed-cornell-spec",
            "cornell-large-light", "bright-cornell-glass", "closed-cornell-glass", "cornell-frank",
            "cornell-bunny"]


def _strip_comments(text: str) -> str:
    out, i, n, in_str = [], 0, len(text), False
    while i < n:
        c = text[i]
        if in_str:
            out.append(c)
            if c == "\\" and i + 1 < n:
                out.append(text[i + 1])
                i += 2
                continue
            in_str = c != '"'
            i += 1
        elif c == '"':
            in_str = True
            out.append(c)
            i += 1
        elif text.startswith("//", i):
            j = text.find("\n", i)
            i = n if j < 0 else j
        elif text.startswith("/*", i):
            j = text.find("*/", i + 2)
            i = n if j < 0 else j + 2
        else:
            out.append(c)
            i += 1
    return "".join(out)


def read_scene_json(path: str) -> dict:
    with open(path) as f:
        return json.loads(_strip_comments(f.read()))


# ------------------------------------------------------------------ mesh
def _icosahedron():
    t = (1.0 + 5 ** 0.5) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
                  [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5],
                  [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], np.int64)
    return v, f


def _value_noise(p: np.ndarray, seed: int, octaves: int = 4) -> np.ndarray:
    """Sum of `octaves` octaves of 3D value noise (lattice values hashed from
    the seed, smoothstep trilinear interpolation), normalised to [-1, 1]."""
    def lattice(ix, iy, iz):
        h = (ix * 73856093) ^ (iy * 19349663) ^ (iz * 83492791) ^ (seed * 2654435761)
        h = (h ^ (h >> 13)) * 1274126177
        h = h ^ (h >> 16)
        return ((h & 0xFFFFFF).astype(np.float64) / float(0xFFFFFF)) * 2.0 - 1.0

    total = np.zeros(p.shape[0])
    amp, freq, norm = 1.0, 2.0, 0.0
    for _ in range(octaves):
        q = p * freq
        i0 = np.floor(q).astype(np.int64)
        f = q - i0
        s = f * f * (3 - 2 * f)
        acc = np.zeros(p.shape[0])
        for dx in (0, 1):
            for dy in (0, 1):
                for dz in (0, 1):
                    w = (s[:, 0] if dx else 1 - s[:, 0]) * (s[:, 1] if dy else 1 - s[:, 1]) * \
                        (s[:, 2] if dz else 1 - s[:, 2])
                    acc += w * lattice(i0[:, 0] + dx, i0[:, 1] + dy, i0[:, 2] + dz)
        total += amp * acc
        norm += amp
        amp *= 0.5
        freq *= 2.0
    return total / norm


def displaced_icosphere(freq: int, seed: int, radius: float = 0.8, amplitude: float = 0.15) -> np.ndarray:
    """(20*freq^2, 9) float32 triangle vertices around the origin."""
    v, faces = _icosahedron()
    tris = []
    for a, b, c in faces:
        A, B, Cc = v[a], v[b], v[c]
        ii, jj = np.meshgrid(np.arange(freq + 1), np.arange(freq + 1), indexing="ij")
        mask = ii + jj <= freq
        ii, jj = ii[mask], jj[mask]
        # canonical point formula: shared edge points come out bit-identical
        pts = (A[None] * ((freq - ii - jj) / freq)[:, None] + B[None] * (ii / freq)[:, None]) + \
            Cc[None] * (jj / freq)[:, None]
        index = {(int(i), int(j)): k for k, (i, j) in enumerate(zip(ii, jj))}
        for i in range(freq):
            for j in range(freq - i):
                p0, p1, p2 = index[(i, j)], index[(i + 1, j)], index[(i, j + 1)]
                tris.append((pts[p0], pts[p1], pts[p2]))
                if i + j + 1 < freq:
                    p3 = index[(i + 1, j + 1)]
                    tris.append((pts[p1], pts[p3], pts[p2]))
    T = np.asarray(tris, np.float64).reshape(-1, 3)
    T /= np.linalg.norm(T, axis=1, keepdims=True)
    r = radius * (1.0 + amplitude * _value_noise(T, seed))
    return (T * r[:, None]).reshape(-1, 9).astype(np.float32)


def write_obj(path: str, tris: np.ndarray) -> None:
    n = tris.shape[0]
    with open(path, "w") as f:
        f.write(f"# displaced icosphere, {n} triangles\n")
        v = tris.reshape(-1, 3)
        f.write("".join("v %.9g %.9g %.9g\n" % tuple(p) for p in v))
        idx = np.arange(1, 3 * n + 1).reshape(n, 3)
        f.write("".join("f %d %d %d\n" % tuple(t) for t in idx))


def cache_dir() -> str:
    d = os.environ.get("PCR_WORKLOAD_CACHE", "/tmp/pcr_workloads")
    os.makedirs(d, exist_ok=True)
    return d


def mesh_scene(freq: int = 59, seed: int = 1, glass: bool = False, scenes_dir: str = DEFAULT_SCENES,
               position=(0.13, -1.05, -4.5), base: str = "cornell", name: str | None = None) -> str:
    """Writes (once) <cache>/<key>/scene.json + mesh.obj and returns the JSON path."""
    key = hashlib.sha1(f"{freq}-{seed}-{glass}-{position}-{base}-{name}".encode()).hexdigest()[:12]
    d = os.path.join(cache_dir(), key)
    js = os.path.join(d, "scene.json")
    if os.path.exists(js):
        return js
    os.makedirs(d, exist_ok=True)
    write_obj(os.path.join(d, "mesh.obj"), displaced_icosphere(freq, seed))
    sc = read_scene_json(os.path.join(scenes_dir, base + ".json"))
    sc["name"] = name or f"cornell-ico{freq}-{'glass' if glass else 'diffuse'}"
    sc["version"] = "1.0.0"
    sc["materials"]["mesh"] = ({"albedo": [0.95, 0.95, 0.95], "transparent": True, "ior": 1.5, "cauchyB": 0.013}
                               if glass else {"albedo": [0.85, 0.72, 0.55]})
    # keep only the walls and the light of the base box
    sc["primitives"] = [p for p in sc["primitives"] if p.get("type") == "plane" and
                        (p.get("light") or not str(p.get("name", "")).startswith(("tall", "short")))]
    sc["primitives"].insert(len(sc["primitives"]) - 1,
                            {"type": "mesh", "file": "mesh.obj", "position": list(position), "material": "mesh"})
    tmp = js + ".tmp"
    with open(tmp, "w") as f:
        json.dump(sc, f, indent=1)
    os.replace(tmp, js)
    return js


def bunny_stand_in(scenes_dir: str = DEFAULT_SCENES) -> str:
    """cornell-bunny with a displaced icosphere of the bunny's size (69,451
    triangles -> freq 59) at the bunny's pose and material."""
    key = "bunny-standin"
    d = os.path.join(cache_dir(), key)
    js = os.path.join(d, "scene.json")
    if os.path.exists(js):
        return js
    os.makedirs(d, exist_ok=True)
    write_obj(os.path.join(d, "mesh.obj"), displaced_icosphere(59, 2))
    sc = read_scene_json(os.path.join(scenes_dir, "cornell-bunny.json"))
    for p in sc["primitives"]:
        if p.get("type") == "mesh":
            p.update({"file": "mesh.obj", "scale": 1, "rotation": [0, 0, 0], "position": [0.13, -1.05, -4.5]})
    tmp = js + ".tmp"
    with open(tmp, "w") as f:
        json.dump(sc, f, indent=1)
    os.replace(tmp, js)
    return js


def scene_path(variant: str, scenes_dir: str = DEFAULT_SCENES, bunny_obj: str | None = None) -> str:
    if variant == "cornell-bunny":
        obj = bunny_obj or os.path.join(os.path.dirname(scenes_dir), "models", "stanford-bunny.obj")
        if os.path.exists(os.path.join(scenes_dir, "cornell-bunny.json")) and os.path.exists(obj):
            return os.path.join(scenes_dir, "cornell-bunny.json")
        return bunny_stand_in(scenes_dir)
    return os.path.join(scenes_dir, variant + ".json")


def _log_uniform_int(rng, lo, hi):
    return int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))


def batch_requests(n: int = 64, seed: int = 2026, res=(128, 1024), depth=(2, 8), spp=(1, 64), shadow=(1, 8),
                   variants=VARIANTS):
    """The uneven batch: list of dicts (variant, width, height, depth, samples, shadow, seed)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        side = _log_uniform_int(rng, *res)
        out.append({"variant": variants[int(rng.integers(len(variants)))], "width": side, "height": side,
                    "depth": int(rng.integers(depth[0], depth[1] + 1)), "samples": _log_uniform_int(rng, *spp),
                    "shadow": int(rng.integers(shadow[0], shadow[1] + 1)), "seed": int(rng.integers(1, 2 ** 31))})
    return out


def request_stream(n: int, rate: float, seed: int = 7, res=(64, 1024), mesh_fraction: float = 0.2,
                   heavy_fraction: float = 0.0, heavy=None):
    """Poisson arrivals at `rate` req/s: list of dicts with an `arrival` time (s)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        if heavy_fraction and rng.uniform() < heavy_fraction:
            r = dict(heavy)
        else:
            side = _log_uniform_int(rng, *res)
            variant = "mesh" if rng.uniform() < mesh_fraction else VARIANTS[int(rng.integers(len(VARIANTS)))]
            r = {"variant": variant, "width": side, "height": side, "depth": int(rng.integers(2, 9)),
                 "samples": _log_uniform_int(rng, 1, 64), "shadow": int(rng.integers(1, 9))}
        r["seed"] = int(rng.integers(1, 2 ** 31))
        r["arrival"] = t
        out.append(r)
    return out
