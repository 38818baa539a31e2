"""Test infrastructure only: Python side of the CPU restatement oracle.

`pcr_oracle.c` (built into oracle/libpcroracle.so by oracle/Makefile) holds
the arithmetic; this module loads scenes the way the reference loader does
(code/Scenes/SceneLoader.cpp:475-516) and hands flat arrays to the C code.
It is the checker for the CUDA path: only tests/, __graft_entry__.smoke()
and bench.py's CPU-baseline leg may import it.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpcroracle.so")
SPEC_N = 61


class OMaterial(C.Structure):
    _fields_ = [("albedo", C.c_float * 3), ("emissive", C.c_float * 3),
                ("metallic", C.c_int), ("transparent", C.c_int), ("useTabA", C.c_int),
                ("useTabE", C.c_int), ("ior", C.c_float), ("cauchyB", C.c_float),
                ("afit", C.c_float * 4), ("efit", C.c_float * 4),
                ("tabA", C.c_float * SPEC_N), ("tabE", C.c_float * SPEC_N)]


class OPlane(C.Structure):
    _fields_ = [("origin", C.c_float * 3), ("u", C.c_float * 3), ("v", C.c_float * 3),
                ("N", C.c_float * 3), ("area", C.c_float), ("matIdx", C.c_int)]


class OSphere(C.Structure):
    _fields_ = [("center", C.c_float * 3), ("radius", C.c_float), ("matIdx", C.c_int)]


class OTriangle(C.Structure):
    _fields_ = [("v0", C.c_float * 3), ("v1", C.c_float * 3), ("v2", C.c_float * 3),
                ("n0", C.c_float * 3), ("n1", C.c_float * 3), ("n2", C.c_float * 3),
                ("flatN", C.c_float * 3), ("smooth", C.c_int), ("matIdx", C.c_int)]


class ONode(C.Structure):
    _fields_ = [("bmin", C.c_float * 3), ("bmax", C.c_float * 3), ("leftOrFirst", C.c_int),
                ("rightChild", C.c_int), ("count", C.c_int)]


class OLight(C.Structure):
    _fields_ = [("kind", C.c_int), ("totalArea", C.c_float), ("plane", OPlane),
                ("triOffset", C.c_int), ("triCount", C.c_int)]


class OScene(C.Structure):
    _fields_ = [("camPos", C.c_float * 3), ("fov", C.c_float),
                ("nMat", C.c_int), ("mats", C.POINTER(OMaterial)),
                ("nSph", C.c_int), ("sph", C.POINTER(OSphere)),
                ("nPlanes", C.c_int), ("planes", C.POINTER(OPlane)),
                ("nTri", C.c_int), ("tris", C.POINTER(OTriangle)),
                ("nNodes", C.c_int), ("nodes", C.POINTER(ONode)),
                ("nLights", C.c_int), ("lights", C.POINTER(OLight)),
                ("lightTris", C.POINTER(OTriangle)), ("lightCum", C.POINTER(C.c_float))]


class OOpts(C.Structure):
    _fields_ = [(n, C.c_int) for n in (
        "width", "height", "depth", "samples", "shadow", "spectral", "mis", "russian",
        "stratified", "aces", "denoise", "aa", "adaptive", "hero")] + [("seed", C.c_uint64)]


_lib = None


def build() -> None:
    """Compile the restatement (gcc, seconds)."""
    subprocess.run(["make", "-s", "-C", HERE, "port"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        fp, ip, dp = C.POINTER(C.c_float), C.POINTER(C.c_int), C.POINTER(C.c_double)
        u8p, lp = C.POINTER(C.c_ubyte), C.POINTER(C.c_long)
        I, F = C.c_int, C.c_float
        sig = {
            "oracle_fit_sigmoid": ([fp, fp, fp], None),
            "oracle_lut_lookup": ([fp, fp, fp], None),
            "oracle_lut_build": ([fp], None),
            "oracle_populate_material": ([C.POINTER(OMaterial), fp], None),
            "oracle_spectrum_rgb": ([fp, fp], None),
            "oracle_make_plane": ([fp, fp, fp, I, C.POINTER(OPlane)], None),
            "oracle_make_triangle": ([fp, fp, fp, fp, fp, fp, I, C.POINTER(OTriangle)], None),
            "oracle_triangle_cum_area": ([C.POINTER(OTriangle), I, fp], F),
            "oracle_mesh_transform": ([fp, I, fp, fp, fp, I], None),
            "oracle_bvh_build": ([C.POINTER(OTriangle), I, C.POINTER(ONode)], I),
            "oracle_bvh_query": ([C.POINTER(ONode), I, C.POINTER(OTriangle), fp, C.c_long, ip, fp, lp], None),
            "oracle_scene_intersect": ([C.POINTER(OScene), fp, I, ip, fp], None),
            "oracle_render": ([C.POINTER(OScene), C.POINTER(OOpts), I, fp, u8p], None),
            "oracle_render_paths": ([C.POINTER(OScene), C.POINTER(OOpts), I, I, dp], None),
            "oracle_bilateral": ([u8p, I, I], None),
            "oracle_ybar_integral": ([], F),
            "oracle_eval_fit": ([fp, fp, I, fp], None),
            "oracle_eval_spectrum": ([fp, fp, I, fp], None),
            "oracle_eval_cmf": ([fp, I, fp], None),
            "oracle_single_lambda_xyz": ([fp, fp, I, fp], None),
            "oracle_xyz_to_srgb": ([fp, I, fp], None),
            "oracle_tonemap": ([fp, I, I, fp, u8p], None),
            "oracle_spectrum_to_xyz": ([fp, fp], None),
            "oracle_schlick": ([F, F, F], F),
            "oracle_cauchy": ([F, F, F], F),
            "oracle_dielectric": ([fp, I, F, F, fp], None),
            "oracle_hemisphere_dir": ([fp, F, F, fp], None),
            "oracle_count_begin": ([], None),
            "oracle_count_end": ([lp], None),
        }
        for name, (args, res) in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def fptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


# ------------------------------------------------------------------ parsing

def strip_jsonc(text: str) -> str:
    """Drop // and /* */ comments outside strings (nlohmann ignore_comments)."""
    out, i, n = [], 0, len(text)
    in_str = False
    while i < n:
        ch = text[i]
        if in_str:
            out.append(ch)
            if ch == "\\" and i + 1 < n:
                out.append(text[i + 1])
                i += 2
                continue
            if ch == '"':
                in_str = False
            i += 1
            continue
        if ch == '"':
            in_str = True
            out.append(ch)
            i += 1
        elif text.startswith("//", i):
            j = text.find("\n", i)
            i = n if j < 0 else j
        elif text.startswith("/*", i):
            j = text.find("*/", i + 2)
            i = n if j < 0 else j + 2
        else:
            out.append(ch)
            i += 1
    return "".join(out)


_libc = C.CDLL(None)
_libc.strtof.restype = C.c_float
_libc.strtof.argtypes = [C.c_char_p, C.POINTER(C.c_char_p)]


def _strtof(s: str) -> np.float32:
    return np.float32(_libc.strtof(s.encode(), None))


def spd_resample(pairs) -> np.ndarray:
    """SpdLoader interp onto the 61-sample grid (code/SpdLoader.cpp:20-35, 77-78)."""
    lam = [p[0] for p in pairs]
    val = [p[1] for p in pairs]
    out = np.zeros(SPEC_N, np.float32)
    for i in range(SPEC_N):
        l = np.float32(400.0) + np.float32(i) * np.float32(5.0)
        if l <= lam[0]:
            out[i] = val[0]
        elif l >= lam[-1]:
            out[i] = val[-1]
        else:
            hi = next(k for k in range(len(lam)) if lam[k] > l)
            lo = hi - 1
            t = np.float32((l - lam[lo]) / np.float32(lam[hi] - lam[lo]))
            out[i] = np.float32(val[lo] + np.float32(t * np.float32(val[hi] - val[lo])))
    return out


def load_spd(path: str) -> np.ndarray:
    pairs = []
    with open(path) as fh:
        for line in fh:
            s = line.lstrip(" \t").rstrip("\n")
            if not s or s.startswith("#"):
                continue
            parts = s.split()
            pairs.append((_strtof(parts[0]), _strtof(parts[1])))
    if not pairs:
        raise ValueError(f"no data samples in {path}")
    for a, b in zip(pairs, pairs[1:]):
        if not b[0] > a[0]:
            raise ValueError(f"{path}: wavelengths must be strictly ascending")
    return spd_resample(pairs)


def load_obj(path: str):
    """Positions and triangle faces (position indices) of an OBJ file."""
    verts, normals, faces = [], [], []
    with open(path) as fh:
        for line in fh:
            if line.startswith("v "):
                verts.append([float(x) for x in line.split()[1:4]])
            elif line.startswith("vn "):
                normals.append([float(x) for x in line.split()[1:4]])
            elif line.startswith("f "):
                idx = []
                for tok in line.split()[1:]:
                    parts = tok.split("/")
                    vi = int(parts[0])
                    ni = int(parts[2]) if len(parts) > 2 and parts[2] else 0
                    vi = vi - 1 if vi > 0 else len(verts) + vi
                    ni = (ni - 1 if ni > 0 else len(normals) + ni) if ni else -1
                    idx.append((vi, ni))
                for k in range(1, len(idx) - 1):
                    faces.append((idx[0], idx[k], idx[k + 1]))
    return np.asarray(verts, np.float32), np.asarray(normals, np.float32), faces


class Scene:
    """A scene in the restatement's flat form.  Keeps the ctypes arrays alive."""

    def __init__(self):
        self.name = ""
        self.version = ""
        self.cam = (0.0, 0.0, 0.0)
        self.fov = 65.0
        self.materials = []
        self.spheres = []
        self.walls = []
        self.triangles = []
        self.lights = []          # (kind, plane | tri list)
        self.nodes = None
        self._c = None

    # --- flat views (numpy) used by tests to compare against other loaders
    def material_table(self) -> np.ndarray:
        rows = []
        for m in self.materials:
            rows.append(np.concatenate([
                np.asarray(m.albedo, np.float32), np.asarray(m.emissive, np.float32),
                np.asarray([m.metallic, m.transparent, m.ior, m.cauchyB, m.useTabA, m.useTabE], np.float32),
                np.asarray(m.afit, np.float32), np.asarray(m.efit, np.float32),
                np.asarray(m.tabA, np.float32), np.asarray(m.tabE, np.float32)]))
        return np.asarray(rows, np.float32)

    def plane_table(self) -> np.ndarray:
        return np.asarray([list(p.origin) + list(p.u) + list(p.v) + list(p.N) + [p.area, p.matIdx]
                           for p in self.render_planes()], np.float32).reshape(-1, 14)

    def render_planes(self):
        """Renderer order: light planes first, then walls (Renderer.cpp:123-130)."""
        return [L[1] for L in self.lights if L[0] == 0] + list(self.walls)

    def cstruct(self) -> OScene:
        if self._c is not None:
            return self._c
        S = OScene()
        S.camPos[:] = self.cam
        S.fov = self.fov
        self._mats = (OMaterial * max(1, len(self.materials)))(*self.materials)
        self._sph = (OSphere * max(1, len(self.spheres)))(*self.spheres)
        planes = self.render_planes()
        self._pl = (OPlane * max(1, len(planes)))(*planes)
        self._tr = (OTriangle * max(1, len(self.triangles)))(*self.triangles)
        lt, cum, lights = [], [], []
        for kind, payload in self.lights:
            L = OLight()
            L.kind = kind
            if kind == 0:
                L.plane = payload
                L.totalArea = payload.area
            else:
                arr = (OTriangle * len(payload))(*payload)
                c = np.zeros(len(payload), np.float32)
                L.totalArea = lib().oracle_triangle_cum_area(arr, len(payload), fptr(c))
                L.triOffset = len(lt)
                L.triCount = len(payload)
                lt.extend(payload)
                cum.extend(c.tolist())
            lights.append(L)
        self._lights = (OLight * max(1, len(lights)))(*lights)
        self._lt = (OTriangle * max(1, len(lt)))(*lt)
        self._cum = np.asarray(cum or [0.0], np.float32)
        S.nMat, S.mats = len(self.materials), self._mats
        S.nSph, S.sph = len(self.spheres), self._sph
        S.nPlanes, S.planes = len(planes), self._pl
        S.nTri, S.tris = len(self.triangles), self._tr
        n_nodes = 0 if self.nodes is None else len(self.nodes)
        S.nNodes = n_nodes
        S.nodes = self.nodes if n_nodes else (ONode * 1)()
        S.nLights, S.lights = len(lights), self._lights
        S.lightTris, S.lightCum = self._lt, fptr(self._cum)
        self._c = S
        return S


def _v3(x, what):
    if not isinstance(x, list) or len(x) != 3:
        raise ValueError(f"{what}: expected [x, y, z] array of 3 numbers")
    return (C.c_float * 3)(*[np.float32(v) for v in x])


def load_scene(path: str, data_root: str | None = None, lut: np.ndarray | None = None) -> Scene:
    """Restatement of loadSceneFromFile (code/Scenes/SceneLoader.cpp:89-516).
    data_root holds spd/ (code/SpdLoader.cpp:93-98)."""
    L = lib()
    with open(path) as fh:
        j = json.loads(strip_jsonc(fh.read()))
    major = int(str(j["schema"]).split(".")[0])
    if major != 1:
        raise ValueError(f"{path}: schema major version {major} is not supported")
    sc = Scene()
    sc.name, sc.version = j["name"], j["version"]
    cam = j.get("camera", {})
    sc.cam = tuple(np.float32(v) for v in cam.get("position", [0, 0, 0]))
    sc.fov = np.float32(cam.get("fov", 65.0))
    name_to_idx = {}
    spd_dir = os.path.join(data_root or os.path.dirname(path), "spd")
    # nlohmann::json objects iterate in key order (std::map)
    for name in sorted(j["materials"].keys()):
        m = j["materials"][name]
        mat = OMaterial()
        mat.ior = np.float32(1.5)
        if "albedo" in m:
            mat.albedo = _v3(m["albedo"], "albedo")
        if "emissive" in m:
            mat.emissive = _v3(m["emissive"], "emissive")
        if "albedo_spd" in m:
            tab = load_spd(os.path.join(spd_dir, m["albedo_spd"] + ".spd"))
            mat.tabA[:] = tab.tolist()
            mat.useTabA = 1
            if "albedo" not in m:
                rgb = np.zeros(3, np.float32)
                L.oracle_spectrum_rgb(fptr(tab), fptr(rgb))
                mat.albedo[:] = rgb.tolist()
        if "emissive_spd" in m:
            tab = load_spd(os.path.join(spd_dir, m["emissive_spd"] + ".spd"))
            if "emissive_scale" in m:
                tab = (tab * np.float32(m["emissive_scale"])).astype(np.float32)
            mat.tabE[:] = tab.tolist()
            mat.useTabE = 1
            if "emissive" not in m:
                rgb = np.zeros(3, np.float32)
                L.oracle_spectrum_rgb(fptr(tab), fptr(rgb))
                mat.emissive[:] = rgb.tolist()
        mat.metallic = int(bool(m.get("metallic", False)))
        mat.transparent = int(bool(m.get("transparent", False)))
        if "ior" in m:
            mat.ior = np.float32(m["ior"])
        if "cauchyB" in m:
            mat.cauchyB = np.float32(m["cauchyB"])
        if mat.metallic and mat.transparent:
            raise ValueError(f"{path}: material {name} cannot be both metallic and transparent")
        name_to_idx[name] = len(sc.materials)
        sc.materials.append(mat)
    scene_dir = os.path.dirname(os.path.abspath(path))
    for p in j["primitives"]:
        t = p["type"]
        light = bool(p.get("light", False))
        if t == "sphere":
            s = OSphere()
            s.center = _v3(p["center"], "center")
            s.radius = np.float32(p["radius"])
            s.matIdx = name_to_idx[p["material"]]
            sc.spheres.append(s)
        elif t == "plane":
            pl = OPlane()
            L.oracle_make_plane(_v3(p["origin"], "o"), _v3(p["u"], "u"), _v3(p["v"], "v"),
                                name_to_idx[p["material"]], C.byref(pl))
            if light:
                sc.lights.append((0, pl))
            else:
                sc.walls.append(pl)
        elif t == "triangle":
            tr = OTriangle()
            ns = [p.get(k) for k in ("n0", "n1", "n2")]
            nargs = [_v3(x, "n") for x in ns] if all(x is not None for x in ns) else [None] * 3
            L.oracle_make_triangle(_v3(p["v0"], "v0"), _v3(p["v1"], "v1"), _v3(p["v2"], "v2"),
                                   *nargs, name_to_idx[p["material"]], C.byref(tr))
            if light:
                sc.lights.append((1, [tr]))
            sc.triangles.append(tr)
        elif t == "mesh":
            tris = load_mesh(os.path.join(scene_dir, p["file"]), p, name_to_idx, sc)
            if light:
                sc.lights.append((1, list(tris)))
            sc.triangles.extend(tris)
        else:
            raise ValueError(f"{path}: unknown primitive type {t}")
    if not sc.lights:
        raise ValueError(f"{path}: at least one primitive must have \"light\": true; found none")
    finish_scene(sc, lut)
    return sc


def load_mesh(obj_path, p, name_to_idx, sc):
    """MeshLoader::loadMesh restated for position-only / v//vn OBJ files
    (code/Scenes/MeshLoader.cpp:139-298)."""
    L = lib()
    verts, normals, faces = load_obj(obj_path)
    pos = np.asarray(p.get("position", [0, 0, 0]), np.float32)
    rot = np.asarray(p.get("rotation", [0, 0, 0]), np.float32)
    sc_ = p.get("scale", [1, 1, 1])
    scale = np.asarray([sc_] * 3 if not isinstance(sc_, list) else sc_, np.float32)
    vt = f32(verts.copy())
    L.oracle_mesh_transform(fptr(vt), len(vt), fptr(pos), fptr(rot), fptr(scale), 0)
    nt = f32(normals.copy()) if len(normals) else None
    if nt is not None:
        L.oracle_mesh_transform(fptr(nt), len(nt), fptr(pos), fptr(rot), fptr(scale), 1)
    if "material" in p:
        mat = name_to_idx[p["material"]]
    else:
        key = "__pcr_mesh_fallback_grey"
        if key not in name_to_idx:
            m = OMaterial()
            m.albedo[:] = [0.7, 0.7, 0.7]
            m.ior = 1.5
            name_to_idx[key] = len(sc.materials)
            sc.materials.append(m)
        mat = name_to_idx[key]
    smooth_ok = bool(p.get("smooth", True))
    out = []
    for (a, b, c) in faces:
        tr = OTriangle()
        have_n = a[1] >= 0 and b[1] >= 0 and c[1] >= 0 and nt is not None and smooth_ok
        va, vb, vc = (vt[a[0]], vt[b[0]], vt[c[0]])
        args = [fptr(f32(va)), fptr(f32(vb)), fptr(f32(vc))]
        if have_n:
            args += [fptr(f32(nt[a[1]])), fptr(f32(nt[b[1]])), fptr(f32(nt[c[1]]))]
        else:
            args += [None, None, None]
        L.oracle_make_triangle(*args, mat, C.byref(tr))
        out.append(tr)
    return out


def triangles_from_array(tris9: np.ndarray):
    """Flat (N, 9) vertex array -> OTriangle list with matIdx = input index."""
    L = lib()
    t = f32(tris9)
    out = []
    for i in range(t.shape[0]):
        tr = OTriangle()
        L.oracle_make_triangle(fptr(t[i, 0:3]), fptr(t[i, 3:6]), fptr(t[i, 6:9]), None, None, None,
                               i, C.byref(tr))
        out.append(tr)
    return out


def finish_scene(sc: Scene, lut=None) -> None:
    """BVH build (permutes triangles) then populateSpectra (SceneLoader.cpp:508-513)."""
    L = lib()
    n = len(sc.triangles)
    if n:
        arr = (OTriangle * n)(*sc.triangles)
        nodes = (ONode * (2 * n))()
        cnt = L.oracle_bvh_build(arr, n, nodes)
        sc.triangles = list(arr)
        sc.nodes = (ONode * cnt).from_buffer_copy(nodes, 0)
    for m in sc.materials:
        L.oracle_populate_material(C.byref(m), fptr(f32(lut)) if lut is not None else None)


def bvh_build(tris9: np.ndarray):
    """Restated Bvh::build over flat triangles: (boxes6, ints3, perm)."""
    L = lib()
    trs = triangles_from_array(tris9)
    n = len(trs)
    arr = (OTriangle * n)(*trs)
    nodes = (ONode * (2 * n))()
    cnt = L.oracle_bvh_build(arr, n, nodes)
    boxes = np.zeros((cnt, 6), np.float32)
    ints = np.zeros((cnt, 3), np.int32)
    for i in range(cnt):
        boxes[i, :3] = nodes[i].bmin[:]
        boxes[i, 3:] = nodes[i].bmax[:]
        ints[i] = (nodes[i].leftOrFirst, nodes[i].rightChild, nodes[i].count)
    perm = np.asarray([arr[i].matIdx for i in range(n)], np.int32)
    return boxes, ints, perm, arr, (ONode * cnt).from_buffer_copy(nodes, 0)


def bvh_query(nodes, tri_arr, rays: np.ndarray, counts: bool = False):
    """Restated Bvh::intersect per ray; optional [internal nodes, leaf tris] counts."""
    r = f32(rays)
    n = r.shape[0]
    hid = np.zeros(n, np.int32)
    ht = np.zeros(n, np.float32)
    cnt = np.zeros((n, 2), np.int64) if counts else None
    lib().oracle_bvh_query(nodes, len(nodes), tri_arr, fptr(r), n,
                           hid.ctypes.data_as(C.POINTER(C.c_int)), fptr(ht),
                           cnt.ctypes.data_as(C.POINTER(C.c_long)) if counts else None)
    return (hid, ht, cnt) if counts else (hid, ht)


def opts(width, height=None, depth=2, samples=4, shadow=2, spectral=False, mis=False,
         russian=False, stratified=False, aces=False, denoise=False, aa=1, adaptive=False,
         hero=4, seed=12345) -> OOpts:
    return OOpts(width, height or width, depth, samples, shadow, int(spectral), int(mis),
                 int(russian), int(stratified), int(aces), int(denoise), aa, int(adaptive), hero, seed)


def render(sc: Scene, o: OOpts, threads: int = 1):
    """Renderer::render restated: (hdr float32 (H,W,3), rgb8 uint8 (H,W,3))."""
    hdr = np.zeros((o.height, o.width, 3), np.float32)
    rgb = np.zeros((o.height, o.width, 3), np.uint8)
    lib().oracle_render(C.byref(sc.cstruct()), C.byref(o), threads, fptr(hdr),
                        rgb.ctypes.data_as(C.POINTER(C.c_ubyte)))
    return hdr, rgb


def count_render_paths(sc: Scene, o: OOpts, spp: int, threads: int = 1) -> dict:
    """render_paths with the reference traversal's work counted: rays
    (sceneIntersect calls, shadow rays included), plane and sphere tests,
    BVH internal nodes processed and leaf triangles tested."""
    L = lib()
    L.oracle_count_begin()
    try:
        render_paths(sc, o, spp, threads)
    finally:
        c = np.zeros(5, np.int64)
        L.oracle_count_end(c.ctypes.data_as(C.POINTER(C.c_long)))
    return dict(zip(["rays", "plane_tests", "sphere_tests", "bvh_nodes", "bvh_tris"], c.tolist()))


def render_paths(sc: Scene, o: OOpts, spp: int, threads: int = 1) -> np.ndarray:
    """GPU estimator on the CPU: spp paths per pixel centre, FP64 mean, linear sRGB."""
    out = np.zeros((o.height, o.width, 3), np.float64)
    lib().oracle_render_paths(C.byref(sc.cstruct()), C.byref(o), spp, threads,
                              out.ctypes.data_as(C.POINTER(C.c_double)))
    return out


def scene_intersect(sc: Scene, rays: np.ndarray):
    r = f32(rays)
    n = r.shape[0]
    mat = np.zeros(n, np.int32)
    hn = np.zeros((n, 6), np.float32)
    lib().oracle_scene_intersect(C.byref(sc.cstruct()), fptr(r), n,
                                 mat.ctypes.data_as(C.POINTER(C.c_int)), fptr(hn))
    return mat, hn


def tonemap(hdr: np.ndarray, aces: bool = False):
    x = f32(hdr).reshape(-1, 3)
    out = np.zeros_like(x)
    q = np.zeros(x.shape, np.uint8)
    lib().oracle_tonemap(fptr(x), x.shape[0], int(aces), fptr(out), q.ctypes.data_as(C.POINTER(C.c_ubyte)))
    return out.reshape(hdr.shape), q.reshape(hdr.shape)
