"""Test infrastructure only: ctypes bindings for oracle/_ref/libpcrref.so.

That library is the reference CPU renderer compiled from its own sources
(oracle/Makefile, oracle/ref_driver.cpp).  It is one of the two checkers for
the CUDA path (the other is the C restatement in pcr_oracle.c) and the timed
CPU baseline.  Nothing in the product package imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import tempfile
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libpcrref.so")

_lib = None


class RefRenderOpts(C.Structure):
    """Mirror of RefRenderOpts in ref_driver.cpp (Renderer knobs,
    code/Includes/Renderer.h:41-102)."""
    _fields_ = [(n, C.c_int) for n in (
        "width", "height", "depth", "samples", "shadow", "spectral", "mis",
        "russian", "stratified", "aces", "denoise", "aa", "adaptive", "hero")] + [
        ("seed", C.c_uint64)]


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"reference oracle not built: {LIB_PATH}")
        L = C.CDLL(LIB_PATH)
        P, I, F, D = C.c_void_p, C.c_int, C.c_float, C.c_double
        fp = C.POINTER(C.c_float)
        ip = C.POINTER(C.c_int)
        dp = C.POINTER(C.c_double)
        L.ref_scene_load.restype = P
        L.ref_scene_load.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, I]
        L.ref_scene_free.argtypes = [P]
        L.ref_scene_sizes.argtypes = [P, ip]
        L.ref_scene_name.argtypes = [P, C.c_char_p, I, C.c_char_p, I]
        L.ref_scene_camera.argtypes = [P, fp]
        L.ref_scene_materials.argtypes = [P, fp]
        L.ref_scene_planes.argtypes = [P, fp]
        L.ref_scene_planes.restype = I
        L.ref_scene_spheres.argtypes = [P, fp]
        L.ref_scene_triangles.argtypes = [P, fp]
        L.ref_scene_bvh.argtypes = [P, fp, ip]
        L.ref_scene_lights.argtypes = [P, fp]
        L.ref_scene_light_tris.argtypes = [P, I, fp]
        L.ref_material_albedo_at.argtypes = [P, I, F]
        L.ref_material_albedo_at.restype = F
        L.ref_material_emissive_at.argtypes = [P, I, F]
        L.ref_material_emissive_at.restype = F
        L.ref_set_lut.argtypes = [I, C.c_char_p, C.c_char_p, I]
        L.ref_set_lut.restype = I
        L.ref_lut_data.argtypes = [fp]
        L.ref_lut_data.restype = I
        L.ref_lut_save.argtypes = [C.c_char_p]
        L.ref_lut_save.restype = I
        L.ref_render_png.argtypes = [P, C.POINTER(RefRenderOpts), C.c_char_p, C.c_char_p, I]
        L.ref_render_png.restype = I
        L.ref_render_hdr.argtypes = [P, C.POINTER(RefRenderOpts), I, I, I, I, I, dp]
        L.ref_render_hdr.restype = D
        L.ref_render_hdr_rows.argtypes = [P, C.POINTER(RefRenderOpts), I, I, ip, I, dp]
        L.ref_render_hdr_rows.restype = D
        L.ref_scene_intersect.argtypes = [P, fp, I, ip, fp]
        L.ref_bvh_build.argtypes = [fp, I, fp, ip, ip]
        L.ref_bvh_build.restype = I
        L.ref_bvh_intersect.argtypes = [fp, I, fp, C.c_long, ip, fp, I]
        L.ref_bvh_intersect.restype = D
        L.ref_ybar_integral.restype = F
        L.ref_eval_sigmoid_fit.argtypes = [fp, fp, I, fp]
        L.ref_eval_spectrum.argtypes = [fp, fp, I, fp]
        L.ref_eval_cmf.argtypes = [fp, I, fp]
        L.ref_single_lambda_xyz.argtypes = [fp, fp, I, fp]
        L.ref_xyz_to_srgb.argtypes = [fp, I, fp]
        L.ref_srgb_to_xyz.argtypes = [fp, I, fp]
        L.ref_spectrum_to_xyz.argtypes = [fp, fp]
        L.ref_tonemap.argtypes = [fp, I, I, fp]
        L.ref_fit_sigmoid.argtypes = [fp, I, fp]
        L.ref_schlick.argtypes = [F, F, F]
        L.ref_schlick.restype = F
        L.ref_cauchy.argtypes = [F, F, F]
        L.ref_cauchy.restype = F
        L.ref_dielectric.argtypes = [fp, I, F, F, fp]
        _lib = L
    return _lib


def _f(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


@dataclass
class RefScene:
    """A scene loaded by the reference loader, with its flat exports."""
    handle: int
    name: str
    version: str
    camera: np.ndarray
    materials: np.ndarray      # (M, 142)
    planes: np.ndarray         # (P, 14) light planes first
    spheres: np.ndarray        # (S, 5)
    triangles: np.ndarray      # (T, 23) BVH-leaf order
    bvh_boxes: np.ndarray      # (N, 6)
    bvh_ints: np.ndarray       # (N, 3)
    lights: np.ndarray         # (L, 16)

    def __del__(self):
        try:
            if self.handle and _lib is not None:
                _lib.ref_scene_free(self.handle)
        except Exception:
            pass


def load_scene(json_path: str, data_root: str) -> RefScene:
    L = lib()
    err = C.create_string_buffer(1024)
    h = L.ref_scene_load(json_path.encode(), data_root.encode(), err, 1024)
    if not h:
        raise RuntimeError(err.value.decode())
    sz = np.zeros(6, np.int32)
    L.ref_scene_sizes(h, _ip(sz))
    nm, nv = C.create_string_buffer(256), C.create_string_buffer(256)
    L.ref_scene_name(h, nm, 256, nv, 256)
    cam = np.zeros(4, np.float32)
    L.ref_scene_camera(h, _fp(cam))
    mats = np.zeros((sz[0], 142), np.float32)
    L.ref_scene_materials(h, _fp(mats))
    npl = L.ref_scene_planes(h, None)
    planes = np.zeros((npl, 14), np.float32)
    if npl:
        L.ref_scene_planes(h, _fp(planes))
    sph = np.zeros((sz[1], 5), np.float32)
    L.ref_scene_spheres(h, _fp(sph))
    tris = np.zeros((sz[3], 23), np.float32)
    L.ref_scene_triangles(h, _fp(tris))
    boxes = np.zeros((sz[4], 6), np.float32)
    ints = np.zeros((sz[4], 3), np.int32)
    L.ref_scene_bvh(h, _fp(boxes), _ip(ints))
    lights = np.zeros((sz[5], 16), np.float32)
    L.ref_scene_lights(h, _fp(lights))
    return RefScene(h, nm.value.decode(), nv.value.decode(), cam, mats, planes, sph,
                    tris, boxes, ints, lights)


def opts(width, height=None, depth=2, samples=4, shadow=2, spectral=False, mis=False,
         russian=False, stratified=False, aces=False, denoise=False, aa=1,
         adaptive=False, hero=4, seed=12345) -> RefRenderOpts:
    return RefRenderOpts(width, height or width, depth, samples, shadow, int(spectral),
                         int(mis), int(russian), int(stratified), int(aces), int(denoise),
                         aa, int(adaptive), hero, seed)


def set_lut(mode: int, path: str = "") -> None:
    err = C.create_string_buffer(512)
    if lib().ref_set_lut(mode, path.encode(), err, 512):
        raise RuntimeError(err.value.decode())


def render_png_rgb8(scene: RefScene, o: RefRenderOpts) -> np.ndarray:
    """Run Renderer::render (the CLI path) and return the PNG's RGB8 pixels."""
    from PIL import Image
    with tempfile.TemporaryDirectory() as d:
        out = C.create_string_buffer(4096)
        if lib().ref_render_png(scene.handle, C.byref(o), d.encode(), out, 4096):
            raise RuntimeError("reference render failed")
        return np.asarray(Image.open(out.value.decode()).convert("RGB"))


def render_hdr(scene: RefScene, o: RefRenderOpts, mode: int = 0, spp: int = 1,
               threads: int = 1, rows=(0, 0)):
    """HDR linear-sRGB image (H, W, 3) float64 and the loop's wall seconds.
    mode 0: the CPU renderer's branched estimator; mode 1: spp paths per pixel."""
    r0, r1 = rows
    r1 = r1 or o.height
    out = np.zeros((r1 - r0, o.width, 3), np.float64)
    secs = lib().ref_render_hdr(scene.handle, C.byref(o), mode, spp, threads, r0, r1, _dp(out))
    return out, secs


def spread_rows(height: int, n: int) -> np.ndarray:
    """n rows spread evenly over an image of `height` rows (the centre row of
    each of n equal bands), so a row sample sees the image's average
    content rather than, say, the ceiling and the light at the top."""
    n = max(1, min(n, height))
    return ((np.arange(n) + 0.5) * height / n).astype(np.int32)


def render_hdr_rows(scene: RefScene, o: RefRenderOpts, rows, spp: int = 1, threads: int = 0):
    """Paths mode (spp paths per pixel centre) over the given rows only:
    (len(rows), W, 3) float64 linear sRGB and the loop's wall seconds."""
    r = np.ascontiguousarray(rows, np.int32)
    out = np.zeros((r.size, o.width, 3), np.float64)
    secs = lib().ref_render_hdr_rows(scene.handle, C.byref(o), spp, threads, _ip(r), r.size, _dp(out))
    return out, secs


def scene_intersect(scene: RefScene, rays: np.ndarray):
    rays = _f(rays)
    n = rays.shape[0]
    mat = np.zeros(n, np.int32)
    hn = np.zeros((n, 6), np.float32)
    lib().ref_scene_intersect(scene.handle, _fp(rays), n, _ip(mat), _fp(hn))
    return mat, hn


def bvh_build(tris9: np.ndarray):
    t = _f(tris9)
    n = t.shape[0]
    boxes = np.zeros((max(2 * n, 1), 6), np.float32)
    ints = np.zeros((max(2 * n, 1), 3), np.int32)
    perm = np.zeros(n, np.int32)
    nn = lib().ref_bvh_build(_fp(t), n, _fp(boxes), _ip(ints), _ip(perm))
    return boxes[:nn], ints[:nn], perm


def bvh_intersect(tris9: np.ndarray, rays: np.ndarray, threads: int = 0):
    t = _f(tris9)
    r = _f(rays)
    n = r.shape[0]
    hid = np.zeros(n, np.int32)
    ht = np.zeros(n, np.float32)
    secs = lib().ref_bvh_intersect(_fp(t), t.shape[0], _fp(r), n, _ip(hid), _fp(ht), threads)
    return hid, ht, secs
