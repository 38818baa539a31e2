"""ctypes binding of the C ABI in include/pcr_cuda.h (pcr_b200/lib/libpcr_b200.so).

The library is the product: every call here goes to CUDA kernels for
sm_100a.  There is no CPU fallback; importing works without a GPU, but
creating a Context on a machine without one raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libpcr_b200.so")
SPEC_N = 61

STATUS = {0: "PCR_OK", 1: "PCR_ERR_INVALID", 2: "PCR_ERR_CUDA", 3: "PCR_ERR_NO_MEMORY",
          4: "PCR_ERR_NOT_FOUND", 5: "PCR_ERR_SCENE", 6: "PCR_ERR_TIMEOUT", 7: "PCR_ERR_CANCELLED",
          8: "PCR_ERR_DEVICE_STATUS"}

# Every symbol include/pcr_cuda.h declares (checked by the CPU tests).
EXPORTS = [
    "pcr_last_error", "pcr_version", "pcr_ctx_create", "pcr_ctx_destroy", "pcr_ctx_set_device", "pcr_ctx_stream",
    "pcr_scene_upload", "pcr_scene_load_json", "pcr_host_scene_load", "pcr_host_scene_free",
    "pcr_fit_sigmoid", "pcr_lut_build", "pcr_scene_release", "pcr_scene_bytes", "pcr_render", "pcr_render_noalloc",
    "pcr_submit", "pcr_run_until_idle", "pcr_serve_start", "pcr_serve_stop", "pcr_poll", "pcr_wait",
    "pcr_fetch", "pcr_cancel", "pcr_progress", "pcr_l2_bandwidth", "pcr_engine_stats_get", "pcr_engine_stats_reset", "pcr_autotune",
    "pcr_trace_closest", "pcr_trace_bvh", "pcr_trace_shadow", "pcr_bvh_build", "pcr_eval_stage",
    "pcr_tonemap", "pcr_router_create", "pcr_router_destroy", "pcr_router_scene_load_json", "pcr_router_serve_start",
    "pcr_router_serve_stop", "pcr_router_submit", "pcr_router_wait", "pcr_router_fetch", "pcr_router_load",
]


class PcrError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class Material(C.Structure):
    _fields_ = [("albedo", C.c_float * 3), ("emissive", C.c_float * 3), ("metallic", C.c_int32),
                ("transparent", C.c_int32), ("use_tab_albedo", C.c_int32), ("use_tab_emissive", C.c_int32),
                ("ior", C.c_float), ("cauchy_b", C.c_float), ("albedo_fit", C.c_float * 4),
                ("emissive_fit", C.c_float * 4), ("tab_albedo", C.c_float * SPEC_N),
                ("tab_emissive", C.c_float * SPEC_N)]


class Plane(C.Structure):
    _fields_ = [("origin", C.c_float * 3), ("u", C.c_float * 3), ("v", C.c_float * 3), ("n", C.c_float * 3),
                ("area", C.c_float), ("mat", C.c_int32)]


class Sphere(C.Structure):
    _fields_ = [("center", C.c_float * 3), ("radius", C.c_float), ("mat", C.c_int32)]


class Triangle(C.Structure):
    _fields_ = [("v0", C.c_float * 3), ("v1", C.c_float * 3), ("v2", C.c_float * 3), ("n0", C.c_float * 3),
                ("n1", C.c_float * 3), ("n2", C.c_float * 3), ("flat_n", C.c_float * 3), ("smooth", C.c_int32),
                ("mat", C.c_int32)]


class BvhNode(C.Structure):
    _fields_ = [("bmin", C.c_float * 3), ("bmax", C.c_float * 3), ("left_or_first", C.c_int32),
                ("right_child", C.c_int32), ("count", C.c_int32)]


class Light(C.Structure):
    _fields_ = [("kind", C.c_int32), ("total_area", C.c_float), ("plane", Plane), ("tri_offset", C.c_int32),
                ("tri_count", C.c_int32)]


class SceneDesc(C.Structure):
    _fields_ = [("name", C.c_char_p), ("version", C.c_char_p), ("cam_pos", C.c_float * 3), ("fov", C.c_float),
                ("n_materials", C.c_int32), ("materials", C.POINTER(Material)),
                ("n_spheres", C.c_int32), ("spheres", C.POINTER(Sphere)),
                ("n_planes", C.c_int32), ("planes", C.POINTER(Plane)),
                ("n_triangles", C.c_int32), ("triangles", C.POINTER(Triangle)),
                ("n_bvh_nodes", C.c_int32), ("bvh_nodes", C.POINTER(BvhNode)),
                ("n_lights", C.c_int32), ("lights", C.POINTER(Light)),
                ("light_triangles", C.POINTER(Triangle)), ("light_cum_area", C.POINTER(C.c_float)),
                ("triangle_ids", C.POINTER(C.c_int32))]


class RenderDesc(C.Structure):
    _fields_ = [(n, C.c_int32) for n in (
        "width", "height", "depth", "samples", "shadow_samples", "spectral", "hero_samples", "mis", "russian",
        "stratified", "aa_samples", "adaptive", "aces", "denoise")] + [("seed", C.c_uint64), ("priority", C.c_int32),
                                                                ("multi_sample", C.c_int32),
                                                                ("sample_begin", C.c_int32),
                                                                ("sample_end", C.c_int32),
                                                                ("spectral_terminate", C.c_int32)]


class RenderStats(C.Structure):
    _fields_ = [("device_ms", C.c_double), ("latency_ms", C.c_double), ("queue_ms", C.c_double),
                ("paths", C.c_uint64), ("rays", C.c_uint64), ("shadow_rays", C.c_uint64)]


class CtxOpts(C.Structure):
    _fields_ = [("device", C.c_int32), ("memory_budget", C.c_int64), ("queue_capacity", C.c_int32),
                ("block_size", C.c_int32), ("chunk_paths", C.c_int32), ("regen_every", C.c_int32),
                ("use_graph", C.c_int32), ("profile", C.c_int32), ("tuning_cache", C.c_char_p)]


class EngineStats(C.Structure):
    _fields_ = [("stage_ms", C.c_double * 8), ("stage_launches", C.c_int64 * 8), ("iterations", C.c_int64),
                ("paths", C.c_int64), ("rays", C.c_int64), ("shadow_rays", C.c_int64), ("device_bytes", C.c_int64),
                ("queue_capacity", C.c_int32), ("block_size", C.c_int32), ("chunk_paths", C.c_int32),
                ("regen_every", C.c_int32)]


STAGES = ["regen", "extend", "shade", "shadow", "resolve", "schedule", "status", "other"]

_lib = None


def load_library():
    """Loads the in-tree library.  Raises when it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FileNotFoundError(f"{LIB_PATH} missing: run `python -m pcr_b200.build`")
    L = C.CDLL(LIB_PATH)
    P = C.c_void_p
    st = C.c_int
    fp, ip, up = C.POINTER(C.c_float), C.POINTER(C.c_int32), C.POINTER(C.c_uint8)
    L.pcr_last_error.restype = C.c_char_p
    L.pcr_version.restype = C.c_char_p
    sig = {
        "pcr_ctx_create": [C.POINTER(P), C.POINTER(CtxOpts)],
        "pcr_ctx_destroy": [P],
        "pcr_ctx_set_device": [P],
        "pcr_ctx_stream": [P, C.POINTER(P)],
        "pcr_scene_upload": [P, C.POINTER(SceneDesc), ip],
        "pcr_scene_load_json": [P, C.c_char_p, C.c_char_p, C.c_char_p, ip],
        "pcr_scene_release": [P, C.c_int32],
        "pcr_host_scene_load": [C.c_char_p, C.c_char_p, C.c_char_p, C.POINTER(P), C.POINTER(SceneDesc)],
        "pcr_host_scene_free": [P],
        "pcr_fit_sigmoid": [fp, C.c_int64, fp, fp],
        "pcr_lut_build": [fp],
        "pcr_scene_bytes": [P, C.c_int32, C.POINTER(C.c_int64)],
        "pcr_render": [P, C.c_int32, C.POINTER(RenderDesc), fp, up, C.POINTER(RenderStats)],
        "pcr_render_noalloc": [P, C.c_int32, C.POINTER(RenderDesc), fp, up],
        "pcr_submit": [P, C.c_int32, C.POINTER(RenderDesc), C.POINTER(C.c_int64)],
        "pcr_run_until_idle": [P],
        "pcr_serve_start": [P],
        "pcr_serve_stop": [P],
        "pcr_poll": [P, C.c_int64, ip],
        "pcr_wait": [P, C.c_int64, C.c_int64],
        "pcr_fetch": [P, C.c_int64, fp, up, C.POINTER(RenderStats)],
        "pcr_cancel": [P, C.c_int64],
        "pcr_progress": [P, C.c_int64, C.POINTER(C.c_double)],
        "pcr_l2_bandwidth": [P, C.c_int64, C.c_int32, C.POINTER(C.c_double)],
        "pcr_engine_stats_get": [P, C.POINTER(EngineStats)],
        "pcr_engine_stats_reset": [P],
        "pcr_autotune": [P, ip, C.POINTER(RenderDesc), C.c_int32, ip],
        "pcr_trace_closest": [P, C.c_int32, fp, C.c_int64, ip, ip, fp],
        "pcr_trace_bvh": [P, C.c_int32, fp, C.c_int64, ip, fp, ip],
        "pcr_trace_shadow": [P, C.c_int32, fp, fp, C.c_int64, ip],
        "pcr_bvh_build": [P, fp, C.c_int32, fp, C.c_int32, ip, ip],
        "pcr_tonemap": [P, fp, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_uint8)],
        "pcr_router_create": [C.POINTER(P), C.POINTER(P), C.c_int32],
        "pcr_router_destroy": [P],
        "pcr_router_scene_load_json": [P, C.c_char_p, C.c_char_p, C.c_char_p, ip],
        "pcr_router_serve_start": [P],
        "pcr_router_serve_stop": [P],
        "pcr_router_submit": [P, C.c_int32, C.POINTER(RenderDesc), C.POINTER(C.c_int64)],
        "pcr_router_wait": [P, C.c_int64, C.c_int64],
        "pcr_router_fetch": [P, C.c_int64, fp, C.POINTER(C.c_uint8), C.POINTER(RenderStats)],
        "pcr_router_load": [P, C.POINTER(C.c_int64), C.POINTER(C.c_int64)],
        "pcr_eval_stage": [P, C.c_int32, fp, fp, C.c_int64, fp],
    }
    for name, args in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = st
    _lib = L
    return L


def _check(status: int) -> None:
    if status != 0:
        raise PcrError(status, load_library().pcr_last_error().decode())


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def render_desc(width, height=None, depth=4, samples=16, shadow=4, spectral=True, hero=4, mis=False,
                russian=False, stratified=False, aa=1, adaptive=False, aces=False, denoise=False, seed=1,
                priority=0, multi_sample=False, sample_begin=0, sample_end=0, terminate=False) -> RenderDesc:
    return RenderDesc(width, height or width, depth, samples, shadow, int(spectral), hero, int(mis),
                      int(russian), int(stratified), aa, int(adaptive), int(aces), int(denoise), seed, priority,
                      int(multi_sample), sample_begin, sample_end, int(terminate))


class HostScene:
    """A scene loaded by the library's own host loader (no GPU needed), with
    numpy views of its flat arrays."""

    def __init__(self, path: str, data_root: str | None = None, lut_path: str | None = None):
        self.L = load_library()
        self.h = C.c_void_p()
        self.desc = SceneDesc()
        _check(self.L.pcr_host_scene_load(path.encode(), data_root.encode() if data_root else None,
                                          lut_path.encode() if lut_path else None, C.byref(self.h),
                                          C.byref(self.desc)))

    def _arr(self, ptr, n, ctype, width):
        if n == 0:
            return np.zeros((0, width), np.float32)
        buf = (ctype * n).from_address(C.addressof(ptr.contents))
        return np.frombuffer(buf, np.float32).reshape(n, width).copy()

    def materials(self):
        return self._arr(self.desc.materials, self.desc.n_materials, Material, C.sizeof(Material) // 4)

    def planes(self):
        return self._arr(self.desc.planes, self.desc.n_planes, Plane, 14)

    def spheres(self):
        return self._arr(self.desc.spheres, self.desc.n_spheres, Sphere, 5)

    def triangles(self):
        return self._arr(self.desc.triangles, self.desc.n_triangles, Triangle, 23)

    def bvh(self):
        return self._arr(self.desc.bvh_nodes, self.desc.n_bvh_nodes, BvhNode, 9)

    def triangle_ids(self):
        n = self.desc.n_triangles
        if n == 0:
            return np.zeros(0, np.int32)
        return np.ctypeslib.as_array(self.desc.triangle_ids, shape=(n,)).copy()

    def close(self):
        if self.h:
            self.L.pcr_host_scene_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def fit_sigmoid(rgb: np.ndarray, lut: np.ndarray | None = None) -> np.ndarray:
    x = np.ascontiguousarray(rgb, np.float32).reshape(-1, 3)
    out = np.zeros((x.shape[0], 4), np.float32)
    lp = np.ascontiguousarray(lut, np.float32) if lut is not None else None
    _check(load_library().pcr_fit_sigmoid(_fp(x), x.shape[0], _fp(lp) if lp is not None else None, _fp(out)))
    return out


def lut_build() -> np.ndarray:
    out = np.zeros(3 * 16 ** 3 * 3, np.float32)
    _check(load_library().pcr_lut_build(_fp(out)))
    return out


class Context:
    """One engine on one GPU: device scene cache, request table, queues."""

    def __init__(self, device: int = 0, memory_budget: int = 0, queue_capacity: int = 0, block_size: int = 0,
                 chunk_paths: int = 0, regen_every: int = 0, use_graph: bool = True, profile: bool = False,
                 tuning_cache: str | None = None):
        self.L = load_library()
        self.device = device
        self._cache = tuning_cache.encode() if tuning_cache else None
        o = CtxOpts(device, memory_budget, queue_capacity, block_size, chunk_paths, regen_every, int(use_graph),
                    int(profile), self._cache)
        h = C.c_void_p()
        _check(self.L.pcr_ctx_create(C.byref(h), C.byref(o)))
        self.h = h
        self._keep = {}

    def close(self):
        if getattr(self, "h", None):
            self.L.pcr_ctx_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def stream(self) -> int:
        """cudaStream_t of the engine, as an integer handle."""
        s = C.c_void_p()
        _check(self.L.pcr_ctx_stream(self.h, C.byref(s)))
        return s.value or 0

    # ---------------------------------------------------------------- scenes
    def load_scene_json(self, path: str, data_root: str | None = None, lut_path: str | None = None) -> int:
        sid = C.c_int32()
        _check(self.L.pcr_scene_load_json(self.h, path.encode(), data_root.encode() if data_root else None,
                                          lut_path.encode() if lut_path else None, C.byref(sid)))
        return sid.value

    def upload_scene(self, desc: SceneDesc) -> int:
        sid = C.c_int32()
        _check(self.L.pcr_scene_upload(self.h, C.byref(desc), C.byref(sid)))
        return sid.value

    def release_scene(self, sid: int) -> None:
        _check(self.L.pcr_scene_release(self.h, sid))

    def scene_bytes(self, sid: int) -> int:
        b = C.c_int64()
        _check(self.L.pcr_scene_bytes(self.h, sid, C.byref(b)))
        return b.value

    # ---------------------------------------------------------------- rendering
    def render(self, sid: int, desc: RenderDesc, want_hdr=True, want_rgb=True):
        """Plain method (one render, own launch sequence).  -> (hdr, rgb8, stats)"""
        hdr = np.zeros((desc.height, desc.width, 3), np.float32) if want_hdr else None
        rgb = np.zeros((desc.height, desc.width, 3), np.uint8) if want_rgb else None
        st = RenderStats()
        _check(self.L.pcr_render(self.h, sid, C.byref(desc), _fp(hdr) if want_hdr else None,
                                 rgb.ctypes.data_as(C.POINTER(C.c_uint8)) if want_rgb else None, C.byref(st)))
        return hdr, rgb, st

    def render_noalloc(self, sid: int, desc: RenderDesc, hdr_dev_ptr: int, rgb_dev_ptr: int) -> None:
        """Plain render that allocates no device memory (pcr_render_noalloc):
        outputs go to caller-owned device buffers given as raw pointers."""
        _check(self.L.pcr_render_noalloc(self.h, sid, C.byref(desc), C.cast(C.c_void_p(hdr_dev_ptr), C.POINTER(C.c_float))
                                         if hdr_dev_ptr else None,
                                         C.cast(C.c_void_p(rgb_dev_ptr), C.POINTER(C.c_uint8)) if rgb_dev_ptr else None))

    def submit(self, sid: int, desc: RenderDesc) -> int:
        rid = C.c_int64()
        _check(self.L.pcr_submit(self.h, sid, C.byref(desc), C.byref(rid)))
        self._keep[rid.value] = (desc.width, desc.height)
        return rid.value

    def run_until_idle(self) -> None:
        _check(self.L.pcr_run_until_idle(self.h))

    def serve_start(self) -> None:
        _check(self.L.pcr_serve_start(self.h))

    def serve_stop(self) -> None:
        _check(self.L.pcr_serve_stop(self.h))

    def poll(self, rid: int) -> bool:
        d = C.c_int32()
        _check(self.L.pcr_poll(self.h, rid, C.byref(d)))
        return bool(d.value)

    def wait(self, rid: int, timeout_ms: int = -1) -> None:
        _check(self.L.pcr_wait(self.h, rid, timeout_ms))

    def fetch(self, rid: int, want_hdr=True, want_rgb=True, hdr_out=None, rgb_out=None):
        """Copies a finished request's images to the host: new arrays, or the
        caller's (H, W, 3) float32 / uint8 buffers when given."""
        w, h = self._keep[rid]
        hdr = rgb = None
        if want_hdr:
            hdr = hdr_out if hdr_out is not None else np.zeros((h, w, 3), np.float32)
            if hdr.shape != (h, w, 3) or hdr.dtype != np.float32 or not hdr.flags.c_contiguous:
                raise ValueError("hdr_out must be a C-contiguous float32 (H, W, 3) array")
        if want_rgb:
            rgb = rgb_out if rgb_out is not None else np.zeros((h, w, 3), np.uint8)
            if rgb.shape != (h, w, 3) or rgb.dtype != np.uint8 or not rgb.flags.c_contiguous:
                raise ValueError("rgb_out must be a C-contiguous uint8 (H, W, 3) array")
        st = RenderStats()
        try:
            _check(self.L.pcr_fetch(self.h, rid, _fp(hdr) if want_hdr else None,
                                    rgb.ctypes.data_as(C.POINTER(C.c_uint8)) if want_rgb else None, C.byref(st)))
        except PcrError as e:
            if e.status == 7:      # cancelled: the library released it
                del self._keep[rid]
            raise
        del self._keep[rid]
        return hdr, rgb, st

    def cancel(self, rid: int) -> None:
        _check(self.L.pcr_cancel(self.h, rid))

    def l2_bandwidth(self, nbytes: int = 32 << 20, reps: int = 400) -> float:
        """Measured L2 read bandwidth of this context's device, GB/s."""
        g = C.c_double()
        _check(self.L.pcr_l2_bandwidth(self.h, nbytes, reps, C.byref(g)))
        return g.value

    def progress(self, rid: int) -> float:
        f = C.c_double()
        _check(self.L.pcr_progress(self.h, rid, C.byref(f)))
        return f.value

    def stats(self) -> dict:
        s = EngineStats()
        _check(self.L.pcr_engine_stats_get(self.h, C.byref(s)))
        return {"stage_ms": dict(zip(STAGES, list(s.stage_ms))),
                "stage_launches": dict(zip(STAGES, list(s.stage_launches))),
                "iterations": s.iterations, "paths": s.paths, "rays": s.rays, "shadow_rays": s.shadow_rays,
                "device_bytes": s.device_bytes, "queue_capacity": s.queue_capacity, "block_size": s.block_size,
                "chunk_paths": s.chunk_paths, "regen_every": s.regen_every}

    def reset_stats(self) -> None:
        _check(self.L.pcr_engine_stats_reset(self.h))

    def autotune(self, sids, descs):
        n = len(sids)
        s = np.asarray(sids, np.int32)
        arr = (RenderDesc * n)(*descs)
        chosen = np.zeros(4, np.int32)
        _check(self.L.pcr_autotune(self.h, _ip(s), arr, n, _ip(chosen)))
        return dict(zip(["queue_capacity", "block_size", "chunk_paths", "regen_every"], chosen.tolist()))

    # ---------------------------------------------------------------- parity entry points
    def trace_closest(self, sid: int, rays: np.ndarray):
        r = np.ascontiguousarray(rays, np.float32)
        n = r.shape[0]
        mat = np.zeros(n, np.int32)
        prim = np.zeros(n, np.int32)
        t = np.zeros(n, np.float32)
        _check(self.L.pcr_trace_closest(self.h, sid, _fp(r), n, _ip(mat), _ip(prim), _fp(t)))
        return mat, prim, t

    def trace_bvh(self, sid: int, rays: np.ndarray, counts: bool = False):
        r = np.ascontiguousarray(rays, np.float32)
        n = r.shape[0]
        tid = np.zeros(n, np.int32)
        t = np.zeros(n, np.float32)
        cnt = np.zeros((n, 2), np.int32) if counts else None
        _check(self.L.pcr_trace_bvh(self.h, sid, _fp(r), n, _ip(tid), _fp(t), _ip(cnt) if counts else None))
        return (tid, t, cnt) if counts else (tid, t)

    def trace_shadow(self, sid: int, rays: np.ndarray, light_dist2: np.ndarray) -> np.ndarray:
        """Shadow test per ray (origin, unit direction) with its squared light
        distance: 1 where blocked."""
        r = np.ascontiguousarray(rays, np.float32)
        d2 = np.ascontiguousarray(light_dist2, np.float32)
        n = r.shape[0]
        out = np.zeros(n, np.int32)
        _check(self.L.pcr_trace_shadow(self.h, sid, _fp(r), _fp(d2), n, _ip(out)))
        return out

    def build_bvh(self, verts: np.ndarray):
        """Device SAH build over n triangles given as (n, 9) vertices
        (v0 v1 v2): returns (nodes as (m, 9) float32 rows with the last
        three words int32, order) like HostScene.bvh() / triangle_ids()."""
        v = np.ascontiguousarray(verts, np.float32).reshape(-1, 9)
        n = v.shape[0]
        tris = np.zeros((n, 23), np.float32)
        tris[:, :9] = v
        nodes = np.zeros((max(2 * n - 1, 1), 9), np.float32)
        order = np.zeros(n, np.int32)
        m = C.c_int32(0)
        _check(self.L.pcr_bvh_build(self.h, _fp(tris), n, _fp(nodes), nodes.shape[0], C.byref(m), _ip(order)))
        return nodes[:m.value].copy(), order

    def tonemap(self, hdr: np.ndarray, aces=False, denoise=False) -> np.ndarray:
        """8-bit image of a linear sRGB image (H, W, 3), on the device."""
        h = np.ascontiguousarray(hdr, np.float32)
        out = np.zeros(h.shape, np.uint8)
        _check(self.L.pcr_tonemap(self.h, _fp(h), h.shape[1], h.shape[0], int(aces), int(denoise),
                                  out.ctypes.data_as(C.POINTER(C.c_uint8))))
        return out

    def eval_stage(self, what: int, inp: np.ndarray, params: np.ndarray | None = None) -> np.ndarray:
        x = np.ascontiguousarray(inp, np.float32)
        widths_in = {0: 1, 1: 1, 2: 1, 3: 2, 4: 3, 5: 3, 6: 3, 7: 3, 8: 2}
        n = x.size // widths_in[what]
        out = np.zeros((n, 1 if what in (0, 1) else 3), np.float32)
        p = np.ascontiguousarray(params, np.float32) if params is not None else None
        _check(self.L.pcr_eval_stage(self.h, what, _fp(p) if p is not None else None, _fp(x), n, _fp(out)))
        return out


class Router:
    """Request router over several contexts (pcr_router_*): scenes are
    replicated into every context; each request goes to the context with
    the fewest paths outstanding.  The contexts must outlive the router."""

    def __init__(self, contexts):
        self.L = load_library()
        self.ctxs = list(contexts)
        arr = (C.c_void_p * len(self.ctxs))(*[c.h.value for c in self.ctxs])
        h = C.c_void_p()
        _check(self.L.pcr_router_create(C.byref(h), C.cast(arr, C.POINTER(C.c_void_p)), len(self.ctxs)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            _check(self.L.pcr_router_destroy(self.h))
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def load_scene_json(self, path: str, data_root: str | None = None, lut_path: str | None = None) -> int:
        out = C.c_int32()
        _check(self.L.pcr_router_scene_load_json(self.h, path.encode(), data_root.encode() if data_root else None,
                                                 lut_path.encode() if lut_path else None, C.byref(out)))
        return out.value

    def serve_start(self) -> None:
        _check(self.L.pcr_router_serve_start(self.h))

    def serve_stop(self) -> None:
        _check(self.L.pcr_router_serve_stop(self.h))

    def submit(self, sid: int, desc: RenderDesc) -> int:
        t = C.c_int64()
        _check(self.L.pcr_router_submit(self.h, sid, C.byref(desc), C.byref(t)))
        return t.value

    def wait(self, ticket: int, timeout_ms: int = -1) -> None:
        _check(self.L.pcr_router_wait(self.h, ticket, timeout_ms))

    def fetch(self, ticket: int, width: int, height: int, want_hdr=True, want_rgb=True):
        hdr = np.zeros((height, width, 3), np.float32) if want_hdr else None
        rgb = np.zeros((height, width, 3), np.uint8) if want_rgb else None
        st = RenderStats()
        _check(self.L.pcr_router_fetch(self.h, ticket, _fp(hdr) if want_hdr else None,
                                       rgb.ctypes.data_as(C.POINTER(C.c_uint8)) if want_rgb else None, C.byref(st)))
        return hdr, rgb, st

    def load(self):
        n = len(self.ctxs)
        out = (C.c_int64 * n)()
        routed = (C.c_int64 * n)()
        _check(self.L.pcr_router_load(self.h, out, routed))
        return list(out), list(routed)
