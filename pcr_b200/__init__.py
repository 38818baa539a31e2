"""pcr_b200: B200-native (sm_100a) wavefront spectral path tracer behind the
C ABI of include/pcr_cuda.h.

    from pcr_b200 import capi
    ctx = capi.Context()
    sid = ctx.load_scene_json("Scenes/cornell.json")
    hdr, rgb8, stats = ctx.render(sid, capi.render_desc(256, depth=4, samples=16, shadow=4))

`pcr_b200.renderer.Renderer` mirrors the reference renderer's surface
(constructor, quality knobs, render(scene, start, outputDir) writing the PNG).
"""
from . import capi  # noqa: F401

__all__ = ["capi"]
