"""pcr_b200: B200-native (sm_100a) wavefront spectral path tracer behind the
C ABI of include/pcr_cuda.h.

    from pcr_b200 import capi
    ctx = capi.Context()
    sid = ctx.load_scene_json("Scenes/cornell.json")
    hdr, rgb8, stats = ctx.render(sid, capi.render_desc(256, depth=4, samples=16, shadow=4))

The reference renderer's C++ surface (constructor, quality knobs,
render(scene, start, outputDir) writing the PNG) is `CudaRenderer` in
pcr_b200/csrc/cuda_renderer.h, built over the same C ABI; the `pcr-render`
CLI in pcr_b200/lib takes the reference CLI's flags.
"""
from . import capi  # noqa: F401

__all__ = ["capi"]
