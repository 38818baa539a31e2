"""pcr_render_noalloc: a plain render that allocates no device memory.

Some callers cannot allocate during a render: a host that has given all
device memory to its own pool allocator, or a real-time loop that cannot
pay for cudaMalloc / cudaFree, which synchronize the whole device.  For them
the library renders out of one fixed scratch array compiled into it and
writes into device buffers the caller owns.  Here the caller's buffers come
from torch, and the result must equal the ordinary entry point's
(pcr_render) within the tolerance the batched-invariance test uses, on two
calls in a row (the second call must not see the first call's leftovers),
and on a small call made right after a large one (the small call must not
pick up queue, hit or accumulator contents the large one left beyond the
ranges it uses).  A call must leave the device's free memory and the
context's own device bytes unchanged.

This file is named to run last: if it fails, a run that stops at the first
failure has already run every other test.
"""
import numpy as np
import pytest

from conftest import GOLDEN, scene_path

pytestmark = pytest.mark.gpu


def _noalloc(ctx, sid, desc, hdr, rgb):
    import torch
    w, h = desc.width, desc.height
    hdr.fill_(float("nan"))
    rgb.fill_(0)
    torch.cuda.synchronize()
    ctx.render_noalloc(sid, desc, hdr.data_ptr(), rgb.data_ptr())
    torch.cuda.synchronize()
    return hdr[: h * w * 3].cpu().numpy().reshape(h, w, 3), rgb[: h * w * 3].cpu().numpy().reshape(h, w, 3)


def _same(got_hdr, got_rgb, ref_hdr, ref_rgb):
    assert np.isfinite(got_hdr).all()
    assert np.allclose(got_hdr, ref_hdr, rtol=1e-6, atol=1e-7)
    assert np.abs(got_rgb.astype(int) - ref_rgb.astype(int)).max() <= 1


def test_render_noalloc_matches_render_on_two_calls():
    import torch

    from pcr_b200 import capi
    ctx = capi.Context(device=0)
    # dispersive glass: the fork path runs too
    sid = ctx.load_scene_json(scene_path("cornell-glass"), GOLDEN)
    w, h = 96, 80
    desc = capi.render_desc(w, h, depth=4, samples=32, shadow=4, spectral=True, seed=21)
    ref_hdr, ref_rgb, _ = ctx.render(sid, desc)
    hdr = torch.empty(256 * 256 * 3, dtype=torch.float32, device="cuda:0")
    rgb = torch.empty(256 * 256 * 3, dtype=torch.uint8, device="cuda:0")
    for _ in range(2):
        _same(*_noalloc(ctx, sid, desc, hdr, rgb), ref_hdr, ref_rgb)

    # a call allocates nothing: free device memory and the context's bytes
    # are the same before and after it (every kernel is loaded by now)
    free0, ctx0 = torch.cuda.mem_get_info()[0], ctx.stats()["device_bytes"]
    _noalloc(ctx, sid, desc, hdr, rgb)
    assert torch.cuda.mem_get_info()[0] == free0, "pcr_render_noalloc changed the device's free memory"
    assert ctx.stats()["device_bytes"] == ctx0

    # a large call (the size limit, 8 shadow rays, depth 6) and then the
    # small one again: nothing of the large call's scratch leaks into it
    big = capi.render_desc(256, 256, depth=6, samples=4, shadow=8, spectral=True, seed=5)
    big_hdr, big_rgb, _ = ctx.render(sid, big)
    _same(*_noalloc(ctx, sid, big, hdr, rgb), big_hdr, big_rgb)
    _same(*_noalloc(ctx, sid, desc, hdr, rgb), ref_hdr, ref_rgb)

    # requests beyond the fixed scratch are refused with a clear error
    too_big = capi.render_desc(512, depth=2, samples=1, shadow=1, seed=1)
    with pytest.raises(capi.PcrError) as e:
        ctx.render_noalloc(sid, too_big, hdr.data_ptr(), rgb.data_ptr())
    assert e.value.status == 1 and "65536-pixel limit" in str(e.value)
    ctx.close()
