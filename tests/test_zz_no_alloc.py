"""The forward raycast entry point that allocates no device memory.

r3d_cuda_raycast_fwd_noalloc serves callers that must not let the library
allocate while they render: applications that give the renderer a fixed
device-memory budget at start-up and forbid allocation afterwards, and
real-time render threads for which an allocation (which can synchronize the
device) is a frame hitch.  Its per-call scratch lives in a fixed device
array inside the library.  Here it is called through the C-ABI and compared
with the regular entry point, r3d_cuda_raycast_fwd, on two calls in a row
(the second call reuses the scratch the first one left behind); every ray
is computed the same way under every schedule, so the images must be equal
byte for byte.  Two calls are also queued on one non-default stream with a
single synchronize after both: the shared scratch is ordered by the stream.
This file sorts last so that a run stopping at the first failure has already
run every other test; it also passes alone in a fresh process.
"""
import ctypes as C

import pytest

pytestmark = pytest.mark.gpu


def _views(rb, lut, brick_mode, w, h, yaws, modes):
    vs = []
    for i, (yaw, mode) in enumerate(zip(yaws, modes)):
        p = rb.camera_view(yaw, -0.45, 1.7, w, h, lut, step_voxels=0.5, mode=mode, frame_index=i)
        p.brick_mode = brick_mode
        p.view_org = (w * (i % 2)) | ((h * (i // 2)) << 16)
        vs.append(p)
    return vs


def _noalloc(rb, ctx, views, out, W, H, stream):
    arr = (rb.FrameParams * len(views))(*views)
    rc = rb.lib.r3d_cuda_raycast_fwd_noalloc(ctx.h, arr, len(views), out.data_ptr(), W, H,
                                             C.c_void_p(stream))
    assert rc == 0, rb.lib.r3d_cuda_last_error(ctx.h).decode()


def test_noalloc_matches_regular_entry_point():
    import torch

    import render3d_b200 as rb

    ctx = rb.Context(0)
    try:
        lut = rb.scroll_ramp_tf()
        ctx.set_transfer(lut)
        ctx.bricks_build(rb.phantom(256, seed=21), nlev=2)
        w, h = 160, 120
        W, H = 2 * w, 2 * h
        off = _views(rb, lut, ctx.brick_mode, w, h, [0.7], [0])[0]
        off.view_org = (W + 8) | (4 << 16)  # wholly right of the image: skipped
        calls = [_views(rb, lut, ctx.brick_mode, w, h, [0.3, 1.3, 2.3, 3.3], [0, 1, 3, 5]),
                 _views(rb, lut, ctx.brick_mode, w, h, [4.0, 5.0], [0, 0]) + [off]]
        for views in calls:
            want = torch.zeros((H, W, 4), dtype=torch.uint8, device="cuda")
            got = torch.zeros((H, W, 4), dtype=torch.uint8, device="cuda")
            ctx.raycast(views, W, H, out=want, stream=ctx.stream)
            _noalloc(rb, ctx, views, got, W, H, ctx.stream)
            torch.cuda.synchronize()
            assert want.float().mean().item() > 1.0  # something was rendered
            assert torch.equal(got, want), "no-alloc output differs from r3d_cuda_raycast_fwd"
        # two calls queued back to back on a stream of the caller's, one
        # synchronize: the second call's table write waits for the first call
        side = torch.cuda.Stream()
        outs = [torch.zeros((H, W, 4), dtype=torch.uint8, device="cuda") for _ in calls]
        wants = []
        for views in calls:
            wv = torch.zeros((H, W, 4), dtype=torch.uint8, device="cuda")
            ctx.raycast(views, W, H, out=wv, stream=ctx.stream)
            wants.append(wv)
        torch.cuda.synchronize()
        for views, o in zip(calls, outs):
            _noalloc(rb, ctx, views, o, W, H, side.cuda_stream)
        side.synchronize()
        for o, wv in zip(outs, wants):
            assert torch.equal(o, wv)
        # the context's persistent schedule knobs are honoured: results unchanged
        ctx.set_schedule(persistent=0, refill_min=8, tile_shape=1, unroll=2)
        got = torch.zeros((H, W, 4), dtype=torch.uint8, device="cuda")
        _noalloc(rb, ctx, calls[0], got, W, H, ctx.stream)
        torch.cuda.synchronize()
        assert torch.equal(got, wants[0])
        ctx.set_schedule()
        # more views than the fixed scratch holds are rejected, not truncated
        many = (rb.FrameParams * 65)(*([calls[1][0]] * 65))
        out = torch.zeros((H, W, 4), dtype=torch.uint8, device="cuda")
        rc = rb.lib.r3d_cuda_raycast_fwd_noalloc(ctx.h, many, 65, out.data_ptr(), W, H, None)
        assert rc == -1 and b"at most 64" in rb.lib.r3d_cuda_last_error(ctx.h)
    finally:
        ctx.close()
