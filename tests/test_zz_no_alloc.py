"""The forward raycast entry point that allocates no device memory.

r3d_cuda_raycast_fwd_noalloc serves callers that must not let the library
allocate while they render: applications that give the renderer a fixed
device-memory budget at start-up and forbid allocation afterwards, and
real-time render threads for which an allocation (which can synchronize the
device) is a frame hitch.  Its per-call scratch lives in a fixed device
array inside the library.  Here it is called through the C-ABI and compared
with the regular entry point, r3d_cuda_raycast_fwd, on two calls in a row
(the second call reuses the scratch the first one left behind).  This file
sorts last so that a run stopping at the first failure has already run
every other test; it also passes alone in a fresh process.
"""
import ctypes as C
import math

import numpy as np
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
        calls = [_views(rb, lut, ctx.brick_mode, w, h, [0.3, 1.3, 2.3, 3.3], [0, 1, 3, 5]),
                 _views(rb, lut, ctx.brick_mode, w, h, [4.0, 5.0], [0, 0])]
        for views in calls:
            arr = (rb.FrameParams * len(views))(*views)
            want = torch.zeros((H, W, 4), dtype=torch.uint8, device="cuda")
            got = torch.zeros((H, W, 4), dtype=torch.uint8, device="cuda")
            ctx.raycast(views, W, H, out=want, stream=ctx.stream)
            rc = rb.lib.r3d_cuda_raycast_fwd_noalloc(ctx.h, arr, len(views), got.data_ptr(), W,
                                                     H, C.c_void_p(ctx.stream))
            assert rc == 0, rb.lib.r3d_cuda_last_error(ctx.h).decode()
            torch.cuda.synchronize()
            d = (got.int() - want.int()).abs().max().item()
            assert d <= 1, f"no-alloc output differs by {d}"
            assert want.float().mean().item() > 1.0  # something was rendered
        # more views than the fixed scratch holds are rejected, not truncated
        many = (rb.FrameParams * 65)(*([calls[1][0]] * 65))
        out = torch.zeros((H, W, 4), dtype=torch.uint8, device="cuda")
        rc = rb.lib.r3d_cuda_raycast_fwd_noalloc(ctx.h, many, 65, out.data_ptr(), W, H, None)
        assert rc == -1 and b"at most 64" in rb.lib.r3d_cuda_last_error(ctx.h)
    finally:
        ctx.close()
