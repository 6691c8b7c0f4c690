"""The TMA-staged raycast (r3d_cuda_schedule.staging = 1): LOD-brick views
in FULL and MIP mode marched by 8x8 ray tiles that copy slot boxes into
shared memory with cp.async.bulk.tensor.  Its images equal, byte for byte,
those of the one-thread-per-ray kernel (whose parity with the oracle the
other tests establish), at several views, both gradient qualities and half
resolution, with no bounded wait giving up."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lod_scene(rb, ctx, phantom256, scroll_tf):
    ctx.set_transfer(scroll_tf)
    ctx.set_alpha_cutoff(0.99)
    ctx.bricks_build(phantom256, nlev=2)
    yield ctx
    ctx.set_alpha_cutoff(0.98)
    ctx.set_quality(0)
    ctx.set_schedule()


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("quality", [0, 1])
def test_staged_equals_grid(rb, lod_scene, scroll_tf, mode, quality):
    ctx = lod_scene
    if mode == 1 and quality == 1:
        pytest.skip("quality only changes FULL shading")
    ctx.set_quality(quality)
    ctx.status()
    for i, (yaw, pitch, dist) in enumerate([(0.3, -0.4, 1.6), (2.0, 0.2, 1.2), (4.1, -0.9, 2.4)]):
        p = rb.camera_view(yaw, pitch, dist, 320, 200, scroll_tf, step_voxels=0.5, mode=mode,
                           frame_index=i)
        p.brick_mode = ctx.brick_mode
        if i == 2:
            p.view_flags = rb.VIEW_HALF
        ctx.set_schedule()
        want = ctx.raycast(p, 320, 200)
        ctx.set_schedule(staging=1)
        got = ctx.raycast(p, 320, 200)
        ctx.set_schedule()
        assert np.array_equal(got, want), f"view {i}"
        assert want[..., :3].std() > 2
    assert ctx.status() == 0  # no wait ran out


def test_staged_frame_1080p(rb, ctx, scroll_tf):
    """A 1080p orbit frame of a 512^3 cache with four levels: staged equals
    the grid kernel."""
    import torch
    vol = ctx.phantom(512, seed=77)
    ctx.bricks_build(vol, nlev=4)
    del vol
    torch.cuda.empty_cache()
    ctx.set_transfer(scroll_tf)
    try:
        for mode in (0, 1):
            p = rb.orbit_view(0.3, 1920, 1080, scroll_tf, step_voxels=0.5, mode=mode,
                              frame_index=3)
            p.brick_mode = ctx.brick_mode
            want = ctx.raycast(p, 1920, 1080)
            ctx.set_schedule(staging=1)
            got = ctx.raycast(p, 1920, 1080)
            ctx.set_schedule()
            assert np.array_equal(got, want), mode
        assert ctx.status() == 0
    finally:
        ctx.set_schedule()
