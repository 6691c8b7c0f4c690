"""The headless render layer's banded frames on the GPU: r3d_frame draws a
whole-image view as row bands on two streams and r3d_read_frame copies each
band as it completes; the image equals the one-launch raycast bit for bit,
full and half resolution, and frames of several views still render whole.
r3d_cuda_raycast_rows renders any row range of a view exactly like the
whole view."""
import numpy as np
import pytest

from conftest import elev35

pytestmark = pytest.mark.gpu

W, H = 640, 480


@pytest.fixture(scope="module")
def renderer(rb, phantom256, scroll_tf):
    r = rb.Renderer(W, H)
    r.set_transfer(scroll_tf)
    r.set_alpha_cutoff(0.98)
    r.bricks_begin_volume(phantom256, 2)
    c = rb.Context(0)
    c.set_transfer(scroll_tf)
    c.set_alpha_cutoff(0.98)
    c.bricks_build(phantom256, 2)
    yield r, c
    c.close()
    r.close()


@pytest.mark.parametrize("half", [False, True])
def test_banded_frame_equals_whole(rb, renderer, scroll_tf, half):
    import torch
    r, c = renderer
    host = torch.empty((H, W, 4), dtype=torch.uint8, pin_memory=True).numpy()
    for i in range(3):  # consecutive frames reuse the band events
        p = elev35(rb, scroll_tf, W, H, step_voxels=0.5)
        p.frame_index = i
        if half:
            p.view_flags |= rb.VIEW_HALF
        r.bricks_params(p)
        r.frame(p)
        got = r.read_frame(host).copy()
        p.brick_mode = c.brick_mode
        ref = c.raycast(p, W, H)
        assert np.array_equal(got, ref), (half, i)
        assert got[..., :3].std() > 5


def test_multi_view_frame(rb, renderer, scroll_tf):
    r, c = renderer
    views = []
    for k in range(2):
        p = elev35(rb, scroll_tf, W // 2, H, step_voxels=0.5)
        p.view_org = (W // 2) * k
        r.bricks_params(p)
        views.append(p)
    r.frame_views(views)
    got = r.read_frame()
    for p in views:
        p.brick_mode = c.brick_mode
    ref = c.raycast(views, W, H)
    assert np.array_equal(got, ref)


def test_raycast_rows(rb, renderer, scroll_tf):
    import torch
    _, c = renderer
    p = elev35(rb, scroll_tf, W, H, step_voxels=0.5)
    p.brick_mode = c.brick_mode
    ref = c.raycast(p, W, H)
    img = torch.zeros((H, W, 4), dtype=torch.uint8, device="cuda")
    for r0, r1 in [(0, 100), (100, 333), (333, 10 ** 6)]:  # 100 and 333 round down to 96, 328
        c.raycast_rows(p, img, W, H, r0, r1)
    torch.cuda.synchronize()
    assert np.array_equal(img.cpu().numpy(), ref)
    part = torch.zeros((H, W, 4), dtype=torch.uint8, device="cuda")
    c.raycast_rows(p, part, W, H, 200, 240)
    torch.cuda.synchronize()
    a = part.cpu().numpy()
    assert np.array_equal(a[200:240], ref[200:240]) and not a[:200].any() and not a[240:].any()
    with pytest.raises(rb.R3DError):
        c.raycast_rows(p, np.zeros((H, W, 4), np.uint8), W, H, 0, H)  # host image
