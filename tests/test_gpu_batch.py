"""Batched raycast: many views of uneven size, each into its own device
image, in persistent launches; direct launch, CUDA-graph replay and every
autotuned schedule produce the images of single-view raycasts bit for bit."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _views(rb, lut, brick_mode):
    rng = np.random.default_rng(17)
    vs = []
    for i in range(5):  # perspective views of uneven sizes
        w, h = [(192, 108), (96, 200), (64, 64), (250, 90), (33, 47)][i]
        vs.append(rb.camera_view(rng.uniform(0, 6.3), rng.uniform(-0.8, 0.8),
                                 rng.uniform(1.3, 2.2), w, h, lut, step_voxels=0.5,
                                 frame_index=i))
    for i in range(4):  # ortho slice panes at arbitrary normals (oblique slab)
        n = rng.normal(size=3)
        n /= np.linalg.norm(n)
        p = rb.camera_view(0.0, 0.0, 1.0, 96, 54, lut, step_voxels=0.5)
        c = np.array([0.5, 0.5, 0.5]) - n * 0.9
        up = np.cross(n, [1.0, 0.0, 0.0])
        up /= np.linalg.norm(up)
        rt = np.cross(up, n)
        p.cam_origin[:] = c.tolist()
        p.cam_forward[:] = n.tolist()
        p.cam_right[:] = (rt * 0.5).tolist()
        p.cam_up[:] = (up * 0.5 * 54 / 96).tolist()
        p.view_flags = rb.VIEW_ORTHO | rb.VIEW_OBLIQUE
        p.slab_z0, p.slab_depth = 200.0 + 10 * i, 12
        vs.append(p)
    for i in range(3):  # axis slab windows looking down z
        p = rb.camera_view(0.0, 0.0, 1.0, 128, 128, lut, step_voxels=0.5)
        p.cam_origin[:] = [0.5, 0.5, -0.5]
        p.cam_forward[:] = [0.0, 0.0, 1.0]
        p.cam_right[:] = [0.5, 0.0, 0.0]
        p.cam_up[:] = [0.0, 0.5, 0.0]
        p.view_flags = rb.VIEW_ORTHO | rb.VIEW_AXIS(0)
        p.slab_z0, p.slab_depth = 40.0 + 60 * i, 32
        vs.append(p)
    vs[2].mode = rb.MODE_MIP
    vs[6].mode = rb.MODE_HEATMAP
    for v in vs:
        v.brick_mode = brick_mode
    return vs


@pytest.fixture(scope="module")
def batch_scene(rb, ctx, phantom256, scroll_tf):
    ctx.set_transfer(scroll_tf)
    ctx.set_alpha_cutoff(0.98)
    ctx.set_quality(0)
    ctx.bricks_build(phantom256, nlev=2)
    views = _views(rb, scroll_tf, ctx.brick_mode)
    refs, steps = [], 0
    for v in views:
        tot = np.zeros(1, np.uint64)
        refs.append(ctx.raycast(v, v.viewport[0], v.viewport[1], total=tot))
        steps += int(tot[0])
    return views, refs, steps


def _images(views):
    import torch
    return [torch.zeros((v.viewport[1], v.viewport[0], 4), dtype=torch.uint8, device="cuda")
            for v in views]


def _check(imgs, refs):
    for im, ref in zip(imgs, refs):
        assert np.array_equal(im.cpu().numpy(), ref)


def test_batch_launch_matches_single_views(rb, ctx, batch_scene):
    import torch
    views, refs, steps = batch_scene
    imgs = _images(views)
    b = rb.Batch(ctx, views, imgs)
    tot = torch.zeros(1, dtype=torch.int64, device="cuda")
    b.launch(total=tot, stream=ctx.stream)
    torch.cuda.synchronize()
    _check(imgs, refs)
    assert tot.item() == steps
    b.close()


def test_batch_graph_replay(rb, ctx, batch_scene):
    import torch
    views, refs, _ = batch_scene
    imgs = _images(views)
    b = rb.Batch(ctx, views, imgs)
    b.capture(stream=ctx.stream)
    torch.cuda.synchronize()
    _check(imgs, refs)
    for im in imgs:
        im.zero_()
    torch.cuda.synchronize()
    b.replay(stream=ctx.stream)
    b.replay(stream=ctx.stream)
    torch.cuda.synchronize()
    _check(imgs, refs)
    b.close()


def test_batch_autotune_keeps_results(rb, ctx, batch_scene):
    import torch
    views, refs, _ = batch_scene
    imgs = _images(views)
    b = rb.Batch(ctx, views, imgs)
    best, ms = b.autotune(reps=2)
    assert ms > 0 and best == b.schedule()
    for sc in [dict(persistent=0), dict(persistent=1, tile_shape=2, refill_min=24, unroll=2)]:
        for im in imgs:
            im.zero_()
        b.set_schedule(**sc)
        b.launch(stream=ctx.stream)
        torch.cuda.synchronize()
        _check(imgs, refs)
    b.close()
