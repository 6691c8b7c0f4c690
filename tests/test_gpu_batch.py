"""Batched raycast: many views of uneven size, each into its own device
image, in persistent launches; direct launch, CUDA-graph replay and every
autotuned schedule produce the images of single-view raycasts bit for bit,
and those images are checked against the oracle.  A batch may span several
scenes (brick caches of different volumes) and drain them all in one
whole-tile launch; r3d_cuda_raycast_batch renders requests without a plan."""
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
def batch_scene(rb, orc, ctx, phantom256, scroll_tf):
    ctx.set_transfer(scroll_tf)
    ctx.set_alpha_cutoff(0.98)
    ctx.set_quality(0)
    ctx.set_schedule()
    ctx.bricks_build(phantom256, nlev=2)
    views = _views(rb, scroll_tf, ctx.brick_mode)
    refs, steps = [], 0
    for v in views:
        tot = np.zeros(1, np.uint64)
        refs.append(ctx.raycast(v, v.viewport[0], v.viewport[1], total=tot))
        steps += int(tot[0])
    # the single-view renders the batches are compared with equal the oracle
    page, pool = ctx.bricks_read()
    sc = orc.BrickScene(page, pool)
    for v, ref in zip(views, refs):
        want = orc.render(v, sc, scroll_tf, v.viewport[0], v.viewport[1])[0]
        assert np.abs(ref.astype(int) - want.astype(int)).max() <= 1
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
    for sc in [dict(persistent=0), dict(persistent=1, tile_shape=2, refill_min=24, unroll=2),
               dict(persistent=2), dict(persistent=2, blocks_per_sm=1)]:
        for im in imgs:
            im.zero_()
        b.set_schedule(**sc)
        b.launch(stream=ctx.stream)
        torch.cuda.synchronize()
        _check(imgs, refs)
    b.close()


def test_whole_tile_schedule(rb, ctx, batch_scene):
    """persistent = 2: whole 8x4 tiles from one queue, in one call of many
    views into one image and in a plan replayed from a graph (the kernel
    resets its own counters)."""
    import torch
    views, refs, steps = batch_scene
    imgs = _images(views)
    b = rb.Batch(ctx, views, imgs)
    b.set_schedule(persistent=2)
    tot = torch.zeros(1, dtype=torch.int64, device="cuda")
    b.capture(total=tot, stream=ctx.stream)
    for _ in range(3):
        b.replay(stream=ctx.stream)
    torch.cuda.synchronize()
    _check(imgs, refs)
    assert tot.item() == 4 * steps
    b.close()
    # r3d_cuda_raycast_fwd of several views into one image
    w, h = 200, 140
    vs = [v.copy() for v in views[:3]]
    for i, v in enumerate(vs):
        v.viewport[0], v.viewport[1] = 96, 64
        v.view_org = (100 * (i % 2)) | ((70 * (i // 2)) << 16)
    try:
        ctx.set_schedule(persistent=0)
        want = ctx.raycast(vs, w, h)
        ctx.set_schedule(persistent=2)
        got = ctx.raycast(vs, w, h)
        got2 = ctx.raycast(vs, w, h)
        # the automatic schedule (the default) takes whole tiles for these
        # three views and one grid for a call with one
        ctx.set_schedule()
        assert ctx.schedule()["persistent"] == 3
        auto = ctx.raycast(vs, w, h)
        one = [vs[0].copy()]
        one[0].view_org = 0
        one_grid = ctx.raycast(one, w, h)
        ctx.set_schedule(persistent=0)
        one_want = ctx.raycast(one, w, h)
    finally:
        ctx.set_schedule()
    assert np.array_equal(got, want) and np.array_equal(got2, want)
    assert np.array_equal(auto, want) and np.array_equal(one_grid, one_want)


def test_raycast_batch(rb, ctx, batch_scene):
    """r3d_cuda_raycast_batch under every schedule: the requests' images
    equal single-view renders, and the sample count matches."""
    import torch
    views, refs, steps = batch_scene
    try:
        for sc in (dict(), dict(persistent=0), dict(persistent=1), dict(persistent=2)):
            ctx.set_schedule(**sc)
            imgs = _images(views)
            tot = torch.zeros(1, dtype=torch.int64, device="cuda")
            ctx.raycast_batch(views, imgs, total=tot, stream=ctx.stream)
            torch.cuda.synchronize()
            _check(imgs, refs)
            assert tot.item() == steps
    finally:
        ctx.set_schedule()


def test_batch_over_two_scenes(rb, orc, ctx, batch_scene, scroll_tf):
    """Requests over two brick caches (the module's 256^3 cache and a
    160 x 120 x 48 slab cache with its own TF) drain in one whole-tile
    launch per path and mode; each image equals the oracle's render of its
    own scene."""
    import torch
    views, refs, _ = batch_scene
    c2 = rb.Context(0)
    try:
        lut2 = rb.tf_preset(1)
        c2.set_transfer(lut2)
        slab = rb.phantom((160, 120, 48), seed=5)
        c2.bricks_build(slab, nlev=2)
        page, pool = c2.bricks_read()
        sc2 = orc.BrickScene(page, pool)
        extra = []
        for i in range(4):
            p = rb.camera_view(0.5 + i, -0.3, 1.4, 80 + 16 * i, 60, lut2, step_voxels=0.5,
                               target=(0.5, 0.375, 0.15), frame_index=i)
            p.brick_mode = c2.brick_mode
            extra.append(p)
        allv = views + extra
        scenes = [None] * len(views) + [c2] * len(extra)
        imgs = _images(allv)
        b = rb.Batch(ctx, allv, imgs, scenes=scenes)
        assert b.schedule()["persistent"] == 2
        with pytest.raises(rb.R3DError):
            b.set_schedule(persistent=1)  # lane refill drains one scene
        tot = torch.zeros(1, dtype=torch.int64, device="cuda")
        b.capture(total=tot, stream=ctx.stream)
        torch.cuda.synchronize()
        _check(imgs[:len(views)], refs)
        for v, im in zip(extra, imgs[len(views):]):
            want = orc.render(v, sc2, lut2, v.viewport[0], v.viewport[1])[0]
            assert np.abs(im.cpu().numpy().astype(int) - want.astype(int)).max() <= 1
        got = [im.clone() for im in imgs]
        best, _ = b.autotune(reps=1)
        assert best["persistent"] in (0, 2)
        b.set_schedule(persistent=0)
        for im in imgs:
            im.zero_()
        b.launch(stream=ctx.stream)
        torch.cuda.synchronize()
        for a, g in zip(imgs, got):
            assert torch.equal(a, g)
        b.close()
    finally:
        c2.close()
