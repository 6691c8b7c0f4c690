"""XY clipmap on the GPU against the CPU oracle: the device-filled ring
layers of all six levels bit for bit, views whose footprints pick level 0,
levels 2-3, level 5 and the level 0 -> 1 fallback at level 0's coverage
edge, in every mode, single and batched (persistent launch); then focus moves
that recentre levels and window moves through the z rings.  Images within
1/255 per channel, step counts and MIP indices identical."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NX, NY, NZ, DEPTH = 2600, 256, 40, 8


def _cmp(a, b, what, tol=1):
    d = np.abs(a.astype(np.int32) - b.astype(np.int32))
    assert d.max() <= tol, f"{what}: max diff {d.max()} at {np.unravel_index(d.argmax(), d.shape)}"


@pytest.fixture(scope="module")
def clip(rb, scroll_tf):
    vol = rb.phantom((NX, NY, NZ), seed=43)
    c = rb.Context(0)
    c.set_transfer(scroll_tf)
    c.set_alpha_cutoff(0.98)
    c.clip_build(vol, DEPTH)
    yield c, vol
    c.close()


def _views(rb, c, lut, mode):
    ext = (1.0, NY / NX, DEPTH / NX)
    ctr = (0.5, 0.5 * ext[1], 0.5 * ext[2])
    # the oracle's level usage of these views at focus (1500, 128), z0 5:
    # far -> level 5, mid -> levels 2 and 3, near -> level 0, edge -> levels
    # 0 and 1 (its rays leave level 0's coverage, which starts at x = 464)
    vs = [rb.camera_view(0.0, 0.02, 0.7, 256, 64, lut, target=ctr, step_voxels=0.5,
                         lod_bias=0.5, mode=mode),
          rb.camera_view(0.1, -0.1, 0.25, 384, 128, lut, target=(0.6, ctr[1], ctr[2]),
                         step_voxels=0.5, mode=mode),
          rb.camera_view(-0.2, 0.3, 0.03, 256, 256, lut, target=(0.43, ctr[1], ctr[2]),
                         step_voxels=0.5, mode=mode),
          rb.camera_view(0.3, 0.1, 0.05, 256, 192, lut, target=(0.18, ctr[1], ctr[2]),
                         step_voxels=0.5, mode=mode)]
    for p in vs:
        c.clip_params(p)
        p.density = 6.0  # a thin window needs more opacity per sample to show
    return vs


def _check_levels(c, sc, levels=range(6)):
    for l in levels:
        for k in range(sc.tex[l].shape[0]):
            assert np.array_equal(c.clip_read(l, k), sc.tex[l][k]), (l, k)


def test_clip_levels_bit_exact(orc, clip):
    c, vol = clip
    c.clip_frame(1500.0, 128.0, 5)
    sc = orc.ClipScene(vol, DEPTH, orc.clip_origins(NX, NY, 1500.0, 128.0), 5)
    _check_levels(c, sc)


@pytest.mark.parametrize("mode", [0, 1, 2, 3, 5])
def test_clip_views(rb, orc, clip, scroll_tf, mode):
    c, vol = clip
    c.clip_frame(1500.0, 128.0, 5)
    sc = orc.ClipScene(vol, DEPTH, orc.clip_origins(NX, NY, 1500.0, 128.0), 5)
    for i, p in enumerate(_views(rb, c, scroll_tf, mode)):
        w, h = p.viewport[0], p.viewport[1]
        steps = np.zeros((h, w), np.uint32)
        mipi = np.zeros((h, w), np.uint32)
        got = c.raycast(p, w, h, steps=steps, mip_index=mipi)
        ref, rs, rm, _, st = orc.render(p, sc, scroll_tf, w, h)
        assert st == 0
        _cmp(got, ref, f"view {i} mode {mode}")
        assert np.array_equal(steps, rs) and np.array_equal(mipi, rm), f"view {i}"
        if mode == 0:
            assert got[..., :3].astype(int).std() > 2, f"view {i} is blank"


def test_clip_batch(rb, clip, scroll_tf):
    import torch
    c, _ = clip
    c.clip_frame(1500.0, 128.0, 5)
    views = _views(rb, c, scroll_tf, 0) + _views(rb, c, scroll_tf, 1)[:2]
    refs = [c.raycast(v, v.viewport[0], v.viewport[1]) for v in views]
    imgs = [torch.zeros((v.viewport[1], v.viewport[0], 4), dtype=torch.uint8, device="cuda")
            for v in views]
    b = rb.Batch(c, views, imgs)
    for sc in [dict(persistent=1), dict(persistent=0)]:
        for im in imgs:
            im.zero_()
        b.set_schedule(**sc)
        b.launch(stream=c.stream)
        torch.cuda.synchronize()
        for im, ref in zip(imgs, refs):
            assert np.array_equal(im.cpu().numpy(), ref), sc
    b.close()


def test_clip_focus_and_window_moves(rb, orc, clip, scroll_tf):
    c, vol = clip
    c.clip_frame(1500.0, 128.0, 5)
    prev = orc.clip_origins(NX, NY, 1500.0, 128.0)
    # a z scroll inside the rings, a focus move that recentres level 0, a
    # jump to the far end of the volume, and back past the start
    for fx, fy, z0 in ((1500.0, 128.0, 9), (600.0, 100.0, 9), (600.0, 100.0, 30),
                       (2000.0, 20.0, 0)):
        c.clip_frame(fx, fy, z0)
        origins = orc.clip_origins(NX, NY, fx, fy, prev=prev)
        prev = origins
        sc = orc.ClipScene(vol, DEPTH, origins, z0)
        _check_levels(c, sc, levels=(0, 1, 5))
        p = rb.FrameParams()
        c.clip_params(p)
        assert [tuple(p.clip_orig[l]) for l in range(6)] == [tuple(map(float, o)) for o in origins]
        for p in _views(rb, c, scroll_tf, 0)[1:]:
            w, h = p.viewport[0], p.viewport[1]
            ref = orc.render(p, sc, scroll_tf, w, h)[0]
            _cmp(c.raycast(p, w, h), ref, f"focus {fx} z0 {z0}")


def test_clip_view_validation(rb, clip, scroll_tf):
    c, _ = clip
    c.clip_frame(1500.0, 128.0, 5)
    p = _views(rb, c, scroll_tf, 0)[0]
    p.slab_z0 += 1  # not the loaded window
    with pytest.raises(rb.R3DError):
        c.raycast(p, 32, 32)
    c.clip_params(p)
    p.clip_orig[0][0] += 16  # not the loaded level origins
    with pytest.raises(rb.R3DError):
        c.raycast(p, 32, 32)
    c.clip_params(p)
    p.slab_depth = DEPTH + 1  # deeper than the rings hold
    with pytest.raises(rb.R3DError):
        c.raycast(p, 32, 32)
    c.clip_params(p)
    p.overlay_flags = 1  # overlays live in the brick cache only
    with pytest.raises(rb.R3DError):
        c.raycast(p, 32, 32)
    with pytest.raises(rb.R3DError):
        c.clip_read(6, 0)
    fresh = rb.Context(0)
    try:
        p = _views(rb, c, scroll_tf, 0)[0]
        with pytest.raises(rb.R3DError):  # no clipmap loaded
            fresh.raycast(p, 32, 32)
    finally:
        fresh.close()
