"""Parity at the benchmark sizes: the 1024^3 four-level brick cache at
1920x1080 (FULL, MIP, HEATMAP; cutoff 0.99) on sampled rays and on eight
whole frames spread over the bench orbit, and a 2048^3 sparse cache (bricks
with maximum <= 40 left out) at 3840x2160 with LOD bias 0 and 1 on sampled
rays.  Colours (within 1/255), step counts and MIP indices must equal the
oracle's; properties of whole frames are checked beside them."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _sample_xy(w, h, n, seed):
    rng = np.random.default_rng(seed)
    return np.stack([rng.integers(0, w, n), rng.integers(0, h, n)], axis=1).astype(np.uint32)


def _check_frame(rb, orc, ctx, sc, lut, p, w, h, cutoff, n=6000):
    steps = np.zeros((h, w), np.uint32)
    mipi = np.zeros((h, w), np.uint32)
    img = ctx.raycast(p, w, h, steps=steps, mip_index=mipi)
    xy = _sample_xy(w, h, n, p.frame_index + 7)
    rgba, rs, rm = orc.render_pixels(p, sc, lut, xy, cutoff=cutoff)
    got = img[xy[:, 1], xy[:, 0]]
    assert np.abs(got.astype(int) - rgba.astype(int)).max() <= 1
    assert np.array_equal(steps[xy[:, 1], xy[:, 0]], rs)
    if p.mode == rb.MODE_MIP:
        assert np.array_equal(mipi[xy[:, 1], xy[:, 0]], rm)
    return img, steps


@pytest.fixture(scope="module")
def cache1024(rb, orc, ctx):
    import torch
    vol = ctx.phantom(1024, seed=1234)
    ctx.bricks_build(vol, nlev=4)
    del vol
    torch.cuda.empty_cache()
    page, pool = ctx.bricks_read()
    return orc.BrickScene(page, pool)


@pytest.mark.parametrize("mode", [0, 1, 3])
def test_1024_1080p(rb, orc, ctx, cache1024, scroll_tf, mode):
    ctx.set_transfer(scroll_tf)
    ctx.set_alpha_cutoff(0.99)
    ctx.set_quality(0)
    try:
        for fi, ph in enumerate([0.1, 0.55]):
            p = rb.orbit_view(ph, 1920, 1080, scroll_tf, step_voxels=0.5, mode=mode,
                              frame_index=fi)
            p.brick_mode = ctx.brick_mode
            img, steps = _check_frame(rb, orc, ctx, cache1024, scroll_tf, p, 1920, 1080, 0.99)
            assert np.all(img[..., 3] == 255)
            assert steps.max() <= (192 if mode == 0 else 256)  # bricks-LOD budgets
    finally:
        ctx.set_alpha_cutoff(0.98)


@pytest.mark.parametrize("mode", [0, 1, 3])
def test_1024_1080p_whole_frames(rb, orc, ctx, cache1024, scroll_tf, mode):
    """Eight whole 1920x1080 frames spread over the 120-frame bench orbit
    (phases 0, 15, ..., 105 of 120, frame_index = phase), cutoff 0.99: every
    pixel within 1/255 of the oracle, every step count equal, and in MIP
    mode every MIP index equal."""
    ctx.set_transfer(scroll_tf)
    ctx.set_alpha_cutoff(0.99)
    ctx.set_quality(0)
    w, h = 1920, 1080
    try:
        for i in range(0, 120, 15):
            p = rb.orbit_view(i / 120.0, w, h, scroll_tf, step_voxels=0.5, mode=mode,
                              frame_index=i)
            p.brick_mode = ctx.brick_mode
            steps = np.zeros((h, w), np.uint32)
            mipi = np.zeros((h, w), np.uint32)
            img = ctx.raycast(p, w, h, steps=steps, mip_index=mipi)
            ref, rsteps, rmip, _, st = orc.render(p, cache1024, scroll_tf, w, h, cutoff=0.99)
            assert st == 0
            d = np.abs(img.astype(int) - ref.astype(int)).max()
            assert d <= 1, f"phase {i}/120 mode {mode}: {d} LSB"
            assert np.array_equal(steps, rsteps), f"phase {i}/120 mode {mode}: step counts"
            if mode == rb.MODE_MIP:
                assert np.array_equal(mipi, rmip), f"phase {i}/120: MIP indices"
    finally:
        ctx.set_alpha_cutoff(0.98)


def test_2048_sparse_4k(rb, orc, ctx, scroll_tf):
    import torch
    vol = ctx.phantom(2048, seed=99)
    ctx.bricks_build(vol, nlev=4, min_max=41)
    del vol
    torch.cuda.empty_cache()
    info = ctx.bricks_info()
    page, pool = ctx.bricks_read()
    sc = orc.BrickScene(page, pool)
    total = sum(((2048 >> l) // 128) ** 3 for l in range(4))
    assert 0 < info["nslots"] <= total
    ent = page[64:]
    res = ent != 0xFFFFFFFF
    assert res.sum() == info["nslots"] and np.all((ent[res] >> 24) >= 41)
    ctx.set_transfer(scroll_tf)
    ctx.set_alpha_cutoff(0.99)
    try:
        for bias in (0.0, 1.0):
            p = rb.orbit_view(0.3, 3840, 2160, scroll_tf, step_voxels=0.5, lod_bias=bias,
                              frame_index=int(bias))
            p.brick_mode = ctx.brick_mode
            _check_frame(rb, orc, ctx, sc, scroll_tf, p, 3840, 2160, 0.99, n=4000)
    finally:
        ctx.set_alpha_cutoff(0.98)
    assert ctx.status() == 0


def test_sparse_residency_full_frame(rb, orc, ctx, scroll_tf):
    """Many bricks absent (a dimmed half of the volume stays below the
    residency gate): the page walk falls back to coarser levels or skips,
    identically on both sides (whole frames)."""
    vol = rb.phantom(512, seed=31)
    vol[:, :, 256:] //= 8  # <= 31 < 41
    ctx.bricks_build(vol, nlev=3, min_max=41)
    page, pool = ctx.bricks_read()
    sc = orc.BrickScene(page, pool)
    assert (page[64:] == 0xFFFFFFFF).mean() > 0.3
    ctx.set_transfer(scroll_tf)
    for mode in (0, 1, 3):
        p = rb.camera_view(2.2, -0.4, 1.6, 240, 160, scroll_tf, step_voxels=0.5, mode=mode)
        p.brick_mode = ctx.brick_mode
        steps = np.zeros((160, 240), np.uint32)
        got = ctx.raycast(p, 240, 160, steps=steps)
        ref, rsteps, _, _, st = orc.render(p, sc, scroll_tf, 240, 160)
        assert st == 0
        assert np.abs(got.astype(int) - ref.astype(int)).max() <= 1
        assert np.array_equal(steps, rsteps)
