"""The post-decode display filter on the GPU against the oracle's
restatement of src/shaders/postfilt.comp: every primary filter and the
unsharp pass, alone and after a median, bit for bit on the slots of a
resident build (page table unchanged, renders matching the oracle over the
filtered slots); streamed uploads and refilter (the coarsest level keeps
the filter it was uploaded with); overlay targets, the caller's device
buffer left untouched; the render-level calls."""
import numpy as np
import pytest

from conftest import elev35

pytestmark = pytest.mark.gpu

ABSENT = 0xFFFFFFFF


def _cmp(a, b, what, tol=1):
    d = np.abs(a.astype(np.int32) - b.astype(np.int32))
    assert d.max() <= tol, f"{what}: max diff {d.max()} at {np.unravel_index(d.argmax(), d.shape)}"


@pytest.fixture(scope="module")
def noisy(rb):
    vol = rb.phantom(256, seed=41)
    rng = np.random.default_rng(41)
    v = vol.astype(np.int16) + rng.integers(-24, 25, vol.shape)
    v[rng.random(vol.shape) < 0.004] = 255
    return np.clip(v, 0, 255).astype(np.uint8)


@pytest.fixture(scope="module")
def plain(rb, noisy):
    c = rb.Context(0)
    try:
        c.bricks_build(noisy, 2)
        page, pool = c.bricks_read()
    finally:
        c.close()
    return page, pool.reshape(-1, 128, 128, 128)


MODES = [(1, 0.0), (2, 0.0), (3, 0.0), (4, 0.0), (0x100, 1.5), (0x101, 0.8), (0x104, 2.0)]


@pytest.mark.parametrize("mode,amount", MODES)
def test_resident_build_bit_exact(rb, orc, noisy, plain, scroll_tf, mode, amount):
    page0, pool0 = plain
    c = rb.Context(0)
    try:
        c.set_transfer(scroll_tf)
        c.set_alpha_cutoff(0.98)
        c.bricks_postfilter(mode, amount)
        c.bricks_build(noisy, 2)
        page, pool = c.bricks_read()
        assert np.array_equal(page, page0)  # page maxima: the bricks as built
        got = pool.reshape(-1, 128, 128, 128)
        ks = [0, 3, got.shape[0] - 1]  # level 0 bricks and the coarsest
        want = orc.postfilter(pool0[ks], mode, amount)
        for i, k in enumerate(ks):
            assert np.array_equal(got[k], want[i]), f"slot {k}: {np.argwhere(got[k] != want[i])[:5]}"
        assert not np.array_equal(got[ks[0]], pool0[ks[0]])
        p = elev35(rb, scroll_tf, 256, 192, step_voxels=0.5)
        p.brick_mode = c.brick_mode
        ref, _, _, _, st = orc.render(p, orc.BrickScene(page, pool), scroll_tf, 256, 192)
        _cmp(c.raycast(p, 256, 192), ref, f"mode {mode:#x}")
    finally:
        c.close()


def test_unknown_modes_change_nothing(rb, noisy, plain):
    c = rb.Context(0)
    try:
        c.bricks_postfilter(7, 1.0)  # no primary id, no unsharp bit
        c.bricks_build(noisy, 2)
        assert np.array_equal(c.bricks_read()[1].reshape(plain[1].shape), plain[1])
        with pytest.raises(rb.R3DError):
            c.bricks_refilter()  # a resident cache
        with pytest.raises(rb.R3DError):
            c.bricks_postfilter(1, float("nan"))
    finally:
        c.close()


def test_stream_and_refilter(rb, orc, noisy, plain, scroll_tf):
    page0, pool0 = plain

    def resident(c):
        page, pool = c.bricks_read()
        pool = pool.reshape(-1, 128, 128, 128)
        return {b: pool[int(page[b]) & 0xFFFFFF] for b in range(64, page.size) if page[b] != ABSENT}

    coarse = int(page0[8])  # the coarsest level's one brick (page word)
    c = rb.Context(0)
    try:
        c.bricks_postfilter(1)  # before begin: the pinned coarsest level is filtered too
        c.stream_begin(noisy, 2, 6)
        for yaw in (0.3, 1.4):  # close enough for level 0 bricks
            p = rb.camera_view(yaw, -0.4, 1.2, 960, 720, scroll_tf, step_voxels=0.5)
            c.stream_update(p, 4)
        res = resident(c)
        assert coarse in res and len(res) >= 4
        keys = sorted(res)
        want = orc.postfilter(np.stack([pool0[int(page0[b]) & 0xFFFFFF] for b in keys]), 1)
        for i, b in enumerate(keys):
            assert np.array_equal(res[b], want[i]), b
        c.bricks_postfilter(0x104, 1.25)
        c.bricks_refilter()
        res2 = resident(c)
        assert sorted(res2) == keys
        want2 = orc.postfilter(np.stack([pool0[int(page0[b]) & 0xFFFFFF] for b in keys]), 0x104, 1.25)
        for i, b in enumerate(keys):
            assert np.array_equal(res2[b], want[i] if b == coarse else want2[i]), b
    finally:
        c.close()


def test_overlay_targets(rb, orc, noisy, plain):
    ink = np.roll(noisy, 9, axis=1)
    c = rb.Context(0)
    try:
        c.bricks_build(noisy, 2)
        c.overlay_build(0, ink)
        o0 = c.overlay_read(0)
        c.bricks_postfilter(3, 0.0, targets=2)  # max of 3^3 on the ink atlas only
        c.overlay_build(0, ink)
        want = orc.postfilter(o0, 3)
        assert np.array_equal(c.overlay_read(0), want)
        c.overlay_build(1, ink)
        assert np.array_equal(c.overlay_read(1), o0)  # 3D ink not targeted
        c.overlay_load(0, o0)  # host slots
        assert np.array_equal(c.overlay_read(0), want)
        c.bricks_postfilter(2, 0.0, targets=4)  # median of 5^3 on 3D ink
        import torch
        dev = torch.from_numpy(o0).cuda()
        c.overlay_load(1, dev)  # the caller's device buffer stays as it was
        assert np.array_equal(c.overlay_read(1), orc.postfilter(o0, 2))
        assert np.array_equal(dev.cpu().numpy(), o0)
        assert np.array_equal(c.bricks_read()[1].reshape(plain[1].shape), plain[1])  # CT untouched
    finally:
        c.close()


def test_render_level_calls(rb, noisy, scroll_tf):
    r = rb.Renderer(256, 192)
    c = rb.Context(0)
    try:
        for x in (r, c):
            x.set_transfer(scroll_tf)
            x.set_alpha_cutoff(0.98)
            x.bricks_postfilter(0x101, 1.0, 1)
        r.bricks_begin_volume(noisy, 2)
        c.bricks_build(noisy, 2)
        p = elev35(rb, scroll_tf, 256, 192, step_voxels=0.5)
        r.bricks_params(p)
        r.frame(p)
        assert np.array_equal(r.read_frame(), c.raycast(p, 256, 192))
        r.bricks_refilter()  # resident: a no-op
    finally:
        c.close()
        r.close()


@pytest.mark.parametrize("mode", [4, 0x101])
@pytest.mark.parametrize("slot_of", [None, [3, ABSENT, 5, 1, 0, 7, 2, 6]])
def test_shard_atlas(rb, orc, noisy, scroll_tf, mode, slot_of):
    """A single-level shard atlas filters its placed slots before the mips
    and the occupancy derived from them; page maxima stay the bricks'."""
    c = rb.Context(0)
    try:
        c.set_transfer(scroll_tf)
        c.set_alpha_cutoff(0.98)
        c.shard_build(noisy, 2, slot_of)
        page0, a0 = c.shard_read(0)
        c.bricks_postfilter(mode, 1.0)
        c.shard_build(noisy, 2, slot_of)
        want0 = a0.copy()
        used = range(8) if slot_of is None else [s for s in slot_of if s != ABSENT]
        for s in used:
            sx, sy, sz = (s % 2) * 128, ((s // 2) % 2) * 128, (s // 4) * 128
            box = (slice(sz, sz + 128), slice(sy, sy + 128), slice(sx, sx + 128))
            want0[box] = orc.postfilter(a0[box], mode, 1.0)[0]
        assert not np.array_equal(want0, a0)
        sc = orc.ShardScene(page0, want0, 2, 2)
        for m in range(4):
            page, lv = c.shard_read(m)
            assert np.array_equal(page, page0)
            assert np.array_equal(lv, sc.levels[m]), f"mip {m}"
        assert np.array_equal(c.shard_read(-1)[1], sc.occ)
        p = elev35(rb, scroll_tf, 256, 192, step_voxels=0.5)
        p.brick_mode = c.shard_mode
        ref = orc.render(p, sc, scroll_tf, 256, 192)[0]
        _cmp(c.raycast(p, 256, 192), ref, f"shard mode {mode:#x}")
    finally:
        c.close()


def test_targets_together(rb, orc, noisy, plain):
    """Targets 1 | 2: the CT bricks and the ink atlas both filtered; the
    3D ink atlas not."""
    ink = np.roll(noisy, 5, axis=0)
    c = rb.Context(0)
    try:
        c.bricks_build(noisy, 2)
        c.overlay_build(0, ink)
        o0 = c.overlay_read(0)
        c.bricks_postfilter(3, 0.0, targets=3)
        c.bricks_build(noisy, 2)
        c.overlay_build(0, ink)
        c.overlay_build(1, ink)
        assert np.array_equal(c.bricks_read()[1].reshape(plain[1].shape), orc.postfilter(plain[1], 3))
        assert np.array_equal(c.overlay_read(0), orc.postfilter(o0, 3))
        assert np.array_equal(c.overlay_read(1), o0)
    finally:
        c.close()
