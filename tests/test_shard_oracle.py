"""The oracle's single-level brick atlas (render3d's bricks mode without the
LOD flag): builders and march, on the CPU.

With every brick in its own slot, the atlas is the volume itself.  Its mips
and occupancy grid then equal the cube's, and a view of it renders exactly
like the cube path with max_mip = 3 once the skip gate reaches the bricks
floor of 4.5/255 (src/shaders/raycast.slang:659-661,800-805,829-860)."""
import numpy as np
import pytest

from conftest import elev35


@pytest.fixture(scope="module")
def vol256(rb):
    return rb.phantom(256, seed=77)


def _brick(vol, b, bpa=2):
    bx, by, bz = b % bpa, (b // bpa) % bpa, b // (bpa * bpa)
    return vol[bz * 128:(bz + 1) * 128, by * 128:(by + 1) * 128, bx * 128:(bx + 1) * 128]


def test_identity_atlas_is_the_cube(orc, vol256):
    sh = orc.ShardScene.build(vol256)
    cube = orc.CubeScene(vol256)
    assert sh.identity and sh.brick_mode == 2 | (2 << 8) | 0x10000
    for m in range(4):
        assert np.array_equal(sh.levels[m], cube.levels[m]), f"mip {m}"
    assert np.array_equal(sh.occ, cube.occ)
    for b in range(8):
        assert sh.page[b] == b | (int(_brick(vol256, b).max()) << 24)


def test_permuted_atlas_places_bricks(orc, vol256):
    slot_of = np.array([5, 0xFFFFFFFF, 2, 7, 0, 0xFFFFFFFF, 1, 3], np.uint32)
    sh = orc.ShardScene.build(vol256, 2, slot_of)
    assert not sh.identity and sh.brick_mode == 2 | (2 << 8)
    a = sh.levels[0]
    used = set()
    for b, s in enumerate(slot_of):
        if s == 0xFFFFFFFF:
            assert sh.page[b] == 0xFFFFFFFF
            continue
        used.add(int(s))
        sx, sy, sz = s % 2, (s // 2) % 2, s // 4
        got = a[sz * 128:(sz + 1) * 128, sy * 128:(sy + 1) * 128, sx * 128:(sx + 1) * 128]
        assert np.array_equal(got, _brick(vol256, b)), f"brick {b} in slot {s}"
        assert sh.page[b] == s | (int(got.max()) << 24)
    for s in set(range(8)) - used:  # empty slots are zero
        sx, sy, sz = s % 2, (s // 2) % 2, s // 4
        assert not a[sz * 128:(sz + 1) * 128, sy * 128:(sy + 1) * 128, sx * 128:(sx + 1) * 128].any()
    # world occupancy: raw block maxima are 0 under absent bricks, so only
    # the 1-block dilation halo of resident neighbours can be nonzero there
    for b in (1, 5):
        bx, by, bz = b % 2, (b // 2) % 2, b // 4
        inner = sh.occ[bz * 16 + 1:bz * 16 + 15, by * 16 + 1:by * 16 + 15, bx * 16 + 1:bx * 16 + 15]
        assert not inner.any()


def test_identity_renders_like_the_cube(rb, orc, vol256, scroll_tf):
    sh = orc.ShardScene.build(vol256)
    cube = orc.CubeScene(vol256)
    for mode in (0, 1, 3):
        p = elev35(rb, scroll_tf, 160, 160, step_voxels=0.5, max_mip=3.0, mode=mode)
        assert p.skip_gate >= 4.5 / 255
        ref, rs, rm, _, _ = orc.render(p, cube, scroll_tf, 160, 160)
        p.brick_mode = sh.brick_mode
        got, gs, gm, _, st = orc.render(p, sh, scroll_tf, 160, 160)
        assert st == 0
        assert np.array_equal(got, ref), f"mode {mode}"
        assert np.array_equal(gs, rs) and np.array_equal(gm, rm)


def test_page_path_close_to_identity(rb, orc, vol256, scroll_tf):
    """Every brick resident but in shuffled slots: the page path clamps
    fetches inside each brick, so only brick seams may differ."""
    ident = orc.ShardScene.build(vol256)
    perm = orc.ShardScene.build(vol256, 2, np.array([3, 6, 0, 5, 7, 1, 4, 2], np.uint32))
    p = elev35(rb, scroll_tf, 160, 160, step_voxels=0.5, mode=0)
    p.brick_mode = ident.brick_mode
    a = orc.render(p, ident, scroll_tf, 160, 160)[0]
    p.brick_mode = perm.brick_mode
    b, _, _, _, st = orc.render(p, perm, scroll_tf, 160, 160)
    assert st == 0
    d = np.abs(a.astype(int) - b.astype(int))
    assert d.mean() < 1.0, d.mean()


def test_shard_view_validation(rb, orc, vol256, scroll_tf):
    sh = orc.ShardScene.build(vol256)
    p = elev35(rb, scroll_tf, 32, 32)
    p.brick_mode = 4 | (2 << 8)  # bpa does not match the atlas
    with pytest.raises(ValueError):
        orc.render(p, sh, scroll_tf, 32, 32)


def test_overlay_builder(orc, vol256):
    """Overlay slots cut from the CT volume itself are the CT slots; label
    slots at a coarse level stride-sample the level-0 grid."""
    sc = orc.BrickScene.build(vol256, 2, min_max=30)
    assert np.array_equal(sc.build_overlay(0, vol256), sc.pool)
    lab = (np.arange(256 ** 3, dtype=np.uint32).reshape(256, 256, 256) % 9).astype(np.uint8)
    pool = sc.build_overlay(2, lab).reshape(-1, 128, 128, 128)
    off1 = int(sc.page[4 + 4])  # level 1: a single 128^3 brick covering the volume
    e = int(sc.page[off1])
    if e != 0xFFFFFFFF:
        assert np.array_equal(pool[e & 0xFFFFFF], lab[::2, ::2, ::2])
    off0 = int(sc.page[4])
    for b in range(8):
        e = int(sc.page[off0 + b])
        if e == 0xFFFFFFFF:
            continue
        bx, by, bz = b % 2, (b // 2) % 2, b // 4
        assert np.array_equal(pool[e & 0xFFFFFF],
                              lab[bz * 128:(bz + 1) * 128, by * 128:(by + 1) * 128,
                                  bx * 128:(bx + 1) * 128])
