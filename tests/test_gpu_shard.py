"""Single-level brick atlas on the GPU against the CPU oracle: the device
builders (atlas, mips, world occupancy, page table) bit for bit, and views
through the identity layout, a shuffled layout with absent bricks and an
atlas smaller than the shard, in every mode and schedule.  Images within
1/255 per channel, heatmap step counts and MIP indices identical."""
import numpy as np
import pytest

from conftest import elev35

pytestmark = pytest.mark.gpu

ABSENT = 0xFFFFFFFF
LAYOUTS = {
    "identity": (2, None),
    "shuffled": (2, np.array([5, ABSENT, 2, 7, 0, ABSENT, 1, 3], np.uint32)),
    "small_atlas": (1, np.array([ABSENT, ABSENT, ABSENT, 0, ABSENT, ABSENT, ABSENT, ABSENT],
                                np.uint32)),
}


def _cmp(a, b, what, tol=1):
    d = np.abs(a.astype(np.int32) - b.astype(np.int32))
    assert d.max() <= tol, f"{what}: max diff {d.max()} at {np.unravel_index(d.argmax(), d.shape)}"


@pytest.fixture(scope="module")
def vol256(rb):
    return rb.phantom(256, seed=77)


@pytest.fixture(scope="module", params=list(LAYOUTS))
def shard(request, rb, orc, vol256, scroll_tf):
    abpa, slot_of = LAYOUTS[request.param]
    c = rb.Context(0)
    c.set_transfer(scroll_tf)
    c.set_alpha_cutoff(0.98)
    c.shard_build(vol256, abpa, slot_of)
    sc = orc.ShardScene.build(vol256, abpa, slot_of)
    yield request.param, c, sc
    c.close()


def test_shard_builders_bit_exact(shard):
    name, c, sc = shard
    assert c.shard_mode == sc.brick_mode, name
    for m in range(4):
        page, lv = c.shard_read(m)
        assert np.array_equal(page, sc.page)
        assert np.array_equal(lv, sc.levels[m]), f"{name}: mip {m}"
    assert np.array_equal(c.shard_read(-1)[1], sc.occ), f"{name}: occupancy"


SCHED = {"grid": dict(persistent=0), "persist": dict(persistent=1, refill_min=8)}


@pytest.mark.parametrize("sched", list(SCHED))
@pytest.mark.parametrize("mode", [0, 1, 2, 3, 5])
def test_shard_modes(rb, orc, shard, scroll_tf, mode, sched):
    name, c, sc = shard
    c.set_schedule(**SCHED[sched])
    try:
        p = elev35(rb, scroll_tf, 256, 256, step_voxels=0.5, mode=mode)
        p.brick_mode = c.shard_mode
        steps = np.zeros((256, 256), np.uint32)
        mipi = np.zeros((256, 256), np.uint32)
        got = c.raycast(p, 256, 256, steps=steps, mip_index=mipi)
        ref, rs, rm, _, st = orc.render(p, sc, scroll_tf, 256, 256)
        assert st == 0 and c.status() == 0
        _cmp(got, ref, f"{name} mode {mode}")
        assert np.array_equal(steps, rs), f"{name}: steps differ at {np.argwhere(steps != rs)[:4]}"
        assert np.array_equal(mipi, rm), f"{name}: MIP indices differ"
    finally:
        c.set_schedule()


@pytest.mark.parametrize("case", ["fast", "bias", "ortho", "rot", "near", "lowcut"])
def test_shard_view_variants(rb, orc, shard, scroll_tf, case):
    name, c, sc = shard
    kw = dict(step_voxels=0.5)
    dist = 2.0
    if case == "bias":
        kw["lod_bias"] = 1.0
    if case == "near":
        dist = 0.9
    p = rb.camera_view(0.9, -0.4, dist, 256, 192, scroll_tf, **kw)
    if case == "ortho":
        p.view_flags |= rb.VIEW_ORTHO
    if case == "rot":
        rb.set_rotation(p, 0.3, -0.2, 0.5)
    if case == "lowcut":
        p.threshold = 90 / 255
    p.brick_mode = c.shard_mode
    c.set_quality(1 if case == "fast" else 0)
    try:
        got = c.raycast(p, 256, 192)
        ref, _, _, _, st = orc.render(p, sc, scroll_tf, 256, 192, quality=1 if case == "fast" else 0)
    finally:
        c.set_quality(0)
    assert st == 0
    _cmp(got, ref, f"{name} {case}")


def test_identity_shard_matches_cube_path(rb, vol256, scroll_tf):
    """Identity layout vs the cube path at max_mip = 3 (same texture data,
    same gates once the skip gate exceeds 4.5/255): identical images."""
    c = rb.Context(0)
    try:
        c.set_transfer(scroll_tf)
        c.upload_volume(vol256)
        c.shard_build(vol256)
        for mode in (0, 1, 3):
            p = elev35(rb, scroll_tf, 256, 256, step_voxels=0.5, max_mip=3.0, mode=mode)
            cube = c.raycast(p, 256, 256)
            p.brick_mode = c.shard_mode
            assert np.array_equal(c.raycast(p, 256, 256), cube), f"mode {mode}"
    finally:
        c.close()


def test_shard_errors(rb, vol256, scroll_tf):
    c = rb.Context(0)
    try:
        p = elev35(rb, scroll_tf, 32, 32)
        p.brick_mode = 2 | (2 << 8)
        with pytest.raises(rb.R3DError):
            c.raycast(p, 32, 32)  # no atlas loaded
        assert rb.lib.r3d_cuda_shard_build(c.h, 200, vol256.ctypes.data, 1, None) == -1  # R3D_E_INVALID
        with pytest.raises(rb.R3DError):
            c.shard_build(vol256, 1)  # abpa < bpa needs slot_of
        with pytest.raises(rb.R3DError):
            c.shard_build(vol256, 2, np.array([0, 0, 1, 2, 3, 4, 5, 6], np.uint32))  # shared slot
        c.shard_build(vol256)
        p.brick_mode = 2 | (2 << 8)  # identity bit missing
        with pytest.raises(rb.R3DError):
            c.raycast(p, 32, 32)
    finally:
        c.close()


def test_renderer_bricks_begin_shard(rb, orc, vol256, scroll_tf):
    """render.h path: r3d_bricks_begin_shard + r3d_bricks_params + r3d_frame
    + r3d_read_frame equal the oracle's identity-layout render."""
    r = rb.Renderer(256, 256)
    try:
        r.set_transfer(scroll_tf)
        r.bricks_begin_shard(vol256)
        p = elev35(rb, scroll_tf, 256, 256, step_voxels=0.5)
        r.bricks_params(p)
        assert p.brick_mode == 2 | (2 << 8) | 0x10000
        r.frame(p)
        got = r.read_frame()
        ref = orc.render(p, orc.ShardScene.build(vol256), scroll_tf, 256, 256)[0]
        _cmp(got, ref, "renderer shard")
        with pytest.raises(Exception):
            r.bricks_begin_shard(vol256, pool_bpa=1)  # streaming residency: not available
    finally:
        r.close()
