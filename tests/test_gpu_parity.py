"""Parity of the sm_100a kernels with the CPU oracle.

Images must agree within 1/255 per channel (the parity tolerance;
in practice they are identical), heatmap step counts and MIP indices must be
identical, and the device-side builders (mip chain, occupancy grid, LOD
brick pyramid and page table) must be bit-exact."""
import math
import os
import subprocess

import numpy as np
import pytest

from conftest import elev35

pytestmark = pytest.mark.gpu


def _cmp(a, b, what, tol=1):
    d = np.abs(a.astype(np.int32) - b.astype(np.int32))
    assert d.max() <= tol, f"{what}: max diff {d.max()} at {np.unravel_index(d.argmax(), d.shape)}"
    return d


def test_fmath_bits_match_cpu(ctx):
    rng = np.random.default_rng(7)
    x = np.concatenate([rng.uniform(0, 1, 20000), rng.uniform(1, 2048, 20000),
                        rng.uniform(-20, 20, 20000), np.array([0.0, 1.0, 2.0, 0.5, 1e-30,
                                                               1e-40, 128.0, -151.0])])
    x = x.astype(np.float32)
    y = rng.uniform(0.01, 20, x.size).astype(np.float32)
    dev = ctx.fmath_eval(x, y)
    import oracle
    cpu = oracle.fmath_eval(x, y)  # the CPU build of the same header
    # NaN payloads differ between CUDA and glibc; every other result is
    # compared bit for bit
    both_nan = np.isnan(dev) & np.isnan(cpu)
    diff = (dev.view(np.uint32) != cpu.view(np.uint32)) & ~both_nan
    assert not diff.any(), f"{diff.sum()} mismatching results, e.g. x={x[diff.any(1)][:4]}"


@pytest.fixture(scope="module")
def cube256(ctx, orc, phantom256, scroll_tf):
    ctx.upload_volume(phantom256)
    ctx.set_transfer(scroll_tf)
    ctx.set_quality(0)
    ctx.set_alpha_cutoff(0.98)
    return orc.CubeScene(phantom256)


def test_cube_builders_bit_exact(ctx, cube256):
    for m, lv in enumerate(cube256.levels):
        assert np.array_equal(ctx.cube_read(m), lv), f"mip level {m}"
    assert np.array_equal(ctx.cube_read(-1), cube256.occ)


SCHEDULES = {"grid": dict(persistent=0), "grid_shade8": dict(persistent=0, shade_group=8),
             "grid_shade32": dict(persistent=0, shade_group=32),
             "persist": dict(persistent=1, refill_min=8),
             "persist_16x2_u2": dict(persistent=1, refill_min=4, tile_shape=1, unroll=2),
             "persist_32x1": dict(persistent=1, refill_min=24, tile_shape=2, unroll=1)}


@pytest.fixture(params=list(SCHEDULES))
def sched(request, ctx):
    ctx.set_schedule(**SCHEDULES[request.param])
    yield request.param
    ctx.set_schedule()


@pytest.mark.parametrize("mode", [0, 1, 2, 3, 4, 5])
def test_cube_config0_modes(rb, orc, ctx, cube256, scroll_tf, mode, sched):
    p = elev35(rb, scroll_tf, step_voxels=0.5, max_mip=0.0, mode=mode)
    steps = np.zeros((512, 512), np.uint32)
    mipi = np.zeros((512, 512), np.uint32)
    got = ctx.raycast(p, 512, 512, steps=steps, mip_index=mipi)
    ref, rsteps, rmip, _, st = orc.render(p, cube256, scroll_tf, 512, 512)
    assert st == 0
    _cmp(got, ref, f"mode {mode} image")
    assert np.array_equal(steps, rsteps), f"steps differ at {np.argwhere(steps != rsteps)[:5]}"
    if mode == rb.MODE_MIP:
        assert np.array_equal(mipi, rmip)


def test_cube_fast_gradient(rb, orc, ctx, cube256, scroll_tf):
    ctx.set_quality(1)
    try:
        p = elev35(rb, scroll_tf, step_voxels=0.5, max_mip=0.0)
        got = ctx.raycast(p, 512, 512)
        ref = orc.render(p, cube256, scroll_tf, 512, 512, quality=1)[0]
        _cmp(got, ref, "4-tap")
    finally:
        ctx.set_quality(0)


@pytest.mark.parametrize("case", ["lod", "rot", "ortho", "half", "lowcut", "bias"])
def test_cube_view_variants(rb, orc, ctx, cube256, scroll_tf, case, sched):
    w, h = 320, 200
    p = rb.camera_view(1.1, -0.3, 1.2, w, h, scroll_tf, step_voxels=1.0, max_mip=10.0,
                       frame_index=3)
    if case == "rot":
        rb.set_rotation(p, 0.4, -0.3, 0.2, (0.05, -0.02, 0.1))
    elif case == "ortho":
        p.view_flags = rb.VIEW_ORTHO
        s = 0.7
        for a in range(3):
            p.cam_right[a] *= s / math.sqrt(sum(v * v for v in p.cam_right))
            p.cam_up[a] *= s / math.sqrt(sum(v * v for v in p.cam_up))
    elif case == "half":
        p.view_flags = rb.VIEW_HALF
    elif case == "lowcut":
        p.threshold = 90 / 255.0
        p.skip_gate = rb.skip_gate(90.0, scroll_tf)
    elif case == "bias":
        p.lod_bias = 1.5
    for mode in (0, 1, 3):
        p.mode = mode
        steps = np.zeros((h, w), np.uint32)
        got = ctx.raycast(p, w, h, steps=steps)
        ref, rsteps, _, _, _ = orc.render(p, cube256, scroll_tf, w, h)
        _cmp(got, ref, f"{case} mode {mode}")
        assert np.array_equal(steps, rsteps), f"{case} mode {mode} steps"


def test_multiview_rects(rb, orc, ctx, cube256, scroll_tf, sched):
    W, H = 400, 300
    views = []
    for i, (yaw, mode) in enumerate([(0.2, 0), (1.2, 1), (2.2, 3), (3.2, 5)]):
        p = rb.camera_view(yaw, -0.4, 2.0, 200, 150, scroll_tf, mode=mode)
        p.view_org = (200 * (i % 2)) | ((150 * (i // 2)) << 16)
        views.append(p)
    got = ctx.raycast(views, W, H)
    ref = np.zeros((H, W, 4), np.uint8)
    for p in views:
        orc.render(p, cube256, scroll_tf, W, H, img=ref)
    _cmp(got, ref, "multiview")


def test_unsupported_views_error(rb, ctx, cube256, scroll_tf):
    p = elev35(rb, scroll_tf, w=64, h=64)
    # slab, virtual-slab and clip views on a context holding none of them:
    # R3D_E_STATE; overlay atlases on a cube view: R3D_E_UNSUPPORTED
    for field, val, code in [("slab_grid", 1, -5), ("slab_grid", 1 << 24, -5),
                             ("clip_valid", 1, -5), ("overlay_flags", 1, -4)]:
        q = p.copy()
        setattr(q, field, val)
        with pytest.raises(rb.R3DError) as e:
            ctx.raycast(q, 64, 64)
        assert e.value.code == code, field
    q = p.copy()
    q.view_flags = rb.VIEW_SURF
    with pytest.raises(rb.R3DError):
        ctx.raycast(q, 64, 64)


def test_reference_conformance_test_gpu(rb):
    """The reference's own tests/test_gpu.c (built unmodified into
    oracle/_ref) driving r3d_headless: mean <= 2 LSB, max <= 64 LSB."""
    from oracle import REF_TEST_GPU
    if not os.path.exists(REF_TEST_GPU):
        pytest.skip("oracle/_ref/test_gpu not built (needs the reference tree at build time)")
    cli = os.path.join(os.path.dirname(rb.LIB_PATH), "r3d_headless")
    r = subprocess.run([REF_TEST_GPU, cli], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "test_gpu: ok" in r.stdout


# ------------------------------------------------------------------ bricks

def test_brick_builder_bit_exact(rb, orc, ctx):
    vol = rb.phantom((300, 260, 200), seed=99)
    ctx.bricks_build(vol, nlev=3, min_max=60)
    page, pool = ctx.bricks_read()
    ref = orc.BrickScene.build(vol, 3, min_max=60)
    assert np.array_equal(page, ref.page)
    assert np.array_equal(pool, ref.pool)


@pytest.fixture(scope="module")
def bricks256(ctx, orc, phantom256, scroll_tf):
    ctx.set_transfer(scroll_tf)
    ctx.bricks_build(phantom256, nlev=2)
    page, pool = ctx.bricks_read()
    return orc.BrickScene(page, pool)


@pytest.mark.parametrize("mode", [0, 1, 2, 3, 5])
def test_bricks_modes(rb, orc, ctx, bricks256, scroll_tf, mode, sched):
    w, h = 384, 256
    p = rb.camera_view(0.9, -0.5, 1.6, w, h, scroll_tf, step_voxels=0.5, mode=mode)
    p.brick_mode = ctx.brick_mode
    steps = np.zeros((h, w), np.uint32)
    mipi = np.zeros((h, w), np.uint32)
    got = ctx.raycast(p, w, h, steps=steps, mip_index=mipi)
    ref, rsteps, rmip, _, st = orc.render(p, bricks256, scroll_tf, w, h)
    assert st == 0
    _cmp(got, ref, f"bricks mode {mode}")
    assert np.array_equal(steps, rsteps)
    if mode == 1:
        assert np.array_equal(mipi, rmip)


@pytest.mark.parametrize("case", ["crop", "axis_slab", "oblique", "fast", "cutoff99"])
def test_bricks_clips(rb, orc, ctx, bricks256, scroll_tf, case, sched):
    w, h = 256, 192
    p = rb.camera_view(2.0, -0.2, 1.4, w, h, scroll_tf, step_voxels=0.5)
    p.brick_mode = ctx.brick_mode
    quality, cutoff = 0, 0.98
    if case == "crop":
        p.view_flags = rb.VIEW_CROP
        p.slab_x0, p.slab_y0, p.slab_z0 = 40.0, 60.0, 30.0
        p.slab_px, p.slab_py, p.slab_nx = 120.0, 100.0, 150.0
    elif case == "axis_slab":
        p.view_flags = rb.VIEW_AXIS(1)
        p.slab_z0, p.slab_depth = 100.0, 32
    elif case == "oblique":
        p.view_flags = rb.VIEW_OBLIQUE
        p.slab_z0, p.slab_depth = 300.0, 40
    elif case == "fast":
        quality = 1
    elif case == "cutoff99":
        cutoff = 0.99
    ctx.set_quality(quality)
    ctx.set_alpha_cutoff(cutoff)
    try:
        for mode in (0, 3):
            p.mode = mode
            steps = np.zeros((h, w), np.uint32)
            got = ctx.raycast(p, w, h, steps=steps)
            ref, rsteps, _, _, _ = orc.render(p, bricks256, scroll_tf, w, h, cutoff=cutoff,
                                              quality=quality)
            _cmp(got, ref, f"{case} mode {mode}")
            assert np.array_equal(steps, rsteps)
    finally:
        ctx.set_quality(0)
        ctx.set_alpha_cutoff(0.98)


# TFs and gates that move the fetch elision's byte counts to their edges:
# a TF with opacity from 0 (no clear prefix), one clear up to 250, a low
# cut (threshold) and a high skip gate
ELIDE_EDGES = {
    "opaque_from_0": ([(0, (10, 10, 10, 20)), (255, (255, 255, 255, 230))], 0.0, None),
    "clear_to_250": ([(0, (0, 0, 0, 0)), (250, (250, 250, 250, 0)), (255, (255, 255, 255, 255))],
                     0.0, None),
    "low_cut": (None, 90.0, None),
    "high_gate": (None, 0.0, 0.25),
}


@pytest.mark.parametrize("mode", [0, 1, 2, 3, 5])
@pytest.mark.parametrize("case", list(ELIDE_EDGES))
def test_bricks_elision_edges(rb, orc, ctx, bricks256, scroll_tf, case, mode):
    """The elision decides on the byte of a block maximum (and on a fetched
    sample's own eight bytes) against per-view counts; at the counts' edges
    the images, step counts and MIP indices still equal the oracle's."""
    pts, low_cut, gate = ELIDE_EDGES[case]
    lut = rb.tf_build(pts) if pts else scroll_tf
    w, h = 256, 192
    p = rb.camera_view(1.3, -0.4, 1.5, w, h, lut, step_voxels=0.5, mode=mode, low_cut=low_cut)
    p.brick_mode = ctx.brick_mode
    if gate is not None:
        p.skip_gate = gate
    ctx.set_transfer(lut)
    try:
        steps = np.zeros((h, w), np.uint32)
        mipi = np.zeros((h, w), np.uint32)
        got = ctx.raycast(p, w, h, steps=steps, mip_index=mipi)
        ref, rsteps, rmip, _, st = orc.render(p, bricks256, lut, w, h)
        assert st == 0
        _cmp(got, ref, f"{case} mode {mode}")
        assert np.array_equal(steps, rsteps), f"{case} mode {mode}: step counts"
        if mode == 1:
            assert np.array_equal(mipi, rmip), f"{case}: MIP indices"
    finally:
        ctx.set_transfer(scroll_tf)


def test_bad_page_entries_report_status(rb, orc, ctx, scroll_tf):
    """A page table whose entries point past the slot pool must not fault:
    the kernel treats them as absent and raises a status bit, like the
    oracle."""
    vol = rb.phantom(128, seed=5)
    sc = orc.BrickScene.build(vol, 1)
    page = sc.page.copy()
    page[64] = 5 | (200 << 24)  # slot 5 of a 1-slot pool
    ctx.bricks_load(page, sc.pool)
    bad = orc.BrickScene(page, sc.pool)
    p = rb.camera_view(0.3, -0.2, 2.0, 96, 64, scroll_tf)
    p.brick_mode = ctx.brick_mode
    ctx.status(clear=True)
    got = ctx.raycast(p, 96, 64)
    assert ctx.status() & 1
    ref, _, _, _, st = orc.render(p, bad, scroll_tf, 96, 64)
    assert st & 1
    _cmp(got, ref, "bad entries")
