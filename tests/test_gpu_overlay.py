"""Slot-parallel overlay atlases (ink, 3D ink, paint labels, registration)
on the LOD brick cache, GPU against the CPU oracle: every flag
combination in FULL, FLAT and MIP, within 1/255 per channel with identical
step counts and MIP indices; the device builder against slot contents
given directly; and the errors for views that ask for missing atlases."""
import numpy as np
import pytest

from conftest import elev35

pytestmark = pytest.mark.gpu

INK, INK3D, LABELS, REG = 1, 4, 8, 16


def _cmp(a, b, what, tol=1):
    d = np.abs(a.astype(np.int32) - b.astype(np.int32))
    assert d.max() <= tol, f"{what}: max diff {d.max()} at {np.unravel_index(d.argmax(), d.shape)}"


@pytest.fixture(scope="module")
def volumes(rb, phantom256):
    n = 256
    z, y, x = np.mgrid[0:n, 0:n, 0:n].astype(np.float32)
    rng = np.random.default_rng(21)
    ink = np.clip(255 - 1.5 * np.sqrt((x - 140) ** 2 + (y - 120) ** 2 + (z - 128) ** 2), 0, 255)
    ink = (ink + rng.normal(0, 5, ink.shape)).clip(0, 255).astype(np.uint8)
    ink3d = (((x + y) // 24 % 3 == 0) & (z > 96) & (z < 160)).astype(np.uint8) * 180
    labels = ((x // 16 + y // 16) % 9).astype(np.uint8)  # class 0 = unlabelled
    reg = np.roll(phantom256, (2, -3, 4), axis=(0, 1, 2))  # a misregistered second scan
    return {"ink": ink, "ink3d": ink3d, "labels": labels, "reg": reg}


@pytest.fixture(scope="module")
def ovl_scene(rb, orc, phantom256, scroll_tf, volumes):
    c = rb.Context(0)
    c.set_transfer(scroll_tf)
    c.set_alpha_cutoff(0.98)
    c.bricks_build(phantom256, 2)
    page, pool = c.bricks_read()
    sc = orc.BrickScene(page, pool)
    for i, k in enumerate(("ink", "ink3d", "labels", "reg")):
        c.overlay_build(i, volumes[k])
        sc.build_overlay(i, volumes[k])
    yield c, sc
    c.close()


CASES = {"ink": INK, "ink_cyan": INK | (1 << 8), "ink3d": INK3D, "labels": LABELS,
         "reg": REG | (128 << 16), "all": INK | INK3D | LABELS | REG | (200 << 16)}


@pytest.mark.parametrize("mode", [0, 5, 1])
@pytest.mark.parametrize("case", list(CASES))
def test_overlay_views(rb, orc, ovl_scene, scroll_tf, case, mode):
    c, sc = ovl_scene
    p = elev35(rb, scroll_tf, 256, 256, step_voxels=0.5, mode=mode)
    p.brick_mode = c.brick_mode
    p.overlay_flags = CASES[case]
    p.overlay_gain = 1.5
    steps = np.zeros((256, 256), np.uint32)
    mipi = np.zeros((256, 256), np.uint32)
    got = c.raycast(p, 256, 256, steps=steps, mip_index=mipi)
    ref, rs, rm, _, st = orc.render(p, sc, scroll_tf, 256, 256)
    assert st == 0
    _cmp(got, ref, f"{case} mode {mode}")
    assert np.array_equal(steps, rs) and np.array_equal(mipi, rm)
    # the overlay must show: the same view without it differs
    p.overlay_flags = 0
    plain = c.raycast(p, 256, 256)
    assert (np.abs(plain.astype(int) - got.astype(int)).max() > 8), case


def test_overlay_zero_gain_is_the_plain_render(rb, ovl_scene, scroll_tf):
    c, _ = ovl_scene
    p = elev35(rb, scroll_tf, 256, 256, step_voxels=0.5, mode=0)
    p.brick_mode = c.brick_mode
    plain = c.raycast(p, 256, 256)
    p.overlay_flags = INK | INK3D
    p.overlay_gain = 0.0
    assert np.array_equal(c.raycast(p, 256, 256), plain)


def test_overlay_load_equals_build(rb, orc, ovl_scene, scroll_tf):
    """Slot contents uploaded directly give the same images as the device
    builder's, and a persistent schedule renders overlay views the same."""
    c, sc = ovl_scene
    p = elev35(rb, scroll_tf, 256, 256, yaw=2.2, step_voxels=0.5, mode=0)
    p.brick_mode = c.brick_mode
    p.overlay_flags = INK | LABELS | REG | (90 << 16)
    p.overlay_gain = 2.0
    built = c.raycast(p, 256, 256)
    c.set_schedule(persistent=1)
    try:
        assert np.array_equal(c.raycast(p, 256, 256), built)
    finally:
        c.set_schedule()
    for i in (0, 2, 3):
        c.overlay_load(i, sc.ovl[i])
    assert np.array_equal(c.raycast(p, 256, 256), built)


def test_overlay_errors(rb, phantom256, scroll_tf):
    c = rb.Context(0)
    try:
        c.set_transfer(scroll_tf)
        c.upload_volume(phantom256)
        p = elev35(rb, scroll_tf, 64, 64)
        p.overlay_flags = INK
        with pytest.raises(rb.R3DError):
            c.raycast(p, 64, 64)  # overlays need the LOD brick cache
        c.bricks_build(phantom256, 2)
        p.brick_mode = c.brick_mode
        with pytest.raises(rb.R3DError):
            c.raycast(p, 64, 64)  # ink atlas not loaded
        with pytest.raises(rb.R3DError):
            c.overlay_build(0, phantom256[:, :, :200].copy())  # wrong shape
        c.overlay_build(0, phantom256)
        c.raycast(p, 64, 64)
        c.bricks_build(phantom256, 2)  # a new cache drops its overlays
        with pytest.raises(rb.R3DError):
            c.raycast(p, 64, 64)
    finally:
        c.close()
