"""Flattened-segment views on the GPU against the CPU oracle: a curved,
partly invalid segment through the 256^3 scroll phantom's LOD brick cache;
the baked flattened volume (CT and ink bytes) bit for bit at two pitches
(brick levels 0 and 1) and normal offsets, then surf views in FULL, FLAT
and MIP, with the ink tint, the distortion heatmap, the supervision mask
and half resolution, within 1/255 per channel."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GW = GH = 72
W, H, L, NBACK = 160, 144, 24, 12


def segment():
    """A wavy sheet z = 128 + 18 sin(x / 20) + 10 cos(y / 27) over a 72 x 72
    grid of 2.5-voxel cells, with an invalid corner."""
    j, i = np.mgrid[0:GH, 0:GW].astype(np.float64)
    x, y = 38.0 + 2.5 * i, 40.0 + 2.5 * j
    z = 128.0 + 18.0 * np.sin(x / 20.0) + 10.0 * np.cos(y / 27.0)
    dzdx, dzdy = 18.0 / 20.0 * np.cos(x / 20.0), -10.0 / 27.0 * np.sin(y / 27.0)
    n = np.stack([-dzdx, -dzdy, np.ones_like(x)], -1)
    n /= np.linalg.norm(n, axis=-1, keepdims=True)
    coords = np.zeros((GH, GW, 4), np.float32)
    coords[..., 0], coords[..., 1], coords[..., 2], coords[..., 3] = x, y, z, 1.0
    coords[:10, 50:, 3] = 0.0  # invalid quads
    normals = np.zeros((GH, GW, 4), np.float32)
    normals[..., :3] = n
    return coords, normals


def _cmp(a, b, what, tol=1):
    d = np.abs(a.astype(np.int32) - b.astype(np.int32))
    assert d.max() <= tol, f"{what}: max diff {d.max()} at {np.unravel_index(d.argmax(), d.shape)}"


@pytest.fixture(scope="module")
def surf(rb, orc, phantom256, scroll_tf):
    c = rb.Context(0)
    c.set_transfer(scroll_tf)
    c.set_alpha_cutoff(0.98)
    c.bricks_build(phantom256, 2)
    page, pool = c.bricks_read()
    bs = orc.BrickScene(page, pool)
    n = 256
    z, y, x = np.mgrid[0:n, 0:n, 0:n].astype(np.float32)
    ink = np.clip(255 - 2.0 * np.sqrt((x - 130) ** 2 + (y - 110) ** 2 + (z - 128) ** 2), 0, 255)
    ink = ink.astype(np.uint8)
    c.overlay_build(0, ink)
    bs.build_overlay(0, ink)
    coords, normals = segment()
    c.surf_begin(coords, normals)
    c.surfvol_begin(W, H, L, NBACK, 0.4, 0.4)
    mask = np.zeros((71 * 3, 71 * 3), np.uint8)
    mask[40:120, 30:90] = 1
    mask[100:170, 120:200] = 2
    c.surfmask(mask)
    sc = orc.SurfScene(bs, coords, normals, W, H, L, NBACK, 0.4, 0.4, mask=mask)
    yield c, sc
    c.close()


WINDOWS = [(2.0, 3.0, 1.0, 0.0, -1), (-20.0, -8.0, 1.25, 3.5, 0), (5.0, 1.0, 2.5, -2.0, 0)]


@pytest.mark.parametrize("win", range(len(WINDOWS)))
def test_surf_bake_bit_exact(rb, orc, surf, win):
    c, sc = surf
    u0, v0, step, zoff0, ovl = WINDOWS[win]
    c.surfvol_overlay(ovl)
    c.surfvol_window(u0, v0, step, zoff0)
    sc.bake(u0, v0, step, zoff0, ovl)
    got = c.surfvol_read()
    assert got.shape == sc.vol.shape
    assert np.array_equal(got, sc.vol), f"{np.argwhere(got != sc.vol)[:5]}"
    assert sc.vol[..., 0].std() > 5  # the sheet crosses the scroll
    if ovl == 0:
        assert sc.vol[..., 1].max() > 100


def _view(rb, c, sc, w, h, mode, centre, half_w, z0, depth, flags=0, ovl=0, gain=1.5,
          step=0.5, check=True):
    p = rb.FrameParams()
    p.viewport[0], p.viewport[1] = w, h
    p.mode = mode
    p.cam_origin[:] = (centre[0], centre[1], 0.0)
    p.cam_right[:] = (half_w, 0.0, 0.0)
    p.cam_up[:] = (0.0, half_w * h / w, 0.0)
    p.step_voxels, p.density = step, 1.5
    p.threshold = 0.02
    p.slab_z0, p.slab_depth = z0, depth
    p.view_flags = flags
    p.overlay_flags, p.overlay_gain = ovl, gain
    c.surfvol_params(p)
    if not check:
        return p
    q = rb.FrameParams()
    sc.params(q)
    for f in ("slab_x0", "slab_y0", "slab_px", "slab_nx", "slab_ny", "slab_wz", "slab_grid",
              "max_mip", "vol_tx", "vol_ty"):
        assert getattr(p, f) == getattr(q, f), f
    return p


CASES = {
    "full": dict(mode=0),
    "flat": dict(mode=5),
    "mip": dict(mode=1),
    "full_ink": dict(mode=0, ovl=1),
    "mip_ink_cyan": dict(mode=1, ovl=1 | (1 << 8)),
    "heatmap": dict(mode=0, flags=8),
    "mask": dict(mode=5, ovl=32),
    "half": dict(mode=0, flags=32),
    "thin_offset": dict(mode=0, z0=4.0, depth=3),
}


@pytest.mark.parametrize("case", list(CASES))
def test_surf_views(rb, orc, surf, scroll_tf, case):
    c, sc = surf
    u0, v0, step, zoff0, ovl = WINDOWS[1]
    c.surfvol_overlay(ovl)
    c.surfvol_window(u0, v0, step, zoff0)
    sc.bake(u0, v0, step, zoff0, ovl)
    kw = dict(CASES[case])
    mode, flags, ovlf = kw.pop("mode"), kw.pop("flags", 0), kw.pop("ovl", 0)
    z0, depth = kw.pop("z0", 0.0), kw.pop("depth", 16)
    for i, (w, h, centre, half_w) in enumerate([(200, 150, (70.0, 60.0), 80.0),
                                                (120, 120, (40.0, 90.0), 30.0)]):
        p = _view(rb, c, sc, w, h, mode, centre, half_w, z0, depth, flags=flags | 2, ovl=ovlf)
        got = c.raycast(p, w, h)
        ref = orc.render(p, sc, scroll_tf, w, h, want_aux=False)[0]
        _cmp(got, ref, f"{case} view {i}")
        assert got[..., :3].astype(int).std() > 3, f"{case} view {i} is blank"


def test_surf_validation(rb, surf, scroll_tf):
    c, sc = surf
    c.surfvol_window(*WINDOWS[0][:4])
    p = _view(rb, c, sc, 64, 64, 0, (60.0, 60.0), 40.0, 0.0, 8, flags=2, check=False)
    c.raycast(p, 64, 64)
    p.slab_x0 += 1.0  # not the baked window
    with pytest.raises(rb.R3DError):
        c.raycast(p, 64, 64)
    with pytest.raises(rb.R3DError):
        c.surfvol_overlay(2)  # labels are not baked
    with pytest.raises(rb.R3DError):
        c.surf_begin(np.zeros((2, 2, 4), np.float32), np.zeros((2, 2, 4), np.float32))
    fresh = rb.Context(0)
    try:
        with pytest.raises(rb.R3DError):  # no surface volume
            fresh.raycast(p, 64, 64)
    finally:
        fresh.close()


def test_surf_inkpred_bit_exact(rb, orc, surf):
    """A live prediction at a fractional origin and pitch, bilinear and
    clamped at its edge, replaces G over every layer inside it; dropping it
    restores the plain bake."""
    c, sc = surf
    rng = np.random.default_rng(31)
    pred = rng.random((57, 83), np.float32)
    pred[:5] = -0.25  # negative probabilities leave the overlay byte
    c.surfvol_overlay(0)
    try:
        for g0u, g0v, ppg in ((10.3, 5.6, 1.7), (-3.0, 20.25, 0.8)):
            c.surfvol_inkpred(pred, g0u, g0v, ppg)
            c.surfvol_window(2.0, 3.0, 1.0, 0.0)
            sc.inkpred(pred, g0u, g0v, ppg)
            sc.bake(2.0, 3.0, 1.0, 0.0, 0)
            got = c.surfvol_read()
            assert np.array_equal(got, sc.vol), f"{np.argwhere(got != sc.vol)[:5]}"
            col = (got[..., 1] == got[:1, ..., 1]).all(axis=0)  # one value per column
            assert col.mean() > 0.3
    finally:
        c.surfvol_inkpred(None)
        sc.inkpred(None, 0, 0, 0)
    c.surfvol_window(2.0, 3.0, 1.0, 0.0)
    sc.bake(2.0, 3.0, 1.0, 0.0, 0)
    assert np.array_equal(c.surfvol_read(), sc.vol)


def test_surf_inkpred_edges(rb, orc, surf):
    """A 1 x 1 prediction (bilinear and clamp both degenerate), one that
    lies outside the window, and NaN probabilities (never >= 0: the overlay
    byte stays); bad arguments are rejected."""
    c, sc = surf
    c.surfvol_overlay(0)
    cases = [(np.full((1, 1), 0.7, np.float32), 20.0, 20.0, 10.0),
             (np.full((4, 4), 0.9, np.float32), 500.0, 500.0, 1.0),
             (np.where(np.arange(64).reshape(8, 8) % 3 == 0, np.nan, 0.3).astype(np.float32),
              8.0, 9.0, 0.5)]
    try:
        for pred, g0u, g0v, ppg in cases:
            c.surfvol_inkpred(pred, g0u, g0v, ppg)
            c.surfvol_window(2.0, 3.0, 1.0, 0.0)
            sc.inkpred(pred, g0u, g0v, ppg)
            sc.bake(2.0, 3.0, 1.0, 0.0, 0)
            assert np.array_equal(c.surfvol_read(), sc.vol), (pred.shape, g0u)
        with pytest.raises(rb.R3DError):
            c.surfvol_inkpred(np.ones((2, 2), np.float32), 0.0, 0.0, 0.0)  # no texel pitch
    finally:
        c.surfvol_inkpred(None)
        sc.inkpred(None, 0, 0, 0)
