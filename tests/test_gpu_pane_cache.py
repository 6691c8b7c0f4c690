"""The render layer's pane cache (src/vk/vkbackend.c:7066-7159): a frame of
several views keeps the offscreen between frames, clears the regions no view
covers only when the layout changes, and draws a view only when its
parameters (all but the jitter seed frame_index) or the scene changed.
r3d_frame_stats.panes_drawn counts the views drawn.  Pixels are checked
against the oracle; R3D_NO_PANE_CACHE=1 draws every view every frame."""
import numpy as np
import pytest

from conftest import elev35

pytestmark = pytest.mark.gpu

W, H = 256, 160
CLEAR = np.array([13, 13, 15, 255], np.uint8)  # (0.05, 0.05, 0.06, 1) as RGBA8


def _views(rb, lut, yaws, orgs, frame=0):
    vs = []
    for yaw, (ox, oy) in zip(yaws, orgs):
        p = elev35(rb, lut, 112, 96, yaw=yaw, step_voxels=0.5, frame_index=frame)
        p.view_org = ox | (oy << 16)
        vs.append(p)
    return vs


def _draw(rb, r, views):
    st = rb.FrameStats()
    r.frame_views(views, st)
    return r.read_frame().copy(), st.panes_drawn


def _pane(img, p):
    ox, oy = p.view_org & 0xFFFF, p.view_org >> 16
    return img[oy:oy + p.viewport[1], ox:ox + p.viewport[0]]


def _oracle_pane(orc, scene, lut, p):
    q = p.copy()
    q.view_org = 0
    return orc.render(q, scene, lut, q.viewport[0], q.viewport[1])[0]


def test_pane_cache(rb, orc, scroll_tf, phantom256):
    vol = phantom256
    scene = orc.CubeScene(vol)
    r = rb.Renderer(W, H)
    try:
        r.set_transfer(scroll_tf)
        r.upload_volume(vol)
        orgs = [(8, 8), (136, 40)]
        vs = _views(rb, scroll_tf, [0.4, 2.1], orgs)
        img, n = _draw(rb, r, vs)
        assert n == 2
        for p in vs:
            assert np.abs(_pane(img, p).astype(int) - _oracle_pane(orc, scene, scroll_tf, p)
                          .astype(int)).max() <= 1
        mask = np.ones((H, W), bool)
        for p in vs:
            ox, oy = p.view_org & 0xFFFF, p.view_org >> 16
            mask[oy:oy + p.viewport[1], ox:ox + p.viewport[0]] = False
        assert np.all(img[mask] == CLEAR)  # uncovered regions cleared
        # only the jitter seed changed: nothing is drawn, the pixels stay
        img2, n = _draw(rb, r, _views(rb, scroll_tf, [0.4, 2.1], orgs, frame=7))
        assert n == 0 and np.array_equal(img2, img)
        # one camera moved: that pane alone is drawn
        vs3 = _views(rb, scroll_tf, [0.4, 2.6], orgs)
        img3, n = _draw(rb, r, vs3)
        assert n == 1
        assert np.array_equal(_pane(img3, vs3[0]), _pane(img, vs[0]))
        assert np.abs(_pane(img3, vs3[1]).astype(int) -
                      _oracle_pane(orc, scene, scroll_tf, vs3[1]).astype(int)).max() <= 1
        # a scene change (a new TF) draws every pane again
        lut2 = rb.tf_preset(1)
        r.set_transfer(lut2)
        img4, n = _draw(rb, r, vs3)
        assert n == 2
        for p in vs3:
            assert np.abs(_pane(img4, p).astype(int) -
                          _oracle_pane(orc, scene, lut2, p).astype(int)).max() <= 1
        # a layout change clears the offscreen and draws every pane
        vs5 = _views(rb, scroll_tf, [0.4, 2.6], [(0, 0), (120, 60)])
        img5, n = _draw(rb, r, vs5)
        assert n == 2
        assert np.all(img5[156:, :] == CLEAR) and np.all(img5[:60, 112:120] == CLEAR)
        # one view at the origin renders uncached, every frame
        one = _views(rb, scroll_tf, [1.0], [(0, 0)])
        _, n = _draw(rb, r, one)
        _, n2 = _draw(rb, r, one)
        assert n == 1 and n2 == 1
    finally:
        r.close()


def test_pane_cache_off(rb, scroll_tf, phantom256, monkeypatch):
    monkeypatch.setenv("R3D_NO_PANE_CACHE", "1")
    r = rb.Renderer(W, H)
    try:
        r.set_transfer(scroll_tf)
        r.upload_volume(phantom256)
        vs = _views(rb, scroll_tf, [0.4, 2.1], [(8, 8), (136, 40)])
        a, n = _draw(rb, r, vs)
        b, n2 = _draw(rb, r, vs)
        assert n == 2 and n2 == 2 and np.array_equal(a, b)
    finally:
        r.close()
