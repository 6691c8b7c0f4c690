"""The render.h-level calls of the section modes, streaming, overlays and
flattened views (r3d_render.h) on the GPU: each frame drawn through
r3d_frame + r3d_read_frame (banded for whole-image views) equals, bit for
bit, the same frame drawn through the r3d_cuda_* calls on a separate
context, whose parity with the oracle the other tests establish."""
import numpy as np
import pytest

from conftest import elev35

pytestmark = pytest.mark.gpu

W, H = 320, 256


def _pair(rb, lut):
    r = rb.Renderer(W, H)
    r.set_transfer(lut)
    r.set_alpha_cutoff(0.98)
    c = rb.Context(0)
    c.set_transfer(lut)
    c.set_alpha_cutoff(0.98)
    return r, c


def _frame(r, p):
    r.frame(p)
    return r.read_frame().copy()


def _face_on(rb, lut, nx, ny, depth, tx=0.5, dist=0.3):
    ext = (1.0, ny / nx, depth / nx)
    return rb.camera_view(0.1, 0.05, dist, W, H, lut, target=(tx, 0.5 * ext[1], 0.5 * ext[2]),
                          step_voxels=0.5)


def test_slab_calls(rb, scroll_tf):
    vol = rb.phantom((2600, 200, 24), seed=51)
    r, c = _pair(rb, scroll_tf)
    try:
        r.slab_init(vol.shape, 12)
        c.slab_build(vol, 12, 3)
        for z0 in (3, 7, 40):  # build, scroll, a start past the end (clamped to 12)
            r.slab_window(vol, z0)
            if z0 != 3:
                c.slab_window(min(z0, 12))
            p = _face_on(rb, scroll_tf, 2600, 200, 10)
            r.slab_params(p)
            q = p.copy()
            c.slab_params(q)
            assert q.slab_z0 == p.slab_z0 == float(min(z0, 12))
            p.slab_depth = q.slab_depth = 10
            p.density = q.density = 6.0
            got = _frame(r, p)
            assert np.array_equal(got, c.raycast(q, W, H)), z0
            assert got[..., :3].std() > 2
    finally:
        c.close()
        r.close()


def test_clip_and_vslab_calls(rb, scroll_tf):
    vol = rb.phantom((2600, 1800, 40), seed=52)
    r, c = _pair(rb, scroll_tf)
    try:
        r.clip_begin_volume(vol, 8)
        c.clip_build(vol, 8)
        for fx, z0 in ((1500.0, 5), (500.0, 20)):
            p = _face_on(rb, scroll_tf, 2600, 1800, 8)
            r.clip_frame(fx, 900.0, z0, p)
            q = p.copy()
            c.clip_frame(fx, 900.0, z0, q)
            p.density = q.density = 6.0
            assert np.array_equal(_frame(r, p), c.raycast(q, W, H)), fx
        r.vslab_begin_volume(vol, 1200, 900, 8, 4)
        c.vslab_begin(vol, 1200, 900, 8, 4)
        for fx, fy, z0 in ((1300.0, 900.0, 20), (1300.0, 900.0, 20), (1500.0, 800.0, 21)):
            p = _face_on(rb, scroll_tf, 1200, 900, 8)
            r.vslab_frame(fx, fy, z0, 6, p)
            q = p.copy()
            st = c.vslab_frame(fx, fy, z0, 6, q)
            o, pending = r.vslab_get()
            assert o == st["origin"] and pending == st["pending"]
            p.density = q.density = 6.0
            assert np.array_equal(_frame(r, p), c.raycast(q, W, H)), (fx, z0)
    finally:
        c.close()
        r.close()


def test_stream_and_overlay_calls(rb, phantom256, scroll_tf):
    r, c = _pair(rb, scroll_tf)
    try:
        r.bricks_begin_stream(phantom256, 2, 5)  # 9 bricks, 5 device slots
        c.stream_begin(phantom256, 2, 5)
        for i in range(3):
            p = elev35(rb, scroll_tf, W, H, step_voxels=0.5)
            p.frame_index = i
            r.bricks_params(p)
            v = rb.StreamView()
            e = (rb.C.c_float * 3)(1.0, 1.0, 1.0)
            rb.lib.r3d_cuda_stream_view_of(rb.C.byref(p), e, 4, rb.C.byref(v))
            r.bricks_stream(v)
            c.stream_update(p, 4)
            st = r.bricks_stats()
            assert st.hot_cap == 5 and st.nlevels == 2 and st.nb == 9 and st.hot <= 5
            assert np.array_equal(_frame(r, p), c.raycast(p, W, H)), i
        # the multi-view pump: a box and a point into one frame
        assert r.bricks_stream_begin()
        r.bricks_stream_box((0.1, 0.2, 0.3), (0.6, 0.5, 0.6), 0.6 / 256)
        r.bricks_stream_point((0.8, 0.8, 0.2), 0)
        r.bricks_stream_submit(3)
        c.stream_collect_begin()
        c.stream_collect_box((0.1, 0.2, 0.3), (0.6, 0.5, 0.6), 0.6 / 256)
        c.stream_collect_point((0.8, 0.8, 0.2), 0)
        st = c.stream_submit(3)
        assert r.bricks_stats().inflight == st["uploaded"]
        p = elev35(rb, scroll_tf, W, H, step_voxels=0.5)
        r.bricks_params(p)
        assert np.array_equal(_frame(r, p), c.raycast(p, W, H))
        r.close()
        c.close()
        r, c = _pair(rb, scroll_tf)
        assert not r.bricks_stream_begin()  # not streaming
        ink = np.roll(phantom256, 5, axis=2)
        r.bricks_begin_volume(phantom256, 2)
        r.bricks_overlay_volume(0, ink)
        c.bricks_build(phantom256, 2)
        c.overlay_build(0, ink)
        p = elev35(rb, scroll_tf, W, H, step_voxels=0.5)
        r.bricks_params(p)
        p.overlay_flags, p.overlay_gain = 1, 1.5
        assert np.array_equal(_frame(r, p), c.raycast(p, W, H))
    finally:
        c.close()
        r.close()


def test_surf_calls(rb, phantom256, scroll_tf):
    from test_gpu_surf import segment
    coords, normals = segment()
    r, c = _pair(rb, scroll_tf)
    try:
        ink = np.roll(phantom256, 7, axis=1)
        for x in (r, c):
            if x is r:
                x.bricks_begin_volume(phantom256, 2)
                x.bricks_overlay_volume(0, ink)
            else:
                x.bricks_build(phantom256, 2)
                x.overlay_build(0, ink)
            x.surf_begin(coords, normals)
            x.surfvol_begin(160, 144, 24, 12, 0.4, 0.4)
        r.surfvol_overlay_enable(True)
        c.surfvol_overlay(0)
        for win in ((2.0, 3.0, 1.0, 0.0), (2.0, 3.0, 1.0, 0.0), (-20.0, -8.0, 1.25, 3.5)):
            r.surfvol_window(*win)
            c.surfvol_window(*win)
            p = rb.FrameParams()
            p.viewport[0], p.viewport[1] = W, H
            p.cam_origin[:] = (70.0, 60.0, 0.0)
            p.cam_right[:] = (80.0, 0.0, 0.0)
            p.cam_up[:] = (0.0, 64.0, 0.0)
            p.step_voxels, p.density, p.threshold = 0.5, 1.5, 0.02
            p.slab_depth, p.overlay_flags, p.overlay_gain = 16, 1, 1.5
            r.surfvol_params(p)
            q = p.copy()
            c.surfvol_params(q)
            assert np.array_equal(_frame(r, p), c.raycast(q, W, H)), win
        # the bake's overlay pick: 3D ink, once loaded, wins over ink; the
        # registration tap over both; a live prediction over the pick
        ink3, reg = np.roll(phantom256, -9, axis=0), np.roll(phantom256, 4, axis=2)
        pred = np.random.default_rng(3).random((40, 50), np.float32)
        for which, arr in ((1, ink3), (3, reg)):
            r.bricks_overlay_volume(which, arr)
            c.overlay_build(which, arr)
        for regtap, want, use_pred in ((False, 1, False), (True, 3, False), (True, 3, True),
                                       (False, 1, True), (False, 1, False)):
            r.surfvol_regtap(regtap)
            c.surfvol_overlay(want)
            if use_pred:
                r.surfvol_inkpred(pred, 20.0, 18.0, 1.5)
                c.surfvol_inkpred(pred, 20.0, 18.0, 1.5)
            else:
                r.surfvol_inkpred_clear()
                c.surfvol_inkpred(None)
            p = rb.FrameParams()
            p.viewport[0], p.viewport[1] = W, H
            p.cam_origin[:] = (70.0, 60.0, 0.0)
            p.cam_right[:] = (80.0, 0.0, 0.0)
            p.cam_up[:] = (0.0, 64.0, 0.0)
            p.step_voxels, p.density, p.threshold = 0.5, 1.5, 0.02
            p.slab_depth, p.overlay_flags, p.overlay_gain = 16, 1, 1.5
            r.surfvol_params(p)
            q = p.copy()
            c.surfvol_params(q)
            assert np.array_equal(_frame(r, p), c.raycast(q, W, H)), (regtap, use_pred)
            want_vol = c.surfvol_read()
            got_vol = np.empty_like(want_vol)
            assert rb.lib.r3d_cuda_surfvol_read(r.cuda, got_vol.ctypes.data) == 0
            assert np.array_equal(got_vol, want_vol), (regtap, use_pred)
        r.surf_swap(coords, normals, 0.5, 0.5)  # the next window bakes everything
        r.surfvol_window(2.0, 3.0, 1.0, 0.0)
        p = rb.FrameParams()
        r.surfvol_params(p)
        assert p.vol_tx == 0.5 and p.slab_px == 1.0
        assert rb.lib.r3d_max_dim3d(r.r) == 2048
    finally:
        c.close()
        r.close()
