"""Tiled slab on the GPU against the CPU oracle: the device-built tiles of
every level bit for bit, views near (base tiles) and far (overview
levels) in every mode, and after the window moves through the z ring.
Images within 1/255 per channel, step counts and MIP indices identical."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NX, NY, NZ, WZ = 8400, 256, 24, 12


def _cmp(a, b, what, tol=1):
    d = np.abs(a.astype(np.int32) - b.astype(np.int32))
    assert d.max() <= tol, f"{what}: max diff {d.max()} at {np.unravel_index(d.argmax(), d.shape)}"


@pytest.fixture(scope="module")
def slab(rb, scroll_tf):
    vol = rb.phantom((NX, NY, NZ), seed=41)
    c = rb.Context(0)
    c.set_transfer(scroll_tf)
    c.set_alpha_cutoff(0.98)
    c.slab_build(vol, WZ, 3)
    yield c, vol
    c.close()


def _views(rb, c, lut, mode):
    ext = (1.0, NY / NX, (WZ - 2) / NX)
    ctr = (0.5 * ext[0], 0.5 * ext[1], 0.5 * ext[2])
    # face-on views of the thin window: far and mid footprints reach the
    # overview levels (scales 8 and 4), the near one samples base tiles
    far = rb.camera_view(0.0, 0.02, 0.5, 512, 96, lut, target=ctr, step_voxels=0.5, mode=mode,
                         lod_bias=0.5)
    mid = rb.camera_view(0.1, -0.1, 0.2, 384, 256, lut, target=(0.6, ctr[1], ctr[2]),
                         step_voxels=0.5, mode=mode)
    near = rb.camera_view(-0.2, 0.3, 0.04, 256, 256, lut, target=(0.43, ctr[1], ctr[2]),
                          step_voxels=0.5, mode=mode)
    out = []
    for p in (far, near, mid):
        c.slab_params(p)
        p.density = 6.0  # a thin window needs more opacity per sample to show
        out.append(p)
    return out


def test_slab_tiles_bit_exact(orc, slab):
    c, vol = slab
    sc = orc.SlabScene(vol, WZ, 3)
    assert sc.s.nlev == 3  # base + overview scales 4 and 8
    for lev in range(sc.s.nlev):
        for k in range(sc.tiles[lev].shape[0]):
            assert np.array_equal(c.slab_read(lev, k), sc.tiles[lev][k]), (lev, k)


@pytest.mark.parametrize("mode", [0, 1, 2, 3, 5])
def test_slab_views(rb, orc, slab, scroll_tf, mode):
    c, vol = slab
    sc = orc.SlabScene(vol, WZ, 3)
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
            assert (got[..., :3].astype(int).std() > 3), f"view {i} is blank"


def test_slab_window_moves(rb, orc, slab, scroll_tf):
    c, vol = slab
    for z0 in (7, 12, 0):  # ring scroll forward, a jump to the end, and back
        c.slab_window(z0)
        sc = orc.SlabScene(vol, WZ, min(z0, NZ - WZ))
        for lev in range(sc.s.nlev):
            assert np.array_equal(c.slab_read(lev, 0), sc.tiles[lev][0]), (z0, lev)
        for p in _views(rb, c, scroll_tf, 0)[:2]:
            w, h = p.viewport[0], p.viewport[1]
            ref = orc.render(p, sc, scroll_tf, w, h)[0]
            _cmp(c.raycast(p, w, h), ref, f"z0 {z0}")


def test_slab_view_validation(rb, slab, scroll_tf):
    c, _ = slab
    p = _views(rb, c, scroll_tf, 0)[0]
    p.slab_z0 += 1  # not the loaded window
    with pytest.raises(rb.R3DError):
        c.raycast(p, 32, 32)
    c.slab_params(p)
    p.slab_depth = WZ  # deeper than the ring allows
    with pytest.raises(rb.R3DError):
        c.raycast(p, 32, 32)
