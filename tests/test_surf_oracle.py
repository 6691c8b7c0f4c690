"""The oracle's flattened-segment bake on the CPU: a flat segment whose
surface points fall on voxel centres bakes the volume's bytes exactly
(surface + normal * (zoff0 + l - nback), src/shaders/surfvol.comp:128-150),
invalid quads and points outside the volume bake 0, and the second byte
carries the overlay atlas."""
import numpy as np


def test_surf_bake_voxel_centres(orc):
    rng = np.random.default_rng(12)
    n = 128
    vol = rng.integers(0, 256, (n, n, n), dtype=np.uint8)
    bs = orc.BrickScene.build(vol, 1)
    ink = rng.integers(0, 256, (n, n, n), dtype=np.uint8)
    bs.build_overlay(0, ink)
    gh = gw = 40
    j, i = np.mgrid[0:gh, 0:gw].astype(np.float32)
    coords = np.zeros((gh, gw, 4), np.float32)
    coords[..., 0], coords[..., 1], coords[..., 2], coords[..., 3] = 10.5 + i, 20.5 + j, 60.5, 1.0
    coords[30:, 30:, 3] = 0.0  # an invalid corner
    normals = np.zeros((gh, gw, 4), np.float32)
    normals[..., 2] = 1.0
    W, H, L, nback = 36, 34, 10, 4
    sc = orc.SurfScene(bs, coords, normals, W, H, L, nback, 1.0, 1.0)
    # u = u0 + (x + 0.5) * step lands on grid column x + 1 for u0 = 0.5
    sc.bake(0.5, 0.5, 1.0, 2.0, 0)
    for l in range(L):
        z = 60 + 2 + l - nback
        for y in range(H):
            gy = y + 1
            for x in range(W):
                gx = x + 1
                # a quad touching the invalid corner bakes 0
                bad = gx + 1 >= 30 and gy + 1 >= 30
                want = (0, 0) if bad else (vol[z, 20 + gy, 10 + gx], ink[z, 20 + gy, 10 + gx])
                assert tuple(sc.vol[l, y, x]) == want, (l, y, x)
    # points above the volume bake 0
    sc.bake(0.5, 0.5, 1.0, 80.0, 0)
    assert not sc.vol[:, :28, :28].any()


def test_surf_inkpred(orc):
    """The live prediction replaces G over every layer of each column inside
    it (surfvol.comp:127-150), bilinear between prediction texels and
    clamped at their edge; columns outside keep the overlay byte."""
    rng = np.random.default_rng(13)
    n = 128
    vol = rng.integers(0, 256, (n, n, n), dtype=np.uint8)
    bs = orc.BrickScene.build(vol, 1)
    ink = rng.integers(0, 256, (n, n, n), dtype=np.uint8)
    bs.build_overlay(0, ink)
    gh = gw = 40
    j, i = np.mgrid[0:gh, 0:gw].astype(np.float32)
    coords = np.zeros((gh, gw, 4), np.float32)
    coords[..., 0], coords[..., 1], coords[..., 2], coords[..., 3] = 10.5 + i, 20.5 + j, 60.5, 1.0
    normals = np.zeros((gh, gw, 4), np.float32)
    normals[..., 2] = 1.0
    W, H, L = 36, 34, 6
    sc = orc.SurfScene(bs, coords, normals, W, H, L, 2, 1.0, 1.0)
    sc.bake(0.5, 0.5, 1.0, 0.0, 0)
    plain = sc.vol.copy()
    # 2 texels per grid unit over grid [4, 14) x [6, 21): pixel x samples
    # grid x + 1 = g, prediction texel (g - 4) * 2
    pred = rng.random((30, 20), np.float32)
    sc.inkpred(pred, 4.0, 6.0, 2.0)
    sc.bake(0.5, 0.5, 1.0, 0.0, 0)
    got = sc.vol
    assert np.array_equal(got[..., 0], plain[..., 0])
    for y in range(H):
        for x in range(W):
            g = (x + 1, y + 1)
            px, py = (g[0] - 4) * 2, (g[1] - 6) * 2
            if 0 <= px < 20 and 0 <= py < 30:
                want = int(np.floor(np.float32(pred[py, px]) * 255 + 0.5))
                assert np.all(got[:, y, x, 1] == want), (x, y)
            else:
                assert np.array_equal(got[:, y, x, 1], plain[:, y, x, 1]), (x, y)
    # half-texel offset: the average of two neighbours (clamped at the edge)
    sc.inkpred(pred, 4.25, 6.0, 2.0)
    sc.bake(0.5, 0.5, 1.0, 0.0, 0)
    x, y = 5, 9  # grid (6, 10): texel (3.5, 8)
    want = np.float32(pred[8, 3]) + np.float32(0.5) * (pred[8, 4] - pred[8, 3])
    assert abs(int(sc.vol[0, y, x, 1]) - want * 255) <= 0.51
    sc.inkpred(None, 0, 0, 0)
    sc.bake(0.5, 0.5, 1.0, 0.0, 0)
    assert np.array_equal(sc.vol, plain)
