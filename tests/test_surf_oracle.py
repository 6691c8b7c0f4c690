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
