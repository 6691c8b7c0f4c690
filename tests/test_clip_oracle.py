"""The oracle's XY clipmap on the CPU: the level origin policy against the
reference's own known answers (tests/test_quick.c:672-699), and the ring
layers of every level against a numpy restatement of the fill rules
(src/vk/vkclip.c:101-199, tools/mkpyramid/main.c:53-69)."""
import numpy as np


def test_clip_origin_pins(orc):
    n = 43008
    o = orc.clip_origins(n, n, 21504, 21504)
    assert o[0][0] % 16 == 0 and o[2][0] % 64 == 0
    assert 21504 - 1200 <= o[0][0] <= 21504 - 900
    assert o[5] == (0, 0)  # level 5 covers the whole cross-section
    assert orc.clip_origins(n, n, 0, 0, prev=o)[5] == (0, 0)  # and never recentres
    # recentre policy at level 0: a quarter of the coverage
    assert orc.clip_origins(n, n, 21504 + 400, 21504, prev=o)[0] == o[0]
    assert orc.clip_origins(n, n, 21504 + 600, 21504, prev=o)[0] != o[0]
    # recentring clamps at the volume edges
    assert orc.clip_origins(n, n, 0, 0)[1] == (0, 0)
    far = orc.clip_origins(n, n, n, n)[1]
    assert far[0] + 2046 * 2 <= n and far[1] + 2046 * 2 <= n


def _down2(v):
    z, y, x = (s // 2 for s in v.shape)
    v = v[: 2 * z, : 2 * y, : 2 * x].astype(np.uint32)
    s = sum(v[dz::2, dy::2, dx::2] for dz in (0, 1) for dy in (0, 1) for dx in (0, 1))
    return (s // 8).astype(np.uint8)


def _expect(vol, depth, origins, z0):
    nz, ny, nx = vol.shape
    pyr = [vol, _down2(vol)]
    for _ in range(2, 6):
        pyr.append(_down2(pyr[-1]))
    t = np.arange(2048)
    out = []
    for l in range(6):
        wzl = max(depth // (1 << l) + 3, 4)
        tex = np.zeros((wzl, 2048, 2048), np.uint8)
        vx0, vy0 = origins[l][0] // (1 << l) - 1, origins[l][1] // (1 << l) - 1
        for k in range(wzl):
            ls = (z0 >> l) + k
            layer = tex[ls % wzl]
            if l == 0 and ls < nz:
                layer[:] = vol[ls][np.ix_(np.clip(vy0 + t, 0, ny - 1), np.clip(vx0 + t, 0, nx - 1))]
            elif l == 1:
                acc = np.zeros((2048, 2048), np.uint32)
                for dz in (0, 1):
                    if 2 * ls + dz >= nz:
                        continue
                    for dy in (0, 1):
                        for dx in (0, 1):
                            rows = np.clip(2 * (vy0 + t) + dy, 0, ny - 1)
                            cols = np.clip(2 * (vx0 + t) + dx, 0, nx - 1)
                            acc += vol[2 * ls + dz][np.ix_(rows, cols)]
                layer[:] = acc // 8
            elif l >= 2 and ls < pyr[l].shape[0]:
                pz, py, px = pyr[l].shape
                layer[:] = pyr[l][ls][np.ix_(np.clip(vy0 + t, 0, py - 1), np.clip(vx0 + t, 0, px - 1))]
        out.append(tex)
    return out


def test_clip_fill_levels(orc):
    rng = np.random.default_rng(5)
    nz, ny, nx, depth = 21, 70, 2600, 4
    vol = rng.integers(0, 256, (nz, ny, nx), dtype=np.uint8)
    for fx, fy, z0 in ((1800.0, 30.0, 3), (10.0, 5.0, 17)):  # interior, and the far z end
        origins = orc.clip_origins(nx, ny, fx, fy)
        sc = orc.ClipScene(vol, depth, origins, z0)
        # ring depths: window / 2^l + 3 slices, at least 4 (test_quick.c:678-679)
        assert list(sc.c.wzl) == [7, 5, 4, 4, 4, 4]
        want = _expect(vol, depth, origins, z0)
        for l in range(6):
            assert np.array_equal(sc.tex[l], want[l]), (fx, z0, l)
    # level 0 of the first focus sits at the right edge of the volume
    o = orc.clip_origins(nx, ny, 1800.0, 30.0)
    assert o[0] == (544, 0) and o[1] == (0, 0)
