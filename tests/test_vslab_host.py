"""Virtual slab host logic on the CPU: the layout against the reference's own
known answers (tests/test_quick.c:629-669), the fill scheduler against an
independent Python restatement of the reference's frame loop
(vkbackend.c:6390-6620) over scripted pans, z scrolls and jumps, and the
oracle's fill against numpy."""
import ctypes as C

import numpy as np
import pytest


def _range(rb, h, o, n, span):
    c0, c1 = C.c_int64(), C.c_int64()
    rb.lib.r3d_host_vslab_range(C.byref(h.v), 0, o, n, span, C.byref(c0), C.byref(c1))
    return c0.value, c1.value


def _zrange(rb, h, z0):
    a, b = C.c_int64(), C.c_int64()
    rb.lib.r3d_host_vslab_zrange(C.byref(h.v), z0, C.byref(a), C.byref(b))
    return a.value, b.value


def test_vslab_layout_pins(rb, orc):
    n = 43008
    h = rb.VslabHost(n, n, 68608, 12096, 12096, 16)
    v = h.v
    assert (v.wz, v.px, v.gx[0], v.gy[0]) == (18, 1536, 10, 10)
    assert list(v.gx) == [10, 4, 3, 0, 0] and v.ntiles == 100 + 16 + 9
    assert _range(rb, h, 10000, n, 12096) == (6, 14)
    assert _range(rb, h, n - 12096, n, 12096)[1] == 27
    deep = rb.VslabHost(n, n, 68608, 2048, 2048, 2044).v
    assert (deep.px, deep.wz, deep.gx[0], deep.gx[1], deep.ntiles) == (256, 2046, 10, 0, 100)
    whole = rb.VslabHost(n, n, 68608, n, n, 4).v
    assert (whole.px, whole.wz, whole.gx[0], whole.gy[0]) == (2016, 6, 22, 22)
    assert whole.gx[1] == 6 and whole.gx[4] == 1 and whole.ntiles == 484 + 36 + 9 + 4 + 1
    for args in [(n, n, 68608, 12096, 12096, 2045), (n, n, 68608, n + 1, 4096, 16),
                 (8192, 8192, 23552, 8192, 8192, 8, 1020)]:
        with pytest.raises(ValueError):
            rb.VslabHost(*args)
        assert orc.vslab_layout(*args) is None
    assert rb.lib.r3d_host_vslab_key(3, 5) == (3 | (5 << 10) | 0x80000000)
    m = rb.VslabHost(8192, 8192, 23552, 8192, 8192, 8, 16)
    assert (m.v.D, m.v.z_margin, m.v.wz) == (8, 16, 42)
    assert _zrange(rb, m, 100) == (84, 126)
    assert _zrange(rb, m, 0) == (0, 42)
    assert _zrange(rb, m, 23544) == (23510, 23552)
    # the Python restatement agrees on every layout above
    for h2, args in [(h, (n, n, 68608, 12096, 12096, 16)), (m, (8192, 8192, 23552, 8192, 8192, 8, 16))]:
        py = orc.vslab_layout(*args)
        assert (py["px"], py["wz"], py["ntiles"]) == (h2.v.px, h2.v.wz, h2.v.ntiles)
        assert py["gx"] == list(h2.v.gx) and py["base"] == list(h2.v.base)


SCRIPTS = {
    # (volume, window, z margin, budget, frames of (fx, fy, z0))
    "pan_and_scroll": ((6000, 5000, 400), (2000, 1600, 16), 24, 6,
                       [(3000, 2500, 100)] * 3 + [(3000 + 150 * i, 2500 - 90 * i, 100 + 5 * i)
                                                  for i in range(12)]
                       + [(5900, 100, 380), (10, 4900, 0), (3000, 2500, 200)]),
    "small_budget_back_and_forth": ((3000, 3000, 120), (700, 500, 8), 0, 2,
                                    [(1500, 1500, 10 + 3 * (i % 7)) for i in range(10)]
                                    + [(1500 - 200 * i, 1500, 40 - 4 * i) for i in range(8)]),
    "whole_plane": ((4096, 4096, 64), (4096, 4096, 4), 2, 40,
                    [(2048, 2048, z) for z in (0, 1, 2, 9, 8, 30, 59, 58)]),
}


@pytest.mark.parametrize("name", sorted(SCRIPTS))
def test_vslab_plan_matches_restatement(rb, orc, name):
    (nx, ny, nz), (W, H, D), zm, budget, frames = SCRIPTS[name]
    h = rb.VslabHost(nx, ny, nz, W, H, D, zm)
    v = orc.vslab_layout(nx, ny, nz, W, H, D, zm)
    cells = [[None, None, 0, 0] for _ in range(v["gx"][0] * v["gy"][0])]
    total = 0
    for i, (fx, fy, z0) in enumerate(frames):
        got = h.frame(fx, fy, z0, budget)
        want = orc.vslab_plan(v, cells, fx, fy, z0, budget)
        for j in want:
            orc.vslab_apply(v, cells, j)
        assert got == want, (name, i)
        assert (h.v.x0, h.v.y0, h.v.z0) == (v["x0"], v["y0"], v["z0"]), (name, i)
        for c, py in zip(h.cells, cells):
            if py[0] is not None:
                assert (c.cx, c.cy, c.za, c.zb) == tuple(py), (name, i)
        total += len(got)
    assert total > len(frames)  # the script exercises the scheduler


def test_vslab_oracle_fill(orc):
    rng = np.random.default_rng(9)
    nz, ny, nx = 40, 700, 900
    vol = rng.integers(0, 256, (nz, ny, nx), dtype=np.uint8)
    sc = orc.VSlabScene(vol, 900, 700, 6, 2)
    v = sc.v
    P, T, wz = v["px"], v["px"] + 2, v["wz"]
    assert (P, wz, v["gx"][0], v["gy"][0]) == (128, 12, 8, 6) and v["gx"][1] == 0
    for _ in range(3):  # whole window resident after a few frames
        sc.frame(450, 350, 11, 64)
    za, zb = 9, 21
    for cy in range((ny - 1) // P + 1):
        for cx in range((nx - 1) // P + 1):
            slot = (cy % v["gy"][0]) * v["gx"][0] + cx % v["gx"][0]
            assert tuple(sc.table[slot]) == (cx | (cy << 10) | 0x80000000, za, zb, 0)
            wx = cx * P - 1 + np.arange(T)
            wy = cy * P - 1 + np.arange(T)
            for z in range(za, zb):
                want = vol[z][np.ix_(np.clip(wy, 0, ny - 1), np.clip(wx, 0, nx - 1))].copy()
                want[wy >= ny, :] = 0
                want[:, wx >= nx] = 0
                assert np.array_equal(sc.tiles[slot, z % wz], want), (cx, cy, z)


def test_vslab_oracle_pyramid(orc):
    rng = np.random.default_rng(10)
    nz, ny, nx = 4, 4096, 4096
    vol = rng.integers(0, 256, (nz, ny, nx), dtype=np.uint8)
    sc = orc.VSlabScene(vol, nx, ny, 2, 0)
    v = sc.v
    P, wz = v["px"], v["wz"]
    assert (P, v["gx"][0], v["gx"][1], v["gx"][2], wz) == (512, 8, 2, 0, 4)
    jobs = sc.frame(2048, 2048, 0, 64)
    assert len(jobs) == 64 and all(j[2:] == (0, 4) for j in jobs)
    # level 1 (4x): texel t of tile q holds level texel q * P - 1 + t, the
    # truncating 4x4 box of the volume.  The grid fits the level exactly, so
    # the strip of the last cell also reaches tile 2 = tile 0 (toroidal), whose
    # left apron thus holds level texel 1023; the right apron of tile 1 (level
    # texel 1024) is never written
    lev1 = (vol.reshape(nz, ny // 4, 4, nx // 4, 4).astype(np.uint32).sum(axis=(2, 4)) // 16)
    b1 = v["base"][1]
    for qy in range(2):
        for qx in range(2):
            tile = sc.tiles[b1 + qy * 2 + qx]
            for z in range(nz):
                ty = qy * P - 1 + np.arange(P + 2)
                tx = qx * P - 1 + np.arange(P + 2)
                ty[ty == -1], tx[tx == -1] = 1023, 1023
                iy, ix = (ty >= 0) & (ty < 1024), (tx >= 0) & (tx < 1024)
                want = np.zeros((P + 2, P + 2), np.uint8)
                want[np.ix_(iy, ix)] = lev1[z][np.ix_(ty[iy], tx[ix])]
                assert np.array_equal(tile[z % wz], want), (qx, qy, z)
