"""The oracle's tiled slab on the CPU: layout against the reference's own
known answers (tests/test_quick.c:542-571), the apron mapping of tile
columns, the ring layers and the overview planes."""
import ctypes as C

import numpy as np
import pytest


def _layout(orc, nx, ny):
    lev = ((C.c_uint32 * 4) * 8)()
    ovs = C.c_uint32()
    n = orc.lib.orc_slab_layout(nx, ny, lev, C.byref(ovs))
    return n, [tuple(lev[i]) for i in range(n)], ovs.value


# (nx, ny) -> (gx, gy, px, ovs) from test_quick.c:545-568, -1 = rejected
PINS = [((1024, 1024), (1, 1, 1024, 4)), ((4092, 4092), (2, 2, 2046, None)),
        ((4093, 1024), (3, 1, 1365, None)), ((8184, 8184), (4, 4, 2046, 4)),
        ((8185, 1024), (5, None, None, 8)), ((16368, 16368), (8, 8, 2046, 8)),
        ((32736, 32736), (16, 16, 2046, 16)), ((43008, 43008), (22, 22, 1955, 32)),
        ((3072, 3072), (2, 2, 1536, None)), ((45013, 1024), -1)]


@pytest.mark.parametrize("pin", range(len(PINS)))
def test_slab_layout_pins(orc, pin):
    (nx, ny), want = PINS[pin]
    n, lev, ovs = _layout(orc, nx, ny)
    if want == -1:
        assert n == 0
        return
    gx, gy, px, wovs = want
    assert lev[0][0] == gx
    if gy is not None:
        assert lev[0][1] == gy
    if px is not None:
        assert lev[0][2] == px
    if wovs is not None:
        assert ovs == wovs
    # one overview level per scale 4, 8, ... up to ovs
    assert n - 1 == int(np.log2(ovs)) - 1


def test_slab_tiles_apron_ring_overview(orc):
    rng = np.random.default_rng(3)
    nx, ny, nz, wz, z0 = 4200, 300, 20, 8, 5
    vol = rng.integers(0, 256, (nz, ny, nx), dtype=np.uint8)
    sc = orc.SlabScene(vol, wz, z0)
    gx, gy, px, py = sc.s.lev[0]
    assert (gx, gy, px, py) == (3, 1, 1400, 300)
    t = sc.tiles[0]
    for s in range(z0, z0 + wz):
        layer = s % wz
        for i in range(gx):
            cols = np.clip(np.arange(px + 2) + i * px - 1, 0, nx - 1)
            rows = np.clip(np.arange(py + 2) - 1, 0, ny - 1)
            assert np.array_equal(t[i, layer], vol[s][np.ix_(rows, cols)]), (s, i)
    # overview level 1 (scale 4): truncating 4x4 box of the slice
    ov = sc.tiles[1]
    ogx, ogy, opx, opy = sc.s.lev[1]
    s = z0 + 3
    sl = vol[s].astype(np.int64)
    ref = np.zeros((75, 1050), np.int64)
    for y in range(75):
        for x in range(1050):
            ref[y, x] = sl[4 * y:4 * y + 4, 4 * x:4 * x + 4].sum() // 16
    rows = np.clip(np.arange(opy + 2) - 1, 0, 74)
    cols = np.clip(np.arange(opx + 2) - 1, 0, 1049)
    assert np.array_equal(ov[0, s % wz], ref[np.ix_(rows, cols)].astype(np.uint8))
