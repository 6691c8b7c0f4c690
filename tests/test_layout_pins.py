"""The section modes' layout math pinned to the reference's own code on
seeded random inputs (tests/golden/ref_layout.npz, made by
tests/golden/make_layout_golden.py from src/core/slab.h, clip.h and
vslab.h compiled unmodified): the oracle's tiled-slab layout and clipmap
origin policy, and the library's virtual-slab layout and ranges
(r3d_host_vslab_*) together with the oracle's restatement of them."""
import ctypes as C
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_layout.npz")


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLDEN)


def test_slab_layout_matches_reference(orc, gold):
    checked = 0
    for (nx, ny), r in zip(gold["slab_args"], gold["slab_out"]):
        lev = ((C.c_uint32 * 4) * 8)()
        ovs = C.c_uint32()
        n = orc.lib.orc_slab_layout(int(nx), int(ny), lev, C.byref(ovs))
        if r[0] != 0:
            assert n == 0, (nx, ny)
            continue
        gx, gy, px, py, rovs, nov = r[1:7]
        assert n == 1 + nov and ovs.value == rovs, (nx, ny)
        assert tuple(lev[0]) == (gx, gy, px, py), (nx, ny)
        for k in range(min(nov, 6)):
            assert tuple(lev[1 + k]) == tuple(r[7 + 4 * k:11 + 4 * k]), (nx, ny, k)
        checked += 1
    assert checked > 250


def test_clip_origins_match_reference(orc, gold):
    for (nx, ny, _, depth), focus, want, wzl in zip(gold["clip_args"], gold["clip_focus"],
                                                    gold["clip_origins"], gold["clip_wzl"]):
        assert [max(int(depth) // (1 << l) + 3, 4) for l in range(6)] == list(wzl)
        prev = None
        for f, (fx, fy) in enumerate(focus):
            prev = orc.clip_origins(int(nx), int(ny), int(fx), int(fy), prev=prev)
            assert prev == [tuple(int(v) for v in o) for o in want[f]], (nx, ny, f)


def test_vslab_layout_matches_reference(rb, orc, gold):
    valid = 0
    for a, r, rg in zip(gold["vslab_args"], gold["vslab_out"], gold["vslab_ranges"]):
        nx, ny, nz, W, H, D, zm = (int(v) for v in a)
        py = orc.vslab_layout(nx, ny, nz, W, H, D, zm)
        if r[0] != 0:
            assert py is None, tuple(a)
            with pytest.raises(ValueError):
                rb.VslabHost(nx, ny, nz, W, H, D, zm)
            continue
        valid += 1
        px, wz, nt = r[1:4]
        gx, gy, base = list(r[4:9]), list(r[9:14]), list(r[14:19])
        h = rb.VslabHost(nx, ny, nz, W, H, D, zm)
        v = h.v
        assert (v.px, v.wz, v.ntiles) == (px, wz, nt), tuple(a)
        assert list(v.gx) == gx and list(v.gy) == gy and list(v.base) == base, tuple(a)
        assert (py["px"], py["wz"], py["ntiles"], py["gx"], py["gy"], py["base"]) == \
            (px, wz, nt, gx, gy, base), tuple(a)
        o, z0, c0, c1, za, zb = (int(x) for x in rg)
        a0, a1 = C.c_int64(), C.c_int64()
        rb.lib.r3d_host_vslab_range(C.byref(v), 0, o, nx, W, C.byref(a0), C.byref(a1))
        assert (a0.value, a1.value) == (c0, c1), tuple(a)
        rb.lib.r3d_host_vslab_zrange(C.byref(v), z0, C.byref(a0), C.byref(a1))
        assert (a0.value, a1.value) == (za, zb), tuple(a)
    assert valid > 60
