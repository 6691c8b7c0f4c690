"""Data builders of the oracle and the phantom generator, on the CPU: the
(sum+4)/8 box rule (tools/lodpack/main.c:219-227), the dilated 8^3
occupancy (src/vk/vkbackend.c:794-870) and render3d's LOD page-table format
(src/vk/vkbackend.c:4184-4206), checked against direct numpy restatements."""
import numpy as np


def test_downsample_box_rule(orc):
    rng = np.random.default_rng(0)
    src = rng.integers(0, 256, (10, 12, 14), dtype=np.uint8)
    dst = np.empty((5, 6, 7), np.uint8)
    orc.lib.orc_downsample(src.ctypes.data, 14, 12, 10, dst.ctypes.data, 7, 6, 5)
    s = src.astype(np.uint32)
    want = (s[0::2, 0::2, 0::2] + s[0::2, 0::2, 1::2] + s[0::2, 1::2, 0::2] + s[0::2, 1::2, 1::2]
            + s[1::2, 0::2, 0::2] + s[1::2, 0::2, 1::2] + s[1::2, 1::2, 0::2] + s[1::2, 1::2, 1::2]
            + 4) // 8
    assert np.array_equal(dst, want.astype(np.uint8))


def test_mip_chain_sizes(orc):
    import ctypes as C
    dims = ((C.c_uint32 * 3) * 16)()
    assert orc.lib.orc_mip_levels(1024, 1024, 1024, dims) == 11
    assert orc.lib.orc_mip_levels(256, 100, 3, dims) == 9
    assert tuple(dims[8]) == (1, 1, 1) and tuple(dims[2]) == (64, 25, 1)


def test_occupancy_dilated(orc):
    rng = np.random.default_rng(1)
    vol = (rng.random((20, 17, 33)) < 0.01).astype(np.uint8) * rng.integers(1, 256, (20, 17, 33)).astype(np.uint8)
    out = np.empty((3, 3, 5), np.uint8)
    orc.lib.orc_occupancy(vol.ctypes.data, 33, 17, 20, out.ctypes.data)
    raw = np.zeros((3, 3, 5), np.uint8)
    for z in range(3):
        for y in range(3):
            for x in range(5):
                raw[z, y, x] = vol[z * 8:z * 8 + 8, y * 8:y * 8 + 8, x * 8:x * 8 + 8].max()
    want = np.zeros_like(raw)
    for z in range(3):
        for y in range(3):
            for x in range(5):
                want[z, y, x] = raw[max(z - 1, 0):z + 2, max(y - 1, 0):y + 2,
                                    max(x - 1, 0):x + 2].max()
    assert np.array_equal(out, want)


def test_lod_page_table_format(orc, rb):
    vol = rb.phantom((300, 260, 140), seed=9)
    sc = orc.BrickScene.build(vol, 3, min_max=50)
    page = sc.page
    assert page[0] == 3 and tuple(page[1:4]) == (300, 260, 140)
    bd = [(3, 3, 2), (2, 2, 1), (1, 1, 1)]
    off = 64
    for l in range(3):
        assert page[4 + 4 * l] == off
        assert page[5 + 4 * l] == bd[l][0] | bd[l][1] << 10 | bd[l][2] << 20
        assert page[6 + 4 * l] == 1 << l
        off += bd[l][0] * bd[l][1] * bd[l][2]
    assert page.size == off
    assert np.all(page[16:64] == 0)
    # level-0 entries: slot | max << 24 and the slot holds the brick
    nres = 0
    for bi in range(18):
        e = int(page[64 + bi])
        bx, by, bz = bi % 3, (bi // 3) % 3, bi // 9
        blk = np.zeros((128, 128, 128), np.uint8)
        part = vol[bz * 128:bz * 128 + 128, by * 128:by * 128 + 128, bx * 128:bx * 128 + 128]
        blk[:part.shape[0], :part.shape[1], :part.shape[2]] = part
        if blk.max() >= 50:
            assert e >> 24 == blk.max() and (e & 0xFFFFFF) == nres
            slot = sc.pool[nres * 128 ** 3:(nres + 1) * 128 ** 3].reshape(128, 128, 128)
            assert np.array_equal(slot, blk)
            nres += 1
        else:
            assert e == 0xFFFFFFFF
    # level 1 = (sum + 4) / 8 of the zero-padded level 0
    pad = np.zeros((256, 384, 384), np.uint32)
    pad[:140, :260, :300] = vol
    l1 = (pad[0::2, 0::2, 0::2] + pad[0::2, 0::2, 1::2] + pad[0::2, 1::2, 0::2]
          + pad[0::2, 1::2, 1::2] + pad[1::2, 0::2, 0::2] + pad[1::2, 0::2, 1::2]
          + pad[1::2, 1::2, 0::2] + pad[1::2, 1::2, 1::2] + 4) // 8
    e = int(page[64 + 18])  # level 1, brick (0, 0, 0)
    if e != 0xFFFFFFFF:
        slot = sc.pool[(e & 0xFFFFFF) * 128 ** 3:((e & 0xFFFFFF) + 1) * 128 ** 3]
        assert np.array_equal(slot.reshape(128, 128, 128), l1[:128, :128, :128].astype(np.uint8))


def test_phantom_deterministic_and_shaped(rb):
    a = rb.phantom(64, seed=7, threads=1)
    b = rb.phantom(64, seed=7, threads=5)
    assert np.array_equal(a, b)
    c = rb.phantom(64, seed=8, threads=2)
    assert not np.array_equal(a, c)
    v = rb.phantom(256, seed=1234)
    # papyrus sheets ~N(130, 15+6), air ~N(12, 4+6); radius 110 of 256
    hi = v[v > 90]
    lo = v[v < 60]
    assert abs(float(hi.mean()) - 130) < 3 and abs(float(lo.mean()) - 12) < 2
    frac = (v > 90).mean()
    assert 0.1 < frac < 0.4
    # the spiral is a prism along z
    assert abs(float((v[10] > 90).mean()) - float((v[200] > 90).mean())) < 0.01
