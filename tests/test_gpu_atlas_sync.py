"""CPU-sourced slot-parallel atlases on the GPU (labels, registration):
synced through gen / fetch callbacks, a resident cache's label atlas equals
the one cut from the same label volume by overlay_build, bit for bit and
in the rendered tint; a paint stroke re-uploads only the bricks whose
generation moved; re-attaching zeroes then refills; a detached source
syncs nothing; in a streamed cache, slots handed to other bricks are
zeroed first and refilled next; the render-level calls."""
import numpy as np
import pytest

from conftest import elev35

pytestmark = pytest.mark.gpu

ABSENT = 0xFFFFFFFF


def cut(vol, l, bx, by, bz):
    """Level l brick (bx, by, bz) of a label volume: the level-0 voxel at
    each coordinate << l, zero outside the volume."""
    nz, ny, nx = vol.shape
    out = np.zeros((128, 128, 128), np.uint8)
    xs, ys, zs = [(b * 128 + np.arange(128)) << l for b in (bx, by, bz)]
    mx, my, mz = xs < nx, ys < ny, zs < nz
    out[np.ix_(mz, my, mx)] = vol[np.ix_(zs[mz], ys[my], xs[mx])]
    return out


def labels256(seed=5):
    rng = np.random.default_rng(seed)
    z, y, x = np.mgrid[0:256, 0:256, 0:256]
    lab = np.zeros((256, 256, 256), np.uint8)
    lab[(x - 100) ** 2 + (y - 120) ** 2 + (z - 128) ** 2 < 60 ** 2] = 2
    lab[(x > 150) & (x < 220) & (y > 30) & (y < 90)] = 3
    lab[rng.random(lab.shape) < 0.002] = 1
    return lab


class Source:
    def __init__(self, rb, vol):
        self.vol = vol
        self.gens = {}
        self.fetched = 0
        self.src = rb.brick_src(self.gen, self.fetch)

    def gen(self, l, bx, by, bz):
        return self.gens.get((l, bx, by, bz), 1)

    def fetch(self, l, bx, by, bz):
        self.fetched += 1
        return cut(self.vol, l, bx, by, bz)


def test_labels_resident(rb, phantom256, scroll_tf):
    lab = labels256()
    a, b = rb.Context(0), rb.Context(0)
    try:
        for x in (a, b):
            x.set_transfer(scroll_tf)
            x.set_alpha_cutoff(0.98)
            x.bricks_build(phantom256, 2)
        b.overlay_build(2, lab)
        s = Source(rb, lab)
        a.atlas_attach(2, s.src)
        nslots = a.bricks_info()["nslots"]
        assert a.atlas_sync(2, 40) == nslots and a.atlas_sync(2, 0) == 0  # 40: at most 16
        assert np.array_equal(a.overlay_read(2), b.overlay_read(2))
        p = elev35(rb, scroll_tf, 256, 192, step_voxels=0.5)
        p.brick_mode = a.brick_mode
        p.overlay_flags = 8  # labels tint
        assert np.array_equal(a.raycast(p, 256, 192), b.raycast(p, 256, 192))
        # a paint stroke inside level-0 brick (1, 0, 1) and its level-1 parent
        lab[140:170, 20:50, 200:230] = 4
        s.gens[(0, 1, 0, 1)] = 2
        s.gens[(1, 0, 0, 0)] = 2
        s.fetched = 0
        assert a.atlas_sync(2, 0) == 2 and s.fetched == 2
        b.overlay_build(2, lab)
        assert np.array_equal(a.overlay_read(2), b.overlay_read(2))
        # re-attach: zeroed first (budget 4 a round), then refilled
        a.atlas_attach(2, s.src)
        rounds = [a.atlas_sync(2, 4) for _ in range(8)]
        assert rounds[:3] == [4, 4, 1] and sum(rounds) == 2 * nslots
        assert rounds[-1] == 0
        assert np.array_equal(a.overlay_read(2), b.overlay_read(2))
        # detached: the atlas stays, nothing syncs
        a.atlas_detach(2)
        s.gens[(0, 0, 0, 0)] = 9
        assert a.atlas_sync(2, 0) == 0
        assert np.array_equal(a.overlay_read(2), b.overlay_read(2))
        # a brick without content is zeroed
        a.atlas_attach(2, s.src)
        while a.atlas_sync(2, 0):
            pass
        s.gens[(0, 0, 0, 0)] = 0
        assert a.atlas_sync(2, 0) == 1
        page = a.bricks_read(slots=False)[0]
        slot = int(page[int(page[4])]) & 0xFFFFFF  # level 0 brick (0, 0, 0)
        assert not a.overlay_read(2)[slot].any()
    finally:
        a.close()
        b.close()


def test_registration_streamed(rb, phantom256, scroll_tf):
    reg = np.roll(phantom256, 11, axis=2)
    c = rb.Context(0)
    try:
        c.set_transfer(scroll_tf)
        c.set_alpha_cutoff(0.98)
        c.stream_begin(phantom256, 2, 5)

        def load(points):  # level-0 bricks under the points, one frame
            c.stream_collect_begin()
            for q in points:
                c.stream_collect_point(q, 0)
            return c.stream_submit(8)
        assert load([(0.1, 0.1, 0.1), (0.6, 0.1, 0.1), (0.1, 0.6, 0.1), (0.6, 0.6, 0.1)])["uploaded"] == 4
        s = Source(rb, reg)
        c.atlas_attach(3, s.src)
        while c.atlas_sync(3, 0):
            pass

        def check(zero=()):
            page = c.bricks_read(slots=False)[0]
            atlas = c.overlay_read(3)
            nl = int(page[0])
            for b in range(64, page.size):
                if page[b] == ABSENT:
                    continue
                for l in range(nl):
                    off, pk = int(page[4 + 4 * l]), int(page[5 + 4 * l])
                    dx, dy, dz = pk & 1023, (pk >> 10) & 1023, pk >> 20
                    if off <= b < off + dx * dy * dz:
                        loc = b - off
                        k = (l, loc % dx, (loc // dx) % dy, loc // (dx * dy))
                        break
                slot = int(page[b]) & 0xFFFFFF
                want = np.zeros((128,) * 3, np.uint8) if slot in zero else cut(reg, *k)
                assert np.array_equal(atlas[slot], want), (b, slot)
        check()
        before = c.bricks_read(slots=False)[0]
        assert load([(0.1, 0.1, 0.6), (0.6, 0.6, 0.6)])["evicted"] == 2
        after = c.bricks_read(slots=False)[0]
        moved = {int(after[b]) & 0xFFFFFF for b in range(64, after.size)
                 if after[b] != ABSENT and before[b] != after[b]}
        assert len(moved) == 2
        assert c.atlas_sync(3, 0) == 2  # stale slots zeroed first
        check(zero=moved)
        assert c.atlas_sync(3, 0) == 2  # then refilled
        check()
    finally:
        c.close()


def test_render_level_calls(rb, phantom256, scroll_tf):
    lab = labels256(7)
    r = rb.Renderer(256, 192)
    c = rb.Context(0)
    try:
        for x in (r, c):
            x.set_transfer(scroll_tf)
            x.set_alpha_cutoff(0.98)
        r.bricks_begin_volume(phantom256, 2)
        c.bricks_build(phantom256, 2)
        s, t = Source(rb, lab), Source(rb, np.roll(phantom256, 3, axis=1))
        r.bricks_labels(s.src)
        r.bricks_labels_sync(0)
        r.bricks_regatlas(t.src)
        r.bricks_regatlas_sync(0)
        c.overlay_build(2, lab)
        c.atlas_attach(3, t.src)
        c.atlas_sync(3, 0)
        p = elev35(rb, scroll_tf, 256, 192, step_voxels=0.5)
        r.bricks_params(p)
        p.overlay_flags = 8 | 16 | (128 << 16)  # labels, registration at alpha 128
        r.frame(p)
        assert np.array_equal(r.read_frame(), c.raycast(p, 256, 192))
        r.bricks_regatlas_detach()
        t.gens[(0, 0, 0, 0)] = 5
        r.bricks_regatlas_sync(0)  # detached: nothing
        assert t.fetched == c.bricks_info()["nslots"] * 2
    finally:
        c.close()
        r.close()
