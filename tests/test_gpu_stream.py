"""The streaming LOD cache (brick residency pump) on the GPU: after every
update the render equals the oracle's over the device's own page table and
slots (read back), the budget and the pool bound hold, a still camera
converges, a moving one evicts least-recently-used slots, and the
coarsest level stays resident."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cmp(a, b, what, tol=1):
    d = np.abs(a.astype(np.int32) - b.astype(np.int32))
    assert d.max() <= tol, f"{what}: max diff {d.max()} at {np.unravel_index(d.argmax(), d.shape)}"


@pytest.fixture(scope="module")
def vol512(rb):
    return rb.phantom(512, seed=12)


def _view(rb, lut, yaw, pitch, dist, w=320, h=240):
    return rb.camera_view(yaw, pitch, dist, w, h, lut, step_voxels=0.5)


def test_stream_parity_budget_and_convergence(rb, orc, vol512, scroll_tf):
    c = rb.Context(0)
    try:
        c.set_transfer(scroll_tf)
        c.set_alpha_cutoff(0.98)
        c.stream_begin(vol512, 3, 24)
        info = c.bricks_info()
        assert info["nslots"] == 24 and info["nlev"] == 3
        page, _ = c.bricks_read(slots=False)
        assert page[int(page[4 + 8])] != 0xFFFFFFFF  # the coarsest brick is resident
        path = [(0.3 + 0.35 * i, -0.4 + 0.05 * i, 1.1 + 0.15 * (i % 3)) for i in range(8)]
        evicted = 0
        for i, (yaw, pitch, dist) in enumerate(path):
            p = _view(rb, scroll_tf, yaw, pitch, dist)
            p.brick_mode = c.brick_mode
            st = c.stream_update(p, budget=6)
            assert st["uploaded"] <= 6 and st["resident"] <= 24
            assert st["requested"] <= st["desired"]
            evicted += st["evicted"]
            got = c.raycast(p, 320, 240)
            page, pool = c.bricks_read()
            ref, _, _, _, stt = orc.render(p, orc.BrickScene(page, pool), scroll_tf, 320, 240)
            assert stt == 0 and c.status() == 0
            _cmp(got, ref, f"frame {i}")
            assert page[int(page[4 + 8])] != 0xFFFFFFFF
        assert evicted > 0  # the pool (24 slots) is smaller than the views' needs
        # a still camera converges: nothing left to copy in
        p = _view(rb, scroll_tf, 1.0, -0.3, 1.6)
        p.brick_mode = c.brick_mode
        for _ in range(30):
            st = c.stream_update(p, budget=4)
            if st["uploaded"] == 0:
                break
        assert st["uploaded"] == 0 and st["evicted"] == 0
        page, pool = c.bricks_read()
        ref = orc.render(p, orc.BrickScene(page, pool), scroll_tf, 320, 240)[0]
        _cmp(c.raycast(p, 320, 240), ref, "converged")
    finally:
        c.close()


def test_stream_errors(rb, vol512, scroll_tf):
    c = rb.Context(0)
    try:
        p = _view(rb, scroll_tf, 0.5, -0.3, 2.0)
        with pytest.raises(rb.R3DError):
            c.stream_update(p, budget=4)  # no streaming cache
        with pytest.raises(rb.R3DError):
            c.stream_begin(vol512, 3, 100)  # more slots than bricks (73)
        c.stream_begin(vol512, 3, 8)
        c.bricks_build(vol512, 3)  # a resident cache replaces the stream
        with pytest.raises(rb.R3DError):
            c.stream_update(p, budget=4)
    finally:
        c.close()


def test_stream_collects(rb, orc, vol512, scroll_tf):
    """The multi-view pump: a box, points and a cone collected into one
    frame upload the host request set's bricks nearest first; a cone alone
    through begin / collect_view / submit equals stream_update; collects
    outside an open frame fail."""
    full = orc.BrickScene.build(vol512, 3).page  # every brick of the pyramid
    box = ((0.2, 0.25, 0.3), (0.7, 0.6, 0.45), 0.6 / 512)
    pts = [((0.5, 0.5, 0.35), 0), ((0.05, 0.9, 0.9), 1)]
    c, d = rb.Context(0), rb.Context(0)
    try:
        for x in (c, d):
            x.set_transfer(scroll_tf)
            x.set_alpha_cutoff(0.98)
            x.stream_begin(vol512, 3, 30)
        with pytest.raises(rb.R3DError):
            c.stream_collect_box(*box)  # no open frame
        with pytest.raises(rb.R3DError):
            c.stream_submit(4)
        c.stream_collect_begin()
        c.stream_collect_box(*box)
        for p, lvl in pts:
            c.stream_collect_point(p, lvl)
        st = c.stream_submit(budget=12)
        col = rb.StreamCollect(full)
        col.box(*box)
        for p, lvl in pts:
            col.point(p, lvl)
        want = col.sorted()
        assert st["desired"] == col.n and st["uploaded"] == min(12, st["requested"])
        page, pool = c.bricks_read()
        coarse = int(page[4 + 8])
        req = [int(b) for b in want["brick"] if b != coarse]
        assert st["requested"] == len(req)
        assert all(page[b] != 0xFFFFFFFF for b in req[:12])  # nearest first
        assert all(page[b] == 0xFFFFFFFF for b in req[12:])
        p = _view(rb, scroll_tf, 0.8, -0.3, 1.4)
        p.brick_mode = c.brick_mode
        ref = orc.render(p, orc.BrickScene(page, pool), scroll_tf, 320, 240)[0]
        _cmp(c.raycast(p, 320, 240), ref, "after collects")
        # a cone alone, two ways: d through stream_update, e through the collects
        for i in range(3):
            p = _view(rb, scroll_tf, 0.3 + 0.4 * i, -0.35, 1.2)
            p.brick_mode = d.brick_mode
            s1 = d.stream_update(p, budget=5)
            assert s1["uploaded"] <= 5
        e = rb.Context(0)
        try:
            e.set_transfer(scroll_tf)
            e.set_alpha_cutoff(0.98)
            e.stream_begin(vol512, 3, 30)
            for i in range(3):
                p = _view(rb, scroll_tf, 0.3 + 0.4 * i, -0.35, 1.2)
                p.brick_mode = e.brick_mode
                e.stream_collect_begin()
                e.stream_collect_view(p)
                s2 = e.stream_submit(budget=5)
            assert np.array_equal(e.bricks_read(slots=False)[0], d.bricks_read(slots=False)[0])
            assert s2 == s1
        finally:
            e.close()
    finally:
        c.close()
        d.close()
