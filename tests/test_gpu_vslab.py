"""Virtual slab on the GPU against the CPU oracle, frame by frame: the same
fill schedule (device: r3d_host_vslab_plan; oracle: its Python
restatement), every tile and the validity table bit for bit after each
frame, and views rendered from partly and fully resident windows, in every
mode, near (base tiles) and far (pyramid levels).  Images within 1/255 per
channel, step counts and MIP indices identical."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cmp(a, b, what, tol=1):
    d = np.abs(a.astype(np.int32) - b.astype(np.int32))
    assert d.max() <= tol, f"{what}: max diff {d.max()} at {np.unravel_index(d.argmax(), d.shape)}"


def _check_state(c, sc, what):
    assert np.array_equal(c.vslab_table(), sc.table), what
    for k in range(sc.v["ntiles"]):
        assert np.array_equal(c.vslab_read(k), sc.tiles[k]), (what, k)


def _views(rb, c, sc, lut, mode, dists):
    v = sc.v
    ext = (1.0, v["H"] / v["W"], v["D"] / v["W"])
    out = []
    for i, (dist, w, h, tx) in enumerate(dists):
        p = rb.camera_view(0.15 * (i - 1), 0.05, dist, w, h, lut,
                           target=(tx, 0.5 * ext[1], 0.5 * ext[2]), step_voxels=0.5, mode=mode)
        c.vslab_params(p)
        q = rb.FrameParams()
        sc.params(q)
        for f in ("slab_grid", "brick_mode", "slab_wz", "slab_z0", "slab_nx", "slab_ny",
                  "slab_px", "slab_depth", "slab_x0", "slab_y0"):
            assert getattr(p, f) == getattr(q, f), f
        p.density = 6.0  # thin windows need more opacity per sample to show
        out.append(p)
    return out


def _render_cmp(c, orc, sc, p, lut, what):
    w, h = p.viewport[0], p.viewport[1]
    steps = np.zeros((h, w), np.uint32)
    mipi = np.zeros((h, w), np.uint32)
    got = c.raycast(p, w, h, steps=steps, mip_index=mipi)
    ref, rs, rm, _, st = orc.render(p, sc, lut, w, h)
    assert st == 0
    _cmp(got, ref, what)
    assert np.array_equal(steps, rs) and np.array_equal(mipi, rm), what
    return got


NEAR = [(0.3, 192, 144, 0.5), (0.12, 160, 160, 0.3), (0.5, 224, 168, 0.7)]


@pytest.fixture(scope="module")
def moving(rb, scroll_tf):
    vol = rb.phantom((2600, 1800, 48), seed=47)
    c = rb.Context(0)
    c.set_transfer(scroll_tf)
    c.set_alpha_cutoff(0.98)
    c.vslab_begin(vol, 1200, 900, 8, 4)
    yield c, vol
    c.close()


def test_vslab_frames(rb, orc, moving, scroll_tf):
    c, vol = moving
    sc = orc.VSlabScene(vol, 1200, 900, 8, 4)
    assert sc.v["gx"][1] == 0 and sc.v["px"] == 160
    # partial residency (budget 6), margins growing, pans with prefetch, a z
    # scroll, a jump across the volume and back
    frames = [(1300, 900, 20)] * 4 + [(1300 + 120 * i, 900 - 60 * i, 20 + i) for i in range(1, 6)] \
        + [(2500, 1700, 39), (100, 100, 0), (1300, 900, 20)]
    for i, (fx, fy, z0) in enumerate(frames):
        st = c.vslab_frame(fx, fy, z0, 6)
        jobs = sc.frame(fx, fy, z0, 6)
        assert st["jobs"] == len(jobs) and st["origin"] == (sc.v["x0"], sc.v["y0"], sc.v["z0"])
        _check_state(c, sc, f"frame {i}")
        if i in (0, 3, 6, 9, 10):
            for k, p in enumerate(_views(rb, c, sc, scroll_tf, 0, NEAR)):
                got = _render_cmp(c, orc, sc, p, scroll_tf, f"frame {i} view {k}")
                if i == 3 and k == 0:
                    assert got[..., :3].astype(int).std() > 3, "blank view"


@pytest.mark.parametrize("mode", [1, 2, 3, 5])
def test_vslab_modes(rb, orc, moving, scroll_tf, mode):
    c, vol = moving
    sc = orc.VSlabScene(vol, 1200, 900, 8, 4)
    for _ in range(12):  # the whole window and its margin resident
        c.vslab_frame(1300, 900, 20, 64)
        sc.frame(1300, 900, 20, 64)
    for k, p in enumerate(_views(rb, c, sc, scroll_tf, mode, NEAR)):
        _render_cmp(c, orc, sc, p, scroll_tf, f"mode {mode} view {k}")


def test_vslab_pyramid(rb, orc, scroll_tf):
    vol = rb.phantom((8320, 8320, 6), seed=49)
    c = rb.Context(0)
    try:
        c.set_transfer(scroll_tf)
        c.set_alpha_cutoff(0.98)
        c.vslab_begin(vol, 8192, 8192, 4)
        sc = orc.VSlabScene(vol, 8192, 8192, 4)
        v = sc.v
        assert (v["px"], v["gx"][:4]) == (1024, [10, 4, 3, 0])
        for i in range(2):  # 81 cells, at most 64 listed a frame
            c.vslab_frame(4160, 4160, 1, 64)
            sc.frame(4160, 4160, 1, 64)
        _check_state(c, sc, "pyramid")
        # the oracle's level usage: the two far views sample pyramid level 2
        # (scale 8), the mid one level 1 (scale 4) and the base, the near one the base
        far = [(1.2, 96, 96, 0.5), (0.5, 128, 96, 0.4), (0.05, 128, 128, 0.55),
               (0.012, 128, 128, 0.45)]
        for mode in (0, 1):
            for k, p in enumerate(_views(rb, c, sc, scroll_tf, mode, far)):
                got = _render_cmp(c, orc, sc, p, scroll_tf, f"pyramid mode {mode} view {k}")
                if mode == 0:
                    assert got[..., :3].astype(int).std() > 2, f"view {k} is blank"
    finally:
        c.close()


def test_vslab_validation(rb, moving, scroll_tf):
    c, vol = moving
    c.vslab_frame(1300, 900, 20, 6)
    p = rb.camera_view(0.0, 0.05, 0.3, 64, 64, scroll_tf)
    c.vslab_params(p)
    c.raycast(p, 64, 64)
    for field, delta in [("slab_x0", 16.0), ("slab_z0", 1.0), ("brick_mode", 1), ("slab_wz", 1)]:
        q = p.copy()
        setattr(q, field, getattr(q, field) + delta)
        with pytest.raises(rb.R3DError):
            c.raycast(q, 64, 64)
    q = p.copy()
    q.slab_depth = 9  # deeper than the window
    with pytest.raises(rb.R3DError):
        c.raycast(q, 64, 64)
    with pytest.raises(rb.R3DError):
        c.vslab_read(10 ** 6)
    with pytest.raises(rb.R3DError):  # wider than the volume
        c.vslab_begin(vol, 2601, 900, 8)
