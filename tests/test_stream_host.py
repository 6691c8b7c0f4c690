"""The streamer's request set on the CPU: r3d_host_stream_desired against a
restatement of render3d's view-cone LOD request (src/vk/vkbackend.c:
3075-3106,5416-5500) written here in float32 Python, for several cameras,
slice windows and gates, on a 512^3 pyramid of 3 levels."""
import math

import numpy as np
import pytest

f32 = np.float32


def _axis(eye, radius, edge, n):
    a = int(math.ceil(f32(f32(eye - radius) / edge) - f32(0.5)))
    b = int(math.floor(f32(f32(eye + radius) / edge) - f32(0.5))) + 1
    return min(max(a, 0), n), min(max(b, 0), n)


def _restated(orc, page, eye, fwd, half_tan, pixel_cone, gate, z0, depth):
    nlev, shape = int(page[0]), [int(page[1]), int(page[2]), int(page[3])]
    maxdim = f32(max(shape))
    tanw = f32(f32(half_tan) * f32(1.15)) + f32(1e-3)
    g8 = max(int(f32(f32(gate) * f32(255.0)) + f32(0.5)), 5)
    lod_factor = max(f32(f32(pixel_cone) * maxdim), f32(1e-6))
    eye = [f32(x) for x in eye]
    fwd = [f32(x) for x in fwd]
    seen, out = set(), []
    for li in range(nlev - 1):
        off, packed, scale = int(page[4 + 4 * li]), int(page[5 + 4 * li]), int(page[6 + 4 * li])
        bd = (packed & 1023, (packed >> 10) & 1023, packed >> 20)
        poff, pp = int(page[4 + 4 * (li + 1)]), int(page[5 + 4 * (li + 1)])
        pbd = (pp & 1023, (pp >> 10) & 1023)
        edge = f32(f32(128 * scale) / maxdim)
        brad = f32(f32(0.8660254) * edge)
        outer = f32(f32(2.0 ** (li + 1)) / lod_factor) + brad
        x0, x1 = _axis(eye[0], outer, edge, bd[0])
        y0, y1 = _axis(eye[1], outer, edge, bd[1])
        zr = _axis(eye[2], outer, edge, bd[2])
        z0_, z1_ = zr
        if depth:
            zlast = min(z0 + depth, shape[2])
            zb = 128 * scale
            z0_, z1_ = max(z0_, z0 // zb), min(z1_, (zlast + zb - 1) // zb)
        for bz in range(z0_, z1_):
            for by in range(y0, y1):
                for bx in range(x0, x1):
                    c = [f32(f32(f32(b) + f32(0.5)) * edge) - e for b, e in zip((bx, by, bz), eye)]
                    d2 = f32(f32(c[0] * c[0]) + f32(c[1] * c[1])) + f32(c[2] * c[2])
                    along = f32(f32(c[0] * fwd[0]) + f32(c[1] * fwd[1])) + f32(c[2] * fwd[2])
                    vis = d2 < f32(f32(edge + brad) * f32(edge + brad))
                    if not vis and along > 0:
                        perp2 = f32(d2 - f32(along * along))
                        rad = f32(f32(along * tanw) + brad)
                        vis = perp2 < f32(rad * rad)
                    if not vis:
                        continue
                    if orc.lib.orc_lod_pick(float(np.sqrt(d2)), pixel_cone, float(maxdim),
                                            nlev) != li:
                        continue
                    cands = (poff + ((bz >> 1) * pbd[1] + (by >> 1)) * pbd[0] + (bx >> 1),
                             off + (bz * bd[1] + by) * bd[0] + bx)
                    for pri, b in enumerate(cands):
                        e = int(page[b])
                        if b in seen or e == 0xFFFFFFFF or (e >> 24) < g8:
                            continue
                        seen.add(b)
                        out.append((float(d2), b, pri))
    out.sort(key=lambda t: (t[2], t[0], t[1]))
    return out


@pytest.fixture(scope="module")
def page512(rb, orc):
    vol = rb.phantom(512, seed=5)
    return orc.BrickScene.build(vol, 3).page


CAMS = [  # eye, fwd, half_tan, pixel_cone, gate, z0, depth
    ((0.5, 0.5, -1.2), (0, 0, 1), 0.66, 2 * 0.577 / 1080, 0.0, 0, 0),
    ((0.5, 0.5, 0.3), (0, 0.6, 0.8), 0.66, 2 * 0.577 / 720, 40 / 255, 0, 0),
    ((1.6, 0.2, 0.7), (-0.8, 0.3, -0.1), 0.4, 2 * 0.3 / 512, 0.0, 0, 0),
    ((0.5, 0.5, 0.5), (1, 0, 0), 1.2, 2 * 1.0 / 256, 0.1, 100, 64),
    ((0.1, 0.9, 0.4), (0.5, -0.5, 0.7), 0.66, 2 * 0.577 / 4320, 0.0, 0, 0),
]


@pytest.mark.parametrize("cam", range(len(CAMS)))
def test_request_set_matches_restatement(rb, orc, page512, cam):
    eye, fwd, ht, pc, gate, z0, depth = CAMS[cam]
    fwd = np.array(fwd, np.float64)
    fwd = tuple(float(x) for x in fwd / np.linalg.norm(fwd))
    got = rb.stream_desired(page512, eye, fwd, ht, pc, gate, z0, depth)
    ref = _restated(orc, page512, eye, fwd, ht, pc, gate, z0, depth)
    assert len(ref) > 0 or cam == 2
    assert [(int(b), int(p)) for _, b, p in got] == [(b, p) for _, b, p in ref]
    assert np.array_equal(got["d2"], np.array([d for d, _, _ in ref], np.float32))
    # every listed brick is a real, bright enough brick of a non-coarsest
    # level or the parent of one
    for b in got["brick"]:
        assert 64 <= b < page512.size and page512[b] != 0xFFFFFFFF


def _level(page, li, maxdim):
    off, packed, scale = int(page[4 + 4 * li]), int(page[5 + 4 * li]), int(page[6 + 4 * li])
    return off, (packed & 1023, (packed >> 10) & 1023, packed >> 20), f32(f32(128 * scale) / maxdim)


def _add(page, out, seen, b, d2, pri, g8):
    e = int(page[b])
    if b in seen or e == 0xFFFFFFFF or (e >> 24) < g8:
        return
    seen.add(b)
    out.append((float(d2), b, pri))


def _box_restated(page, lo, hi, pixel_cone, gate, out, seen):
    """r3d_bricks_stream_box (vkbackend.c:5330-5382) over a full page table."""
    nlev = int(page[0])
    maxdim = f32(max(int(page[1]), int(page[2]), int(page[3])))
    g8 = max(int(f32(f32(gate) * f32(255.0)) + f32(0.5)), 5)
    vpp = max(f32(f32(pixel_cone) * maxdim), f32(1.0))
    desired = min(int(math.floor(math.log2(float(vpp)))), nlev - 1)
    lo, hi = [f32(x) for x in lo], [f32(x) for x in hi]
    while True:
        off, bd, edge = _level(page, desired, maxdim)
        rng = []
        for a in range(3):
            a0 = max(int(math.floor(f32(lo[a] / edge))), 0)
            a1 = min(int(math.floor(f32(hi[a] / edge))) + 1, bd[a])
            rng.append((a0, max(a1, a0)))
        count = math.prod(b - a for a, b in rng)
        if count <= 2048 or desired + 1 >= nlev:
            break
        desired += 1
    c0 = [f32(f32(a + b) * f32(0.5)) for a, b in zip(lo, hi)]
    parent = desired + 1 < nlev
    if parent:
        poff, pbd, _ = _level(page, desired + 1, maxdim)
    for bz in range(*rng[2]):
        for by in range(*rng[1]):
            for bx in range(*rng[0]):
                d = [f32(f32(f32(b) + f32(0.5)) * edge) - c for b, c in zip((bx, by, bz), c0)]
                d2 = f32(f32(d[0] * d[0]) + f32(d[1] * d[1])) + f32(d[2] * d[2])
                if parent:
                    _add(page, out, seen, poff + ((bz >> 1) * pbd[1] + (by >> 1)) * pbd[0] + (bx >> 1),
                         d2, 0, g8)
                _add(page, out, seen, off + (bz * bd[1] + by) * bd[0] + bx, d2, 1, g8)
    return desired


def _point_restated(page, p, level, gate, out, seen):
    """r3d_bricks_stream_point (vkbackend.c:5384-5414)."""
    nlev = int(page[0])
    maxdim = f32(max(int(page[1]), int(page[2]), int(page[3])))
    g8 = max(int(f32(f32(gate) * f32(255.0)) + f32(0.5)), 5)
    level = min(level, nlev - 1)
    off, bd, edge = _level(page, level, maxdim)
    bc = [min(max(int(f32(f32(x) / edge)), 0), n - 1) for x, n in zip(p, bd)]
    if level + 1 < nlev:
        poff, pbd, _ = _level(page, level + 1, maxdim)
        _add(page, out, seen, poff + ((bc[2] >> 1) * pbd[1] + (bc[1] >> 1)) * pbd[0] + (bc[0] >> 1),
             f32(0), 0, g8)
    _add(page, out, seen, off + (bc[2] * bd[1] + bc[1]) * bd[0] + bc[0], f32(0), 1, g8)


def _synth_page(shape, nlev, seed):
    """A full pyramid page table of a large volume without building it:
    random brick maxima, about 10 % absent."""
    levels, off = [], 64
    for li in range(nlev):
        s = 128 << li
        bd = [(n + s - 1) // s for n in shape]
        levels.append((off, bd[0] | (bd[1] << 10) | (bd[2] << 20), 1 << li))
        off += math.prod(bd)
    page = np.zeros(off, np.uint32)
    page[0], page[1:4] = nlev, shape
    for li, lv in enumerate(levels):
        page[4 + 4 * li:7 + 4 * li] = lv
    rng = np.random.default_rng(seed)
    n = off - 64
    page[64:] = (rng.integers(0, 256, n).astype(np.uint32) << 24) | np.arange(n, dtype=np.uint32)
    page[64:][rng.random(n) < 0.1] = 0xFFFFFFFF
    return page


BOXES = [  # lo, hi, pixel_cone, gate
    ((0.40, 0.40, 0.45), (0.60, 0.55, 0.50), 0.3 / 8192, 0.0),  # finest level
    ((0.10, 0.20, 0.30), (0.35, 0.30, 0.33), 3.1 / 8192, 0.2),  # level 1 by pitch
    ((0.0, 0.0, 0.0), (1.0, 1.0, 0.5), 0.5 / 8192, 0.0),  # coarsened to the last level
    ((-0.3, 0.9, 0.2), (0.2, 1.4, 0.21), 0.7 / 8192, 0.0),  # past the y extent (0.75): empty
    ((-0.3, 0.6, 0.2), (0.2, 0.9, 0.21), 0.7 / 8192, 0.0),  # clamped at the edges
    ((0.2, 0.2, 0.3), (0.6, 0.5, 0.36), 1.5 / 8192, 0.0),  # coarsened once
]


def test_box_and_point_collects_match_restatement(rb):
    page = _synth_page((8192, 6144, 4096), 3, 21)
    for i, (lo, hi, pc, gate) in enumerate(BOXES):
        col = rb.StreamCollect(page)
        col.box(lo, hi, pc, gate)
        ref, seen = [], set()
        lev = _box_restated(page, lo, hi, pc, gate, ref, seen)
        got = np.ctypeslib.as_array(col.out)[:col.n]
        assert [(int(b), int(p)) for _, b, p in got] == [(b, p) for _, b, p in ref], i
        assert np.array_equal(got["d2"], np.array([d for d, _, _ in ref], np.float32)), i
        assert (len(ref) == 0) == (i == 3), i
        if i == 2:
            assert lev == 2
        if i == 5:
            assert lev == 1
    pts = [((0.51, 0.26, 0.7), 0), ((0.0, 0.0, 0.0), 1), ((1.2, -0.5, 0.49), 0), ((0.9, 0.6, 0.3), 7)]
    col, ref, seen = rb.StreamCollect(page), [], set()
    for p, lvl in pts:
        col.point(p, lvl, 0.0)
        _point_restated(page, p, lvl, 0.0, ref, seen)
    got = np.ctypeslib.as_array(col.out)[:col.n]
    assert [(int(b), int(p)) for _, b, p in got] == [(b, p) for _, b, p in ref]


def test_collects_compose(rb, page512):
    """A frame's request set from a cone, a box and points lists each brick
    once, under its first collect, and sorts as one list."""
    eye, fwd, ht, pc = (0.5, 0.5, -1.2), (0.0, 0.0, 1.0), 0.66, 2 * 0.577 / 1080
    col = rb.StreamCollect(page512)
    col.cone(eye, fwd, ht, pc)
    n_cone = col.n
    col.box((0.3, 0.3, 0.3), (0.7, 0.7, 0.4), 0.6 / 512)
    col.point((0.5, 0.5, 0.35), 0)
    col.point((0.05, 0.9, 0.9), 1)
    got = col.sorted()
    assert col.n > n_cone
    bricks = got["brick"].tolist()
    assert len(set(bricks)) == len(bricks)
    cone = rb.stream_desired(page512, eye, fwd, ht, pc)
    assert set(cone["brick"].tolist()) <= set(bricks)
    keys = [(int(p), float(d), int(b)) for d, b, p in got]
    assert keys == sorted(keys)
    # the same collects through the restatements
    ref, seen = [(float(d), int(b), int(p)) for d, b, p in cone], set(cone["brick"].tolist())
    _box_restated(page512, (0.3, 0.3, 0.3), (0.7, 0.7, 0.4), 0.6 / 512, 0.0, ref, seen)
    _point_restated(page512, (0.5, 0.5, 0.35), 0, 0.0, ref, seen)
    _point_restated(page512, (0.05, 0.9, 0.9), 1, 0.0, ref, seen)
    assert sorted((p, d, b) for d, b, p in ref) == keys
