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
