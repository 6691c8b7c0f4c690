"""The oracle's display filter (src/shaders/postfilt.comp) on the CPU against
independent implementations: scipy.ndimage's median and maximum filters
with edge replication (the shader's clamp to the slot) and a float32
numpy restatement of the unsharp pass, on seeded slots with structure,
noise and saturated voxels; then the two-pass mode words (primary, then
unsharp) and the ids that select nothing."""
import numpy as np
import pytest
from scipy import ndimage

f32 = np.float32


def _slots(n=2, seed=3):
    rng = np.random.default_rng(seed)
    z, y, x = np.mgrid[0:128, 0:128, 0:128].astype(np.float32)
    base = 120 + 80 * np.sin(x / 9.0) * np.cos(y / 13.0) + 30 * np.sin(z / 7.0)
    out = []
    for k in range(n):
        v = base + rng.normal(0, 25, base.shape)
        v[rng.random(base.shape) < 0.01] = 255  # salt
        v[rng.random(base.shape) < 0.01] = 0  # pepper
        out.append(np.clip(np.rint(v), 0, 255).astype(np.uint8))
    return np.stack(out)


def _unsharp(s, amount):
    """centre + amount * (centre - sum / 27), the sum taken in the shader's
    order over byte / 255 floats, stored as round(255 v) (half up)."""
    v = s.astype(np.float32) / f32(255.0)
    p = np.pad(v, 1, mode="edge")
    acc = np.zeros_like(v)
    for dz in range(3):
        for dy in range(3):
            for dx in range(3):
                acc = acc + p[dz:dz + 128, dy:dy + 128, dx:dx + 128]
    out = np.clip(v + f32(amount) * (v - acc / f32(27.0)), f32(0), f32(1))
    return np.floor(out * f32(255.0) + f32(0.5)).astype(np.uint8)


@pytest.fixture(scope="module")
def slots():
    return _slots()


@pytest.mark.parametrize("mode,size,kind", [(1, 3, "median"), (2, 5, "median"), (3, 3, "max"),
                                            (4, 5, "max")])
def test_primary_filters(orc, slots, mode, size, kind):
    got = orc.postfilter(slots, mode)
    f = ndimage.median_filter if kind == "median" else ndimage.maximum_filter
    for k in range(slots.shape[0]):
        want = f(slots[k], size=size, mode="nearest")
        assert np.array_equal(got[k], want), (mode, k)
    assert not np.array_equal(got, slots)


@pytest.mark.parametrize("amount", [0.6, 2.5])
def test_unsharp(orc, slots, amount):
    got = orc.postfilter(slots[:1], 0x100, amount)
    want = _unsharp(slots[0], amount)
    # the float sum and the 1/27 division match the restatement bit for bit
    assert np.array_equal(got[0], want)


def test_median_then_unsharp_and_no_ops(orc, slots):
    got = orc.postfilter(slots[:1], 0x101, 1.0)
    want = _unsharp(ndimage.median_filter(slots[0], size=3, mode="nearest"), 1.0)
    assert np.array_equal(got[0], want)
    for mode in (0, 5, 0xFF, 0x200):  # no primary id, no unsharp bit
        assert np.array_equal(orc.postfilter(slots[:1], mode), slots[:1])
