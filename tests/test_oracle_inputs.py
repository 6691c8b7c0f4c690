"""The benchmark's inputs as the oracle builds them -- seeded scroll phantom,
scroll TF, scripted orbit views -- equal the library's bit for bit, so the
CPU baseline (which builds its own, without loading the library under test)
renders exactly the workload the GPU renders."""
import numpy as np


def test_phantom_equal(rb, orc):
    for shape, seed in (((40, 33, 21), 5), (96, 1234), ((300, 17, 9), 77)):
        assert np.array_equal(orc.phantom(shape, seed=seed), rb.phantom(shape, seed=seed))


def test_scroll_tf_equal(rb, orc):
    assert np.array_equal(orc.scroll_ramp_tf(), rb.scroll_ramp_tf())


def test_orbit_views_equal(rb, orc):
    lut = rb.scroll_ramp_tf()
    for i in range(0, 240, 7):
        for w, h in ((1920, 1080), (512, 512), (3840, 2160)):
            kw = dict(step_voxels=0.5, mode=i % 6, frame_index=i, lod_bias=0.5 * (i % 3),
                      low_cut=float(i % 50))
            p = rb.orbit_view(i / 120, w, h, lut, **kw)
            q = orc.orbit_view(i / 120, w, h, lut, **kw)
            assert bytes(p) == bytes(q), (i, w, h)
