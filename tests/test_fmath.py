"""Accuracy of the project-written log2 / exp2 / pow (include/r3d_fmath.h)
against float64 numpy, on the CPU build.  The device build is checked bit
for bit against this one by the GPU tests."""
import numpy as np


def _ulp(x):
    return np.spacing(np.abs(x).astype(np.float32)).astype(np.float64)


def test_log2_exp2_pow_accuracy(orc):
    rng = np.random.default_rng(1)
    x = np.concatenate([rng.uniform(1e-6, 1, 200000), rng.uniform(1, 4096, 200000),
                        np.float32(2.0) ** np.arange(-126, 127)]).astype(np.float32)
    y = rng.uniform(0.01, 12, x.size).astype(np.float32)
    out = orc.fmath_eval(x, y)
    ref_log = np.log2(x.astype(np.float64))
    err = np.abs(out[:, 0] - ref_log) / np.maximum(_ulp(ref_log), 1e-45)
    assert err[ref_log != 0].max() <= 4.0
    assert np.all(out[-253:, 0] == np.arange(-126, 127))  # exact at powers of two
    xe = rng.uniform(-30, 30, 200000).astype(np.float32)
    oe = orc.fmath_eval(xe, xe)[:, 1]
    ref = np.exp2(xe.astype(np.float64))
    assert (np.abs(oe - ref) / _ulp(ref)).max() <= 1.0
    ints = np.arange(-126, 128, dtype=np.float32)
    assert np.all(orc.fmath_eval(ints, ints)[:, 1] == np.float32(2.0) ** ints)
    # pow(x, y) = exp2(y log2 x): relative error grows with |y log2 x|
    xp = rng.uniform(0.001, 1, 100000).astype(np.float32)
    yp = rng.uniform(0.1, 8, 100000).astype(np.float32)
    op = orc.fmath_eval(xp, yp)[:, 2]
    rp = np.power(xp.astype(np.float64), yp.astype(np.float64))
    bound = 4e-7 * (1 + np.abs(yp * np.log2(xp)))
    assert np.all(np.abs(op - rp) / rp <= bound)
    # special values
    sp = orc.fmath_eval(np.array([0, 1, 0.5], np.float32), np.array([2, 3, 0], np.float32))
    assert sp[0, 0] == -np.inf and sp[1, 0] == 0 and sp[0, 2] == 0 and sp[1, 2] == 1
    assert sp[2, 2] == 1 and sp[1, 1] == 2


def test_powi24(orc):
    x = np.linspace(0, 1, 10001, dtype=np.float32)
    o = orc.fmath_eval(x, x)[:, 3]
    ref = x.astype(np.float64) ** 24
    # five roundings, amplified by the squarings: well under 24 ulp relative
    m = ref > 1e-30
    assert np.all(np.abs(o[m] - ref[m]) / ref[m] <= 24 * 2.0 ** -24)
    assert np.all(np.abs(o[~m]) <= 1e-29)
