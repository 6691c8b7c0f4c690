"""The LOD-brick kernels' fetch elision decides on the byte m of a block
maximum (and of a fetched sample's bytes) with integer compares against two
per-view counts.  Each count must equal the number of bytes whose bound
vub = (float)m / 255 satisfies the float decision the march restates
(raycast.slang:826-869,892-894): below the threshold, below the skip gate,
inside the TF's clear prefix, at most the depth mode's hit level.  Here the
host function the launches use is checked against all 256 byte values, in
float32 arithmetic, over random views and the edges (NaN and infinite
thresholds, TFs clear nowhere or everywhere).  No GPU is needed."""
import ctypes as C

import numpy as np

INV255 = np.float32(1.0) / np.float32(255.0)


def _vub():
    return np.arange(256, dtype=np.float32) * INV255


def _tf_clear(v: np.ndarray, z: float) -> np.ndarray:
    # clamp(fmaf(v, 256, -0.5), 0, 255) < z: the product and the sum are
    # exact in float64, so rounding once to float32 is fmaf
    t = (v.astype(np.float64) * 256.0 - 0.5).astype(np.float32)
    return np.fmin(np.fmax(t, np.float32(0)), np.float32(255)) < np.float32(z)


def _expected(threshold: float, skip_gate: float, mode: int, tf_zero_t: float):
    v = _vub()
    thr = np.float32(threshold)
    # fmaxf: a NaN operand yields the other one (np.fmax)
    bgate = np.fmax(np.fmax(np.float32(skip_gate), np.float32(0.5) / np.float32(255)),
                    np.float32(4.5) / np.float32(255))
    n_cut = int((v < thr).sum())
    n_void = max(n_cut, int((v < bgate).sum()))
    n_dec = n_cut
    if mode in (0, 5):  # FULL, FLAT
        n_dec = max(n_cut, int(_tf_clear(v, tf_zero_t).sum()))
    elif mode == 2:  # DEPTH
        n_dec = max(n_cut, int((v <= np.float32(0.05)).sum()))
    return n_void, n_dec


def _counts(rb, threshold, skip_gate, mode, tf_zero_t):
    p = rb.FrameParams()
    p.threshold, p.skip_gate, p.mode = threshold, skip_gate, mode
    out = (C.c_uint32 * 2)()
    rb.lib.r3d_cuda_elide_counts(C.byref(p), C.c_float(tf_zero_t), out)
    return out[0], out[1]


def test_counts_match_every_byte(rb):
    rng = np.random.default_rng(11)
    cases = []
    for _ in range(400):
        cases.append((float(rng.uniform(0, 1)), float(rng.uniform(0, 0.5)),
                      int(rng.integers(0, 6)), float(rng.integers(-1, 256))))
    # thresholds and gates on byte boundaries, where the decision flips
    for m in (0, 1, 39, 40, 41, 127, 128, 254, 255):
        x = float(np.float32(m) * INV255)
        for mode in (0, 1, 2, 3, 5):
            cases += [(x, 0.0, mode, 39.0), (0.0, x, mode, float(m)),
                      (float(np.nextafter(np.float32(x), np.float32(1))), 0.0, mode, 255.0)]
    # edges: no threshold, everything cut, a NaN or infinite threshold, a
    # TF opaque from 0 (clear prefix empty) or clear everywhere
    for mode in (0, 1, 2, 3, 5):
        cases += [(0.0, 0.0, mode, -1.0), (1.0, 0.0, mode, 255.0), (2.0, 1.0, mode, 0.0),
                  (float("nan"), 0.0, mode, 40.0), (float("inf"), 0.0, mode, 40.0),
                  (float("-inf"), float("nan"), mode, 40.0)]
    for thr, gate, mode, z in cases:
        got = _counts(rb, thr, gate, mode, z)
        want = _expected(thr, gate, mode, z)
        assert got == want, f"threshold {thr} gate {gate} mode {mode} tf_zero_t {z}: " \
                            f"{got} != {want}"
