"""Central finite differences against the FP64 adjoint of the differentiable
render (CPU): 512 random voxels with a nonzero gradient, every LUT entry with
a nonzero gradient, and the density scale; h = 1e-2.

The render has discrete decisions -- the 0.003 contribution floor and the
opacity cutoff -- at which the loss jumps, so the differences are taken with
the decisions of the unperturbed render held fixed (the branch the adjoint
differentiates), once with early termination disabled and once at the
reference cutoff 0.98.  The TF is smooth (quadratic alpha) and keeps alpha
inside [0.02, 0.88], so neither its piecewise-linear texels nor the alpha
clamp add kinks larger than the O(h^2) error."""
import math

import numpy as np


import pytest


@pytest.mark.parametrize("cut", [2.0, 0.98])
def test_fd_matches_fp64_adjoint(rb, orc, cut):
    rng = np.random.default_rng(0)
    n = 24
    vol = rb.phantom(n, seed=4).astype(np.float32) / 255.0
    vol += rng.normal(0, 10 / 255, vol.shape).astype(np.float32)
    i = np.arange(256, dtype=np.float32)
    lut = np.stack([i / 255, 0.8 * i / 255, 0.6 * i / 255,
                    0.02 + 0.86 * (i / 255) ** 2], axis=1).astype(np.float32)
    p = rb.camera_view(0.6, -0.5, 2.0, 16, 12, rb.scroll_ramp_tf(), step_voxels=0.5,
                       max_mip=0.0)
    p.density = 1.3
    img, _ = orc.diff_forward32(p, vol, lut, cut)
    target = (img * 0.9).astype(np.float64)

    def loss(v, lt, dens=None):
        q = p.copy()
        if dens is not None:
            q.density = dens
        rgb = orc.diff_grad64(q, v, lt, np.zeros_like(img), cut, decisions32=True,
                              dec_dens=vol, dec_lut=lut)[0]
        return float(((rgb - target) ** 2).sum())

    rgb = orc.diff_grad64(p, vol, lut, np.zeros_like(img), cut, decisions32=True)[0]
    g = (2 * (rgb - target)).astype(np.float32)
    _, gd, gl, gs = orc.diff_grad64(p, vol, lut, g, cut, decisions32=True)
    h = 1e-2
    nz = np.nonzero(np.abs(gd.ravel()) > 0)[0]
    pick = rng.choice(nz, min(512, nz.size), replace=False)
    e = []
    for j in pick:
        a = vol.copy().ravel()
        b = vol.copy().ravel()
        a[j] += h
        b[j] -= h
        e.append((gd.ravel()[j], (loss(a.reshape(vol.shape), lut) -
                                  loss(b.reshape(vol.shape), lut)) / (2 * h)))
    e = np.array(e)
    assert np.linalg.norm(e[:, 0] - e[:, 1]) / np.linalg.norm(e[:, 1]) < 1e-2  # O(h^2) truncation at h = 1e-2
    e = []
    for j in np.nonzero(np.abs(gl.ravel()) > 0)[0]:
        a = lut.copy().ravel()
        b = lut.copy().ravel()
        a[j] += h
        b[j] -= h
        e.append((gl.ravel()[j], (loss(vol, a.reshape(256, 4)) - loss(vol, b.reshape(256, 4))) /
                  (2 * h)))
    e = np.array(e)
    assert len(e) > 50
    assert np.linalg.norm(e[:, 0] - e[:, 1]) / np.linalg.norm(e[:, 1]) < 1e-2  # O(h^2) truncation at h = 1e-2
    fd = (loss(vol, lut, p.density + h) - loss(vol, lut, p.density - h)) / (2 * h)
    assert abs(gs - fd) <= 1e-2 * abs(fd)
