"""The differentiable render's exact skip of samples that cannot contribute.

A sample contributes only when its opacity exceeds 0.003.  When both TF
texels of its density have alpha 0 (the TF's clear prefix), the opacity is
1 - 1^k = 0, so the forward and the backward's re-march skip the TF lookup
and the opacity.  The skip must leave every output bit unchanged: the
forward is compared with the FP32 oracle bit for bit and the adjoint with
the FP64 oracle, for LUTs whose clear prefix is empty (alpha above 0 from
texel 0, or negative alpha, which is not 0), 41 texels (the scroll TF),
120 texels (inside the papyrus density range, so that many samples fall on
both sides of the prefix's end) and the whole table, over the noisy 64^3
phantom of the other adjoint tests (its noise also takes air densities under
the low cut at 0).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))


def _lut(rb, kind):
    lut = rb.scroll_ramp_tf().astype(np.float32) / 255.0
    if kind == "none_clear":  # alpha > 0 from texel 0
        lut[:, 3] = np.maximum(lut[:, 3], 0.004)
    elif kind == "negative_head":  # negative alpha is not 0: no clear prefix
        lut[:20, 3] = -0.05
    elif kind == "long_clear":  # alpha 0 below texel 120
        lut[:120, 3] = 0.0
        lut[120:, 3] = np.maximum(lut[120:, 3], 0.05)
    elif kind == "all_clear":
        lut[:, 3] = 0.0
    return lut


@pytest.fixture(scope="module")
def grid(rb):
    rng = np.random.default_rng(2)
    n = 64
    vol = rb.phantom(n, seed=8).astype(np.float32) / 255.0
    vol += rng.normal(0, 10 / 255, vol.shape).astype(np.float32)
    views = [rb.camera_view(0.4 + 1.3 * i, -0.35 + 0.2 * i, 2.0, 96, 72, rb.scroll_ramp_tf(),
                            step_voxels=0.5, max_mip=0.0, frame_index=i) for i in range(3)]
    views[2].density = 1.4
    return vol, views


@pytest.mark.parametrize("kind", ["scroll", "none_clear", "negative_head", "long_clear",
                                  "all_clear"])
def test_forward_and_adjoint_with_clear_prefix(rb, orc, ctx, grid, kind):
    import torch
    vol, views = grid
    lut = _lut(rb, kind)
    dvol = torch.tensor(vol, device="cuda")
    dlut = torch.tensor(lut, device="cuda")
    ctx.set_alpha_cutoff(0.98)
    sizes = [v.viewport[0] * v.viewport[1] * 3 for v in views]
    rgb = torch.zeros(sum(sizes), device="cuda")
    ctx.diff_forward(dvol, dlut, views, rgb, stream=ctx.stream, tape=True)
    torch.cuda.synchronize()
    got = rgb.cpu().numpy()
    off = 0
    for v, sz in zip(views, sizes):
        ref, _ = orc.diff_forward32(v, vol, lut, 0.98)
        assert np.array_equal(got[off:off + sz].reshape(ref.shape), ref), kind
        off += sz
    g = np.random.default_rng(7).normal(0, 1, sum(sizes)).astype(np.float32)
    dg = torch.tensor(g, device="cuda")
    rd = np.zeros(vol.shape)
    rl = np.zeros((256, 4))
    off = 0
    for v, sz in zip(views, sizes):
        gv = g[off:off + sz].reshape(v.viewport[1], v.viewport[0], 3)
        _, d, lg, _ = orc.diff_grad64(v, vol, lut, gv, 0.98, decisions32=True)
        rd += d
        rl += lg
        off += sz
    for tape in (True, False):
        gd = torch.zeros_like(dvol)
        gl = torch.zeros_like(dlut)
        gs = torch.zeros(1, device="cuda")
        ctx.raycast_bwd(dvol, dlut, views, dg, gd, gl, gs, 32, True, stream=ctx.stream,
                        tape=tape)
        torch.cuda.synchronize()
        if kind == "all_clear":  # nothing contributes: no gradient at all
            assert not gd.any() and not gl.any() and gs.item() == 0.0
            assert np.linalg.norm(rd) == 0.0
            continue
        assert np.linalg.norm(rd) > 0
        assert _rel(gd.cpu().numpy(), rd) < 1e-4
        assert _rel(gl.cpu().numpy(), rl) < 1e-4
