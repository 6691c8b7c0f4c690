"""The differentiable raycast on the GPU: forward bit-exact with the FP32
oracle, adjoint within 1e-4 relative L2 of the FP64 oracle (voxels, LUT,
density scale) for every checkpoint interval, deterministic mode
bit-reproducible, and the autograd wrapper consistent with the C-ABI."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))


@pytest.fixture(scope="module")
def scene(rb):
    import torch
    rng = np.random.default_rng(2)
    n = 64
    vol = rb.phantom(n, seed=8).astype(np.float32) / 255.0
    vol += rng.normal(0, 10 / 255, vol.shape).astype(np.float32)
    lut = rb.scroll_ramp_tf().astype(np.float32) / 255.0
    views = [rb.camera_view(0.4 + 1.3 * i, -0.35 + 0.2 * i, 2.0, 96, 72, rb.scroll_ramp_tf(),
                            step_voxels=0.5, max_mip=0.0, frame_index=i) for i in range(3)]
    views[1].view_flags = rb.VIEW_ORTHO
    for a in range(3):
        views[1].cam_right[a] *= 0.7 / math.tan(math.pi / 6) / (96 / 72)
        views[1].cam_up[a] *= 0.7 / math.tan(math.pi / 6)
    views[2].density = 1.4
    return {"vol": vol, "lut": lut, "views": views,
            "dvol": torch.tensor(vol, device="cuda"), "dlut": torch.tensor(lut, device="cuda")}


def test_diff_forward_bit_exact(rb, orc, ctx, scene):
    import torch
    ctx.set_alpha_cutoff(0.98)
    n = sum(v.viewport[0] * v.viewport[1] * 3 for v in scene["views"])
    rgb = torch.zeros(n, dtype=torch.float32, device="cuda")
    ctx.diff_forward(scene["dvol"], scene["dlut"], scene["views"], rgb, stream=ctx.stream)
    torch.cuda.synchronize()
    got = rgb.cpu().numpy()
    off = 0
    for v in scene["views"]:
        ref, _ = orc.diff_forward32(v, scene["vol"], scene["lut"], 0.98)
        m = ref.size
        assert np.array_equal(got[off:off + m].reshape(ref.shape), ref)
        off += m


@pytest.mark.parametrize("k", [32, 64, 128])
@pytest.mark.parametrize("det", [False, True])
def test_adjoint_vs_fp64_oracle(rb, orc, ctx, scene, k, det):
    import torch
    ctx.set_alpha_cutoff(0.98)
    rng = np.random.default_rng(5)
    views = scene["views"]
    sizes = [v.viewport[0] * v.viewport[1] * 3 for v in views]
    g = rng.normal(0, 1, sum(sizes)).astype(np.float32)
    dg = torch.tensor(g, device="cuda")
    gd = torch.zeros_like(scene["dvol"])
    gl = torch.zeros_like(scene["dlut"])
    gs = torch.zeros(1, dtype=torch.float32, device="cuda")
    ctx.raycast_bwd(scene["dvol"], scene["dlut"], views, dg, gd, gl, gs, k, det,
                    stream=ctx.stream)
    torch.cuda.synchronize()
    rd = np.zeros(scene["vol"].shape)
    rl = np.zeros((256, 4))
    rs = 0.0
    off = 0
    for v, sz in zip(views, sizes):
        gv = g[off:off + sz].reshape(v.viewport[1], v.viewport[0], 3)
        _, d, l, s = orc.diff_grad64(v, scene["vol"], scene["lut"], gv, 0.98, decisions32=True)
        rd += d
        rl += l
        rs += s
        off += sz
    assert np.linalg.norm(rd) > 0 and np.linalg.norm(rl) > 0
    assert _rel(gd.cpu().numpy(), rd) < 1e-4
    assert _rel(gl.cpu().numpy(), rl) < 1e-4
    assert abs(gs.item() - rs) <= 1e-4 * abs(rs)


def test_deterministic_mode_reproducible(rb, ctx, scene):
    import torch
    views = scene["views"]
    n = sum(v.viewport[0] * v.viewport[1] * 3 for v in views)
    dg = torch.randn(n, device="cuda", generator=torch.Generator("cuda").manual_seed(3))
    outs = []
    for _ in range(2):
        gd = torch.zeros_like(scene["dvol"])
        gl = torch.zeros_like(scene["dlut"])
        gs = torch.zeros(1, device="cuda")
        ctx.raycast_bwd(scene["dvol"], scene["dlut"], views, dg, gd, gl, gs, 64, True,
                        stream=ctx.stream)
        torch.cuda.synchronize()
        outs.append((gd.clone(), gl.clone(), gs.clone()))
    for a, b in zip(outs[0], outs[1]):
        assert torch.equal(a, b)


def test_autograd_wrapper(rb, ctx, scene):
    import torch
    from diff_autograd import render
    views = scene["views"][:2]
    dens = scene["dvol"].clone().requires_grad_(True)
    lut = scene["dlut"].clone().requires_grad_(True)
    scale = torch.tensor(1.0, device="cuda", requires_grad=True)
    rgb = render(ctx, dens, lut, scale, views)
    target = (rgb.detach() * 0.8).contiguous()
    loss = ((rgb - target) ** 2).sum()
    loss.backward()
    # same gradients through the C-ABI directly
    g = (2 * (rgb.detach() - target)).contiguous()
    gd = torch.zeros_like(dens)
    gl = torch.zeros_like(lut)
    gs = torch.zeros(1, device="cuda")
    vs = [v.copy() for v in views]
    for v in vs:
        v.density = 1.0
    ctx.raycast_bwd(dens.detach(), lut.detach(), vs, g, gd, gl, gs, 32, True, stream=ctx.stream)
    torch.cuda.synchronize()
    assert torch.allclose(dens.grad, gd, rtol=1e-5, atol=1e-7)
    assert torch.allclose(lut.grad, gl, rtol=1e-5, atol=1e-7)
    assert abs(scale.grad.item() - gs.item()) <= 1e-5 * max(1.0, abs(gs.item()))


def test_adam_reduces_loss(rb, ctx, scene):
    """A few Adam steps on a perturbed grid move it toward the target."""
    import torch
    from diff_autograd import render
    views = scene["views"]
    clean = torch.tensor(rb.phantom(64, seed=8).astype(np.float32) / 255.0, device="cuda")
    with torch.no_grad():
        target = render(ctx, clean, scene["dlut"], torch.tensor(1.0, device="cuda"), views)
    dens = scene["dvol"].clone().requires_grad_(True)
    opt = torch.optim.Adam([dens], lr=3e-3)
    losses = []
    for _ in range(15):
        opt.zero_grad()
        rgb = render(ctx, dens, scene["dlut"], torch.tensor(1.0, device="cuda"), views)
        loss = ((rgb - target) ** 2).sum()
        loss.backward()
        opt.step()
        losses.append(loss.item())
    assert losses[-1] < 0.7 * losses[0]


def _bwd(ctx, dvol, dlut, views, dg, k, det, tape):
    import torch
    gd = torch.zeros_like(dvol)
    gl = torch.zeros_like(dlut)
    gs = torch.zeros(1, device="cuda")
    ctx.raycast_bwd(dvol, dlut, views, dg, gd, gl, gs, k, det, stream=ctx.stream, tape=tape)
    torch.cuda.synchronize()
    return gd, gl, gs


@pytest.mark.parametrize("faint", [False, True])
def test_tape_backward_equals_checkpoint_backward(rb, orc, ctx, scene, faint):
    """The tape of a training forward replaces the backward's forward sweep
    without changing a bit of the deterministic gradients.  faint: a LUT
    whose alpha is 0.01 everywhere makes every sample contribute (hundreds
    per ray), so most rays overflow the 64-entry tape and take the
    checkpoint path inside the same launch."""
    import torch
    ctx.set_alpha_cutoff(0.98)
    views = scene["views"]
    lut = scene["lut"].copy()
    if faint:
        lut[:, 3] = 0.01
    dlut = torch.tensor(lut, device="cuda")
    n = sum(v.viewport[0] * v.viewport[1] * 3 for v in views)
    rgb = torch.zeros(n, device="cuda")
    ctx.diff_forward(scene["dvol"], dlut, views, rgb, stream=ctx.stream, tape=True)
    dg = torch.randn(n, device="cuda", generator=torch.Generator("cuda").manual_seed(11))
    for k in (32, 64):
        a = _bwd(ctx, scene["dvol"], dlut, views, dg, k, True, tape=False)
        b = _bwd(ctx, scene["dvol"], dlut, views, dg, k, True, tape=True)
        for x, y in zip(a, b):
            assert torch.equal(x, y), f"k={k}"
    fa = _bwd(ctx, scene["dvol"], dlut, views, dg, 64, False, tape=True)
    assert torch.allclose(fa[0], a[0], rtol=1e-4, atol=1e-6)
    # and against the FP64 oracle
    g = dg.cpu().numpy()
    rd = np.zeros(scene["vol"].shape)
    off = 0
    for v in views:
        sz = v.viewport[0] * v.viewport[1] * 3
        gv = g[off:off + sz].reshape(v.viewport[1], v.viewport[0], 3)
        rd += orc.diff_grad64(v, scene["vol"], lut, gv, 0.98, decisions32=True)[1]
        off += sz
    assert _rel(b[0].cpu().numpy(), rd) < 1e-4


def test_tape_must_match(rb, ctx, scene):
    import torch
    views = scene["views"]
    n = sum(v.viewport[0] * v.viewport[1] * 3 for v in views)
    rgb = torch.zeros(n, device="cuda")
    ctx.diff_forward(scene["dvol"], scene["dlut"], views, rgb, stream=ctx.stream, tape=True)
    dg = torch.ones(n, device="cuda")
    other = [v.copy() for v in views]
    other[0].frame_index += 1
    with pytest.raises(rb.R3DError):
        _bwd(ctx, scene["dvol"], scene["dlut"], other, dg, 64, True, tape=True)
    lut2 = scene["dlut"].clone()
    with pytest.raises(rb.R3DError):
        _bwd(ctx, scene["dvol"], lut2, views, dg, 64, True, tape=True)
    _bwd(ctx, scene["dvol"], scene["dlut"], views, dg, 64, True, tape=True)
