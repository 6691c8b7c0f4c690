"""The adjoint at the sizes of the differentiable workloads.

* 256^3 FP32 density (scroll phantom / 255 + N(0, 10/255), seeded), the
  scroll TF as FP32, 64 orbit views of 256x256 at step 0.5, L2 loss against
  the unperturbed phantom's render: GPU gradients (voxels, LUT, density
  scale) against the FP64 oracle over all 64 views for both accumulation
  modes, with and without the tape; central finite differences of the GPU
  forward on 512 seeded voxels (h = 1e-2), every LUT entry with a gradient
  and the density scale (h = 1e-3), against the GPU gradient.
* 512^3 FP32 density, 16 orbit views of 512x512 at step 0.25: checkpoint
  intervals K = 32, 64, 128 in atomic and deterministic accumulation, each
  against the FP64 oracle, and deterministic against atomic.  Once with the
  scroll TF at the 0.98 cutoff, and once with a faint TF (alpha 0.013
  everywhere) and no early termination, where every sample contributes --
  past 2000 on the longest rays -- and the gradient comes from the
  checkpoints, not from the 64-entry ring.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))


def _views(rb, n, w, step):
    lut8 = rb.scroll_ramp_tf()
    vs = [rb.orbit_view(i / n, w, w, lut8, step_voxels=step, frame_index=i) for i in range(n)]
    for v in vs:
        v.max_mip = 0.0
    return vs


def _density(rb, n, seed):
    clean = rb.phantom(n, seed=seed).astype(np.float32) / 255.0
    rng = np.random.default_rng(seed)
    noisy = clean + rng.normal(0.0, 10.0 / 255.0, clean.shape).astype(np.float32)
    return clean, noisy


def _nf(views):
    return sum(v.viewport[0] * v.viewport[1] * 3 for v in views)


def _oracle(orc, views, vol, lut, g, cutoff):
    """FP64 gradients summed over the views (decisions of the FP32 render)."""
    rd = np.zeros(vol.shape)
    rl = np.zeros((256, 4))
    rs = 0.0
    off = 0
    for v in views:
        sz = v.viewport[0] * v.viewport[1] * 3
        gv = g[off:off + sz].reshape(v.viewport[1], v.viewport[0], 3)
        _, d, lg, s = orc.diff_grad64(v, vol, lut, gv, cutoff, decisions32=True)
        rd += d
        rl += lg
        rs += s
        off += sz
    return rd, rl, rs


def _bwd(ctx, dvol, dlut, views, dg, k, det, tape):
    import torch
    gd = torch.zeros_like(dvol)
    gl = torch.zeros_like(dlut)
    gs = torch.zeros(1, device="cuda")
    ctx.raycast_bwd(dvol, dlut, views, dg, gd, gl, gs, k, det, stream=ctx.stream, tape=tape)
    torch.cuda.synchronize()
    return gd, gl, gs


def _check(got, ref):
    gd, gl, gs = got
    rd, rl, rs = ref
    assert np.linalg.norm(rd) > 0 and np.linalg.norm(rl) > 0
    assert _rel(gd.cpu().numpy(), rd) < 1e-4
    assert _rel(gl.cpu().numpy(), rl) < 1e-4
    assert abs(gs.item() - rs) <= 1e-4 * abs(rs)


@pytest.fixture(scope="module")
def cfg256(rb):
    import torch
    clean, noisy = _density(rb, 256, 1234)
    lut = rb.scroll_ramp_tf().astype(np.float32) / 255.0
    return {"clean": torch.tensor(clean, device="cuda"), "vol": noisy,
            "dvol": torch.tensor(noisy, device="cuda"), "lut": lut,
            "dlut": torch.tensor(lut, device="cuda"), "views": _views(rb, 64, 256, 0.5)}


def test_256_64views_vs_fp64(rb, orc, ctx, cfg256):
    import torch
    ctx.set_alpha_cutoff(0.98)
    views, n = cfg256["views"], _nf(cfg256["views"])
    target = torch.empty(n, device="cuda")
    rgb = torch.empty(n, device="cuda")
    ctx.diff_forward(cfg256["clean"], cfg256["dlut"], views, target, stream=ctx.stream)
    ctx.diff_forward(cfg256["dvol"], cfg256["dlut"], views, rgb, stream=ctx.stream, tape=True)
    torch.cuda.synchronize()
    dg = (2.0 * (rgb - target)).contiguous()
    ref = _oracle(orc, views, cfg256["vol"], cfg256["lut"], dg.cpu().numpy(), 0.98)
    for det in (True, False):
        _check(_bwd(ctx, cfg256["dvol"], cfg256["dlut"], views, dg, 64, det, tape=True), ref)
    _check(_bwd(ctx, cfg256["dvol"], cfg256["dlut"], views, dg, 64, True, tape=False), ref)


def test_256_64views_finite_differences(rb, ctx, cfg256):
    """Central differences of the GPU forward against the GPU adjoint.  The
    TF is smooth (quadratic alpha in [0.02, 0.88]): every sample contributes
    (no 0.003-floor decisions), its piecewise-linear texels add only O(h^2)
    kinks, the densities stay clear of the low cut and the TF clamp, and
    with the cutoff at 1 rays end only where their opacity rounds to 1, so
    no discrete decision that moves the loss changes under the
    perturbation."""
    import torch
    ctx.set_alpha_cutoff(1.0)
    try:
        views, n = cfg256["views"], _nf(cfg256["views"])
        i = np.arange(256, dtype=np.float32)
        lut = np.stack([i / 255, 0.8 * i / 255, 0.6 * i / 255,
                        0.02 + 0.86 * (i / 255) ** 2], axis=1).astype(np.float32)
        dlut = torch.tensor(lut, device="cuda")
        # densities kept inside [0.02, 0.98]: no sample of a perturbed voxel
        # crosses the low cut at 0 or the TF's clamp at 1
        dens = cfg256["dvol"].clamp(0.02, 0.98)
        target = torch.empty(n, device="cuda")
        rgb = torch.empty(n, device="cuda")
        ctx.diff_forward(cfg256["clean"], dlut, views, target, stream=ctx.stream)
        torch.cuda.synchronize()
        t64 = target.double()
        vs = [v.copy() for v in views]

        def loss(d, lt, scale=None):
            q = vs
            if scale is not None:
                q = [v.copy() for v in vs]
                for v in q:
                    v.density = scale
            ctx.diff_forward(d, lt, q, rgb, stream=ctx.stream)
            torch.cuda.synchronize()
            return float(((rgb.double() - t64) ** 2).sum().item())

        loss(dens, dlut)
        dg = (2.0 * (rgb - target)).contiguous()
        gd, gl, gs = _bwd(ctx, dens, dlut, vs, dg, 64, True, tape=False)
        h = 1e-2
        flat = dens.view(-1)
        g = gd.view(-1).cpu().numpy()
        rng = np.random.default_rng(0)
        pick = rng.choice(np.nonzero(np.abs(g) > 0)[0], 512, replace=False)
        e = []
        for j in pick:
            x = flat[j].item()
            hi, lo = np.float32(x + h), np.float32(x - h)
            flat[j] = float(hi)
            lp = loss(dens, dlut)
            flat[j] = float(lo)
            lm = loss(dens, dlut)
            flat[j] = x
            e.append((g[j], (lp - lm) / float(hi - lo)))
        e = np.array(e)
        assert _rel(e[:, 0], e[:, 1]) < 1e-2  # O(h^2) truncation at h = 1e-2
        # LUT entries (and the density scale) with h = 1e-3: an entry is shared
        # by every sample whose density falls in its texel, hundreds per ray in
        # the air, and a step of 1e-2 moves an air-range alpha (~0.02) by half
        # its value, far outside the range where the transmittance is
        # near-linear in it (measured: 4.8 % relative L2 at 1e-2, 0.05 % at
        # 1e-3)
        lflat = dlut.view(-1)
        gln = gl.view(-1).cpu().numpy()
        e = []
        hl = 1e-3
        for j in np.nonzero(np.abs(gln) > 0)[0]:
            x = lflat[j].item()
            hi, lo = np.float32(x + hl), np.float32(x - hl)
            lflat[j] = float(hi)
            lp = loss(dens, dlut)
            lflat[j] = float(lo)
            lm = loss(dens, dlut)
            lflat[j] = x
            e.append((gln[j], (lp - lm) / float(hi - lo)))
        e = np.array(e)
        assert len(e) > 500
        assert _rel(e[:, 0], e[:, 1]) < 1e-2
        s0 = vs[0].density  # the scale multiplies every sample's opacity exponent
        fd = (loss(dens, dlut, s0 + hl) - loss(dens, dlut, s0 - hl)) / (2 * hl)
        assert abs(gs.item() - fd) <= 1e-2 * abs(fd)
    finally:
        ctx.set_alpha_cutoff(0.98)


@pytest.mark.parametrize("faint", [False, True])
def test_512_16views_step025_checkpoints(rb, orc, ctx, faint):
    import torch
    _, noisy = _density(rb, 512, 77)
    lut = rb.scroll_ramp_tf().astype(np.float32) / 255.0
    if faint:
        lut[:, 3] = 0.013  # opacity 0.0033 per sample at step 0.25: every sample counts
    cutoff = 1.0 if faint else 0.98
    views = _views(rb, 16, 512, 0.25)
    n = _nf(views)
    dvol = torch.tensor(noisy, device="cuda")
    dlut = torch.tensor(lut, device="cuda")
    ctx.set_alpha_cutoff(cutoff)
    try:
        rgb = torch.empty(n, device="cuda")
        tot = torch.zeros(1, dtype=torch.int64, device="cuda")
        ctx.diff_forward(dvol, dlut, views, rgb, total=tot, stream=ctx.stream)
        torch.cuda.synchronize()
        if faint:  # every sample contributes: hundreds per ray on average (misses
            # included), past 2000 on the longest rays
            assert tot.item() / (n // 3) > 300
        dg = torch.randn(n, device="cuda", generator=torch.Generator("cuda").manual_seed(9))
        ref = _oracle(orc, views, noisy, lut, dg.cpu().numpy(), cutoff)
        dets = {}
        for k in (32, 64, 128):
            for det in (False, True):
                got = _bwd(ctx, dvol, dlut, views, dg, k, det, tape=False)
                _check(got, ref)
                if det:
                    dets[k] = got
                else:
                    atomic = got
            # deterministic against atomic accumulation of the same interval
            # (FP32 atomic sums: the same relative L2 bar as against FP64)
            for x, y in zip(dets[k][:2], atomic[:2]):
                assert _rel(y.cpu().numpy(), x.cpu().numpy().astype(np.float64)) < 1e-4
        # the interval changes where the backward re-marches, not the bits
        # of the deterministic sums
        assert torch.equal(dets[32][0], dets[128][0]) and torch.equal(dets[32][1], dets[128][1])
    finally:
        ctx.set_alpha_cutoff(0.98)
