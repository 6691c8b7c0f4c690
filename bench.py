#!/usr/bin/env python3
"""Benchmark of the sm_100a volume raycast on render3d's scale workload.

Workload: a 1024^3 u8 seeded scroll phantom split into 128^3 bricks with a
4-level (sum+4)/8 pyramid and render3d's page table, rendered at 1920x1080
with full gradient shading, ray-cone LOD (bias 0) and early termination at
opacity 0.99, along the 120-frame scripted orbit (frame i at phase
(i mod 120)/120).  One step = one frame.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

value: Gsamples/s (sum of per-ray march iterations / device time), inputs
resident in HBM.  e2e: the same metric through the render3d-facing API
(r3d_frame + r3d_read_frame into pinned host memory, params host->device and
the RGBA8 frame device->host every step), host wall clock.  --impl reference
times the CPU restatement of the reference shader (the reference's Slang
shader cannot be compiled here) on the host cores.  With --gpus N > 1 every
rank renders the orbit independently (the path has no exchange step:
replicas).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

W, H = 1920, 1080
N_EDGE = 1024
NLEV = 4
SEED = 1234
CUTOFF = 0.99
STEP_VOXELS = 0.5
ORBIT_FRAMES = 120
WORKLOAD = "scroll phantom 1024^3 u8, 128^3 bricks x 4 LOD levels, 1920x1080 full shading"
# One ncu capture (--clock-control none, 1 pass) of `python bench.py
# --profile 6`, launches 3 and 4 of k_raycast (orbit phases 2/120 and
# 3/120), the mean per launch of: DRAM bytes (dram__bytes_read.sum +
# dram__bytes_write.sum), warp instructions (smsp__inst_executed.sum) and
# thread instructions (smsp__thread_inst_executed.sum); and the samples of
# those two frames (the counters that `--profile` prints).
FWD_DRAM_TRAFFIC_BYTES = 238.8e6
FWD_WARP_INST = 282.6e6
FWD_THREAD_INST = 5.389e9
FWD_CAPTURED_SAMPLES = 28.31e6
METRIC = "raycast Gsamples/s & fps @1024^3 1080p; fwd+bwd Gsamples/s vs plain, same GPU"


def measured_peaks() -> tuple[float, str]:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """Samples nvidia-smi SM clocks and throttle reasons during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int, period_ms: int = 50):
        self.device = device
        self.period_ms = period_ms
        self.proc = None
        self.lines: list[str] = []
        self.t = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", str(self.period_ms)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            time.sleep(1.0)  # nvidia-smi's own start-up; sampling runs before the region
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            if self.t:
                self.t.join(timeout=2)

    def summary(self) -> dict:
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def reduce_replicas(dist, samples: float, ms: float, device) -> tuple[float, float]:
    """Whole-job totals of independent replicas: samples summed over ranks and
    the device time of the slowest rank."""
    import torch
    if dist is None:
        return samples, ms
    s = torch.tensor([samples], dtype=torch.float64, device=device)
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(s, op=dist.ReduceOp.SUM)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(s.item()), float(t.item())


def orbit_params(rb, lut, i: int, brick_mode: int, mode: int = 0):
    p = rb.orbit_view((i % ORBIT_FRAMES) / ORBIT_FRAMES, W, H, lut, step_voxels=STEP_VOXELS,
                      mode=mode, frame_index=i)
    p.brick_mode = brick_mode
    return p


def algorithmic_bytes(cnt: np.ndarray, pixels: int) -> float:
    """Bytes the march must read/write: 8 per trilinear sample, 6x8 for the
    gradient taps of a shaded sample, 8 per TF lookup (2 RGBA8 texels), 4
    per page-table walk and 4 per output pixel."""
    samples, tf, grad, walks = (float(x) for x in cnt)
    return 8.0 * samples + 48.0 * grad + 8.0 * tf + 4.0 * walks + 4.0 * pixels


def shard_bench(rb, torch, local: int, vol, lut, frames: int) -> dict:
    """The same phantom as a single-level brick atlas (render3d's bricks mode
    without LOD: a 1024^3 shard of 8^3 bricks, all resident in the identity
    layout, atlas mips 0..3), 1920x1080 FULL along the orbit."""
    c = rb.Context(local)
    try:
        c.set_transfer(lut)
        c.set_alpha_cutoff(CUTOFF)
        c.shard_build(vol)
        img = torch.zeros((H, W, 4), dtype=torch.uint8, device=f"cuda:{local}")
        tot = torch.zeros(1, dtype=torch.int64, device=f"cuda:{local}")
        st = torch.cuda.ExternalStream(c.stream, device=local)

        def frame(i):
            p = rb.orbit_view((i % ORBIT_FRAMES) / ORBIT_FRAMES, W, H, lut, step_voxels=STEP_VOXELS,
                              frame_index=i)
            p.brick_mode = c.shard_mode
            c.raycast(p, W, H, out=img, total=tot, stream=c.stream)
        for i in range(20):
            frame(i)
        torch.cuda.synchronize()
        tot.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for i in range(frames):
            frame(i)
        e1.record(st)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / frames
        return {"workload": "scroll phantom 1024^3 as a single-level shard (8^3 bricks, identity "
                            "layout, 4 atlas mips), 1920x1080 full shading",
                "brick_mode": c.shard_mode, "ms_per_frame": ms, "fps": 1e3 / ms,
                "gsamples_per_s": float(tot.item()) / frames / (ms * 1e-3) / 1e9}
    finally:
        c.close()


def overlay_bench(rb, ctx, lut, torch, stream, total, img, frames: int) -> dict:
    """The same orbit in FULL with two slot-parallel overlay atlases cut from
    seeded device phantoms (ink at gain 1.5, a second scan fused at weight
    128/255), per-frame event times."""
    ink = ctx.phantom(N_EDGE, seed=SEED + 7)
    ctx.overlay_build(0, ink)
    reg = ctx.phantom(N_EDGE, seed=SEED + 8)
    ctx.overlay_build(3, reg)
    del ink, reg
    torch.cuda.empty_cache()

    def frame(i):
        p = orbit_params(rb, lut, i, ctx.brick_mode)
        p.overlay_flags = 1 | 16 | (128 << 16)
        p.overlay_gain = 1.5
        ctx.raycast(p, W, H, out=img, total=total, stream=ctx.stream)
    for i in range(32):
        frame(i)
    torch.cuda.synchronize()
    total.zero_()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for i in range(frames):
        frame(i)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / frames
    ctx.overlay_load(0, None)
    ctx.overlay_load(3, None)
    return {"workload": "1024^3 orbit, FULL, ink + registration overlays", "ms_per_frame": ms,
            "fps": 1e3 / ms, "gsamples_per_s": float(total.item()) / frames / (ms * 1e-3) / 1e9}


def mode_stats(rb, ctx, lut, torch, stream, total, img, frames: int) -> dict:
    """Per-frame CUDA-event times (p50/p95/p99, like render3d's frame stats)
    and Gsamples/s of the orbit in FULL, MIP and HEATMAP modes, each after
    its own warm-up; each frame is bracketed by its own pair of events on the
    launching stream."""
    out = {}
    for name, mode in (("full", 0), ("mip", 1), ("heatmap", 3)):
        def frame(i):
            ctx.raycast(orbit_params(rb, lut, i, ctx.brick_mode, mode), W, H, out=img,
                        total=total, stream=ctx.stream)
        for i in range(32):
            frame(i)
        torch.cuda.synchronize()
        total.zero_()
        torch.cuda.synchronize()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(frames)]
        for i, (a, b) in enumerate(ev):
            a.record(stream)
            frame(i)
            b.record(stream)
        torch.cuda.synchronize()
        t = np.array([a.elapsed_time(b) for a, b in ev])
        out[name] = {"frames": frames, "p50_ms": float(np.percentile(t, 50)),
                     "p95_ms": float(np.percentile(t, 95)),
                     "p99_ms": float(np.percentile(t, 99)),
                     "gsamples_per_s": float(total.item()) / (t.sum() * 1e-3) / 1e9}
    return out


def fwd_bwd_bench(rb, ctx, torch, local: int, steps: int, adam_steps: int) -> dict:
    """Differentiable workload: a 256^3 FP32 density grid (scroll phantom / 255
    plus N(0, 10/255), seeded), the scroll TF as FP32, 64 orbit views of
    256x256 at step 0.5; L2 loss against the unperturbed phantom's render.
    Times forward + backward (deterministic fixed-point gradients, K = 64)
    per step; Gsamples/s counts the forward march's samples."""
    dev = f"cuda:{local}"
    n, nv, w = 256, 64, 256
    rng = np.random.default_rng(SEED)
    clean = rb.phantom(n, seed=SEED).astype(np.float32) / 255.0
    noisy = clean + rng.normal(0.0, 10.0 / 255.0, clean.shape).astype(np.float32)
    lut8 = rb.scroll_ramp_tf()
    lut = torch.tensor(lut8.astype(np.float32) / 255.0, device=dev)
    views = [rb.orbit_view(i / nv, w, w, lut8, step_voxels=0.5, frame_index=i) for i in range(nv)]
    for v in views:
        v.max_mip = 0.0
    nf = nv * w * w * 3
    st = torch.cuda.ExternalStream(ctx.stream, device=local)
    dclean = torch.tensor(clean, device=dev)
    dens = torch.tensor(noisy, device=dev)
    target = torch.empty(nf, device=dev)
    rgb = torch.empty(nf, device=dev)
    tot = torch.zeros(1, dtype=torch.int64, device=dev)
    ctx.set_alpha_cutoff(0.98)
    ctx.diff_forward(dclean, lut, views, target, stream=ctx.stream)
    ctx.diff_forward(dens, lut, views, rgb, total=tot, stream=ctx.stream)
    torch.cuda.synchronize()
    samples = float(tot.item())
    gd = torch.empty_like(dens)
    gl = torch.empty_like(lut)
    gs = torch.empty(1, device=dev)
    grad = torch.empty(nf, device=dev)

    def step(tape=True):
        # training forward (records the tape), loss gradient, adjoint
        ctx.diff_forward(dens, lut, views, rgb, stream=ctx.stream, tape=tape)
        with torch.cuda.stream(st):
            torch.sub(rgb, target, out=grad)
            grad.mul_(2.0)
        ctx.raycast_bwd(dens, lut, views, grad, gd, gl, gs, 64, True, stream=ctx.stream,
                        tape=tape)

    def timed(tape):
        for _ in range(3):
            step(tape)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(steps):
            step(tape)
        e1.record(st)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    ms_ck = timed(False)  # backward re-marches every ray from its checkpoints
    ms = timed(True)
    # 100 Adam steps on the voxels, LUT and density scale
    p_dens = dens.clone().requires_grad_(False)
    opt_state = [torch.zeros_like(p_dens), torch.zeros_like(p_dens)]
    loss0 = lossN = None
    t0 = time.perf_counter()
    b1, b2, lr, eps = 0.9, 0.999, 2e-3, 1e-8
    for it in range(1, adam_steps + 1):
        ctx.diff_forward(p_dens, lut, views, rgb, stream=ctx.stream, tape=True)
        with torch.cuda.stream(st):
            torch.sub(rgb, target, out=grad)
            loss = float((grad * grad).sum().item()) if it in (1, adam_steps) else None
            grad.mul_(2.0)
        ctx.raycast_bwd(p_dens, lut, views, grad, gd, gl, gs, 64, True, stream=ctx.stream,
                        tape=True)
        with torch.cuda.stream(st):
            m, v2 = opt_state
            m.mul_(b1).add_(gd, alpha=1 - b1)
            v2.mul_(b2).addcmul_(gd, gd, value=1 - b2)
            den = (v2 / (1 - b2 ** it)).sqrt_().add_(eps)
            p_dens.addcdiv_(m, den, value=-lr / (1 - b1 ** it))
        if it == 1:
            loss0 = loss
        if it == adam_steps:
            lossN = loss
    torch.cuda.synchronize()
    adam_s = time.perf_counter() - t0
    # the plain forward on the same 64 views: the u8 phantom (the clean
    # density's bytes) as a cube volume at level 0, FLAT compositing, the 64
    # views as 256x256 panes of one 2048x2048 image in one call
    pv = []
    for i, v in enumerate(views):
        q = v.copy()
        q.mode = rb.MODE_FLAT
        q.view_org = (w * (i % 8)) | ((w * (i // 8)) << 16)
        pv.append(q)
    ctx.upload_volume(rb.phantom(n, seed=SEED))
    ctx.set_schedule(persistent=2)  # one whole-tile launch drains the 64 small views
    pimg = torch.zeros((8 * w, 8 * w, 4), dtype=torch.uint8, device=dev)
    ptot = torch.zeros(1, dtype=torch.int64, device=dev)
    for _ in range(3):
        ctx.raycast(pv, 8 * w, 8 * w, out=pimg, stream=ctx.stream)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(steps):
        ctx.raycast(pv, 8 * w, 8 * w, out=pimg, total=ptot, stream=ctx.stream)
    e1.record(st)
    torch.cuda.synchronize()
    pms = e0.elapsed_time(e1) / steps
    ctx.set_schedule()
    plain = {"ms_per_step": pms,
             "gsamples_per_s": float(ptot.item()) / steps / (pms * 1e-3) / 1e9,
             "workload": "the same 64 views, u8 phantom as a cube volume, level 0, FLAT, "
                         "one whole-tile launch"}
    return {"plain_same_views": plain,
            "workload": "256^3 FP32 density (phantom/255 + N(0,10/255)), 64 orbit views 256x256, "
                        "step 0.5, L2 loss, tape of 64 contributions per ray (checkpoints "
                        "every 64 samples beyond it), deterministic",
            "value": samples / (ms * 1e-3) / 1e9, "unit": "Gsamples/s", "ms_per_step": ms,
            "ms_per_step_checkpoints_only": ms_ck,
            "samples_per_step": samples, "steps": steps,
            "adam": {"steps": adam_steps, "loss_first": loss0, "loss_last": lossN,
                     "s_per_step": adam_s / adam_steps}}


def batch_requests(rb, lut, rng, bm_scroll: int, bm_slab: int, slab_shape):
    """The 64 seeded requests of the batched workload: 16 perspective views of
    1920x1080 and 24 orthographic slice panes of 960x540 at arbitrary normals
    over the 1024^3 cache, and 24 slab windows of 3072x3072x32 over the
    3072x3072x96 slab cache."""
    persp, panes, slabs = [], [], []
    for i in range(16):
        p = rb.orbit_view(float(rng.uniform()), 1920, 1080, lut, step_voxels=STEP_VOXELS,
                          frame_index=i)
        p.brick_mode = bm_scroll
        persp.append(p)
    for i in range(24):
        n = rng.normal(size=3)
        n /= np.linalg.norm(n)
        up = np.cross(n, [1.0, 0.0, 0.0] if abs(n[0]) < 0.9 else [0.0, 1.0, 0.0])
        up /= np.linalg.norm(up)
        rt = np.cross(up, n)
        p = rb.camera_view(0.0, 0.0, 1.0, 960, 540, lut, step_voxels=STEP_VOXELS, frame_index=i)
        p.cam_origin[:] = (np.array([0.5, 0.5, 0.5]) - n * 1.0).tolist()
        p.cam_forward[:] = n.tolist()
        p.cam_right[:] = (rt * 0.6).tolist()
        p.cam_up[:] = (up * 0.6 * 540 / 960).tolist()
        p.view_flags = rb.VIEW_ORTHO | rb.VIEW_OBLIQUE
        p.slab_z0, p.slab_depth = float(rng.uniform(900, 1100)), 32
        p.brick_mode = bm_scroll
        panes.append(p)
    ext_y = slab_shape[1] / max(slab_shape)
    for i in range(24):
        p = rb.camera_view(0.0, 0.0, 1.0, 3072, 3072, lut, step_voxels=STEP_VOXELS, frame_index=i)
        p.cam_origin[:] = [0.5, 0.5 * ext_y, -0.5]
        p.cam_forward[:] = [0.0, 0.0, 1.0]
        p.cam_right[:] = [0.5, 0.0, 0.0]
        p.cam_up[:] = [0.0, 0.5 * ext_y, 0.0]
        p.view_flags = rb.VIEW_ORTHO | rb.VIEW_AXIS(0)
        p.slab_z0, p.slab_depth = float(rng.integers(0, slab_shape[2] - 32)), 32
        p.brick_mode = bm_slab
        slabs.append(p)
    return persp + panes, slabs


def batch_bench(rb, torch, local: int, ctx, reps: int) -> dict:
    """Batched heterogeneous views (64 requests) over two brick caches -- the
    1024^3 scroll cache and a 3072x3072x96 slab cache -- planned as ONE batch
    over both scenes, autotuned, captured into a CUDA graph and timed by
    graph replay.  The whole-tile schedule drains every request of both
    caches in one launch (one kernel node in the graph)."""
    dev = f"cuda:{local}"
    lut = rb.scroll_ramp_tf()
    slab_shape = (3072, 3072, 96)
    sctx = rb.Context(local)
    sctx.set_transfer(lut)
    sctx.set_alpha_cutoff(CUTOFF)
    slab = rb.phantom(slab_shape, seed=SEED + 1)
    sctx.bricks_build(slab, NLEV)
    del slab
    rng = np.random.default_rng(SEED)
    scroll_views, slab_views = batch_requests(rb, lut, rng, ctx.brick_mode, sctx.brick_mode,
                                              slab_shape)
    views = scroll_views + slab_views
    scenes = [ctx] * len(scroll_views) + [sctx] * len(slab_views)
    imgs = [torch.zeros((v.viewport[1], v.viewport[0], 4), dtype=torch.uint8, device=dev)
            for v in views]
    b = rb.Batch(ctx, views, imgs, scenes=scenes)
    sched, tune_ms = b.autotune(reps=2)
    # every candidate's time per launch, for the record
    cands = {}
    for name, sc in (("grid", dict(persistent=0)), ("whole_tiles", dict(persistent=2))):
        b.set_schedule(**sc)
        b.launch(stream=ctx.stream)
        st = torch.cuda.ExternalStream(ctx.stream, device=local)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(reps):
            b.launch(stream=ctx.stream)
        e1.record(st)
        torch.cuda.synchronize()
        cands[name] = e0.elapsed_time(e1) / reps
    b.set_schedule(**sched)
    tot = torch.zeros(1, dtype=torch.int64, device=dev)
    b.capture(total=tot, stream=ctx.stream)
    torch.cuda.synchronize()
    samples = float(tot.item())
    st = torch.cuda.ExternalStream(ctx.stream, device=local)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(reps):
        b.replay(stream=ctx.stream)
    e1.record(st)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    rays = sum(v.viewport[0] * v.viewport[1] for v in views)
    out = {"requests": len(views),
           "views": "16 persp 1080p + 24 ortho panes 960x540 over the 1024^3 cache, 24 slab "
                    "windows 3072x3072x32 over the 3072x3072x96 cache, one batch",
           "schedule": sched, "autotune_ms": tune_ms,
           "kernel_launches_per_replay": 1 if sched["persistent"] == 2 else len(views),
           "ms_per_launch_by_schedule": cands, "ms_per_batch": ms, "samples": samples,
           "rays": rays, "value": samples / (ms * 1e-3) / 1e9, "unit": "Gsamples/s"}
    b.close()
    del imgs
    sctx.close()
    return out


def noalloc_bench(rb, torch, ctx, lut, img, frames: int) -> dict:
    """The orbit through r3d_cuda_raycast_fwd_noalloc (no allocation per
    call; a persistent kernel with its scratch in a static device array)
    beside r3d_cuda_raycast_fwd, per-frame CUDA events on the same stream."""
    import ctypes as C
    st = torch.cuda.ExternalStream(ctx.stream)
    out = {}
    for name, sched in (("lane_refill", dict()), ("whole_tiles", dict(persistent=2))):
        ctx.set_schedule(**sched)

        def frame(i):
            arr = (rb.FrameParams * 1)(orbit_params(rb, lut, i, ctx.brick_mode))
            rc = rb.lib.r3d_cuda_raycast_fwd_noalloc(ctx.h, arr, 1, img.data_ptr(), W, H,
                                                     C.c_void_p(ctx.stream))
            assert rc == 0, rb.lib.r3d_cuda_last_error(ctx.h)
        for i in range(10):
            frame(i)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for i in range(frames):
            frame(i)
        e1.record(st)
        torch.cuda.synchronize()
        out[name] = {"ms_per_frame": e0.elapsed_time(e1) / frames}
    ctx.set_schedule()
    return out


def split_views_bench(rb, torch, ctx, lut, frames: int) -> dict:
    """One 1920x1080 frame split into 4, 16 and 64 views of the same orbit
    (one r3d_cuda_raycast_fwd call per frame), one thread per ray (a grid
    launch per view) against the automatic schedule (whole tiles of every
    view in one launch); per-frame CUDA events on the context's stream."""
    st = torch.cuda.ExternalStream(ctx.stream)
    img = torch.zeros((H, W, 4), dtype=torch.uint8, device="cuda")
    out = {}
    for cols, rows in ((2, 2), (4, 4), (8, 8)):
        w, h = W // cols, H // rows
        seq = []
        for i in range(frames):
            vs = []
            for k in range(cols * rows):
                p = rb.orbit_view(((i + 7 * k) % ORBIT_FRAMES) / ORBIT_FRAMES, w, h, lut,
                                  step_voxels=STEP_VOXELS, frame_index=i)
                p.brick_mode = ctx.brick_mode
                p.view_org = (w * (k % cols)) | ((h * (k // cols)) << 16)
                vs.append(p)
            seq.append(vs)
        r = {}
        for name, sched in (("grid", dict(persistent=0)), ("auto", dict())):
            ctx.set_schedule(**sched)
            for i in range(5):
                ctx.raycast(seq[i], W, H, out=img, stream=ctx.stream)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            for vs in seq:
                ctx.raycast(vs, W, H, out=img, stream=ctx.stream)
            e1.record(st)
            torch.cuda.synchronize()
            r[f"{name}_ms_per_frame"] = e0.elapsed_time(e1) / frames
        r["speedup"] = r["grid_ms_per_frame"] / r["auto_ms_per_frame"]
        out[f"{cols * rows}x{w}x{h}"] = r
    ctx.set_schedule()
    return out


def cpu_baseline(rb, orc, ctx, vol_pages, lut, frames: list[int], threads: int) -> dict:
    """The oracle (FP32 CPU restatement of the reference shader) on a bounded
    sample of the same workload: whole 1920x1080 frames of the orbit, timed.
    Each oracle frame is also compared with the GPU's frame of the same view
    (pixels, per-ray step counts), and a few more frames are compared in MIP
    (with MIP indices) and HEATMAP mode, untimed: the parity record of the
    benchmark configuration."""
    page, pool, brick_mode = vol_pages
    sc = orc.BrickScene(page, pool)
    total, dt = 0, 0.0
    par = {"frames": {}, "max_lsb": 0, "steps_equal": True, "mip_equal": True}
    gsteps = np.zeros((H, W), np.uint32)
    gmip = np.zeros((H, W), np.uint32)

    def compare(p, ref, rsteps, rmip):
        img = ctx.raycast(p, W, H, steps=gsteps, mip_index=gmip)
        par["max_lsb"] = max(par["max_lsb"], int(np.abs(img.astype(np.int16) -
                                                        ref.astype(np.int16)).max()))
        par["steps_equal"] &= bool(np.array_equal(gsteps, rsteps))
        if p.mode == 1:
            par["mip_equal"] &= bool(np.array_equal(gmip, rmip))

    for i in frames:
        p = orbit_params(rb, lut, i, brick_mode)
        t0 = time.perf_counter()
        ref, rsteps, rmip, tot, _ = orc.render(p, sc, lut, W, H, cutoff=CUTOFF, threads=threads)
        dt += time.perf_counter() - t0
        total += tot
        compare(p, ref, rsteps, rmip)
    par["frames"]["full"] = len(frames)
    for name, mode in (("mip", 1), ("heatmap", 3)):
        picked = frames[::max(1, len(frames) // 4)][:4]
        for i in picked:
            p = orbit_params(rb, lut, i, brick_mode, mode)
            ref, rsteps, rmip, _, _ = orc.render(p, sc, lut, W, H, cutoff=CUTOFF,
                                                 threads=threads)
            compare(p, ref, rsteps, rmip)
        par["frames"][name] = len(picked)
    return {"value": total / dt / 1e9, "unit": "Gsamples/s", "cores": threads, "kind": "port",
            "sample": f"{len(frames)} full 1920x1080 orbit frames (phases "
                      f"{frames[0]}..{frames[-1]} step {frames[1] - frames[0] if len(frames) > 1 else 0}"
                      f" of 120), {total} samples, {dt:.1f} s", "fps": len(frames) / dt,
            "parity": par}


def run_reference(args) -> None:
    """CPU arm: the oracle (the CPU restatement of the reference shader) on all
    host threads, over the same workload built by the oracle itself (phantom,
    brick cache, TF and orbit views bit-equal to the library's), so nothing
    of the library under test is loaded.  Each step renders one whole
    1920x1080 orbit frame when the run has at most 400 frames (about 0.3 s of
    CPU each on 16 threads); longer runs trace an evenly strided 1/16 of each
    frame's rays (every 4th pixel of every 4th row) to stay within minutes."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle as orc
    threads = os.cpu_count() or 1
    vol = orc.phantom(N_EDGE, seed=SEED, threads=threads)
    sc = orc.BrickScene.build(vol, NLEV)  # the oracle's own brick builder
    del vol
    lut = orc.scroll_ramp_tf()
    brick_mode = 9 | (NLEV << 8) | orc.BRICK_LOD_FLAG
    whole = args.warmup + args.steps <= 400
    if not whole:
        ys, xs = np.mgrid[0:H:4, 0:W:4]
        xy = np.stack([xs.ravel(), ys.ravel()], axis=1).astype(np.uint32)
    times, samples = [], []
    for s in range(args.warmup + args.steps):
        p = orc.orbit_view((s % ORBIT_FRAMES) / ORBIT_FRAMES, W, H, lut, step_voxels=STEP_VOXELS,
                           frame_index=s)
        p.brick_mode = brick_mode
        t0 = time.perf_counter()
        if whole:
            tot = orc.render(p, sc, lut, W, H, cutoff=CUTOFF, threads=threads,
                             want_aux=False)[3]
        else:
            tot = float(orc.render_pixels(p, sc, lut, xy, cutoff=CUTOFF, threads=threads)[1].sum())
        dt = time.perf_counter() - t0
        if s >= args.warmup:
            times.append(dt)
            samples.append(float(tot))
    t = sum(times)
    v = sum(samples) / t / 1e9
    sample = ("per step: one whole 1920x1080 orbit frame" if whole else
              f"per step: {xy.shape[0]} rays (every 4th pixel of every 4th row) of one "
              "1920x1080 orbit frame")
    out = {"impl": "reference", "metric": METRIC,
           "value": v, "unit": "Gsamples/s", "n_gpus": args.gpus, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": 1000.0 * t / len(times),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": "synthetic",
           "config": {"workload": WORKLOAD, "cutoff": CUTOFF, "step_voxels": STEP_VOXELS,
                      "sample": sample},
           "cpu_baseline": {"value": v, "unit": "Gsamples/s", "cores": threads, "kind": "port",
                            "sample": sample},
           "e2e": {"value": v, "unit": "Gsamples/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def run_ours(args) -> None:
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(local)
    import render3d_b200 as rb

    lut = rb.scroll_ramp_tf()
    vol = rb.phantom(N_EDGE, seed=SEED)
    ctx = rb.Context(local)
    ctx.set_transfer(lut)
    ctx.set_quality(rb.QUALITY_FULL)
    ctx.set_alpha_cutoff(CUTOFF)
    ctx.bricks_build(vol, NLEV)
    bm = ctx.brick_mode
    info = ctx.bricks_info()
    stream = torch.cuda.ExternalStream(ctx.stream, device=local)
    img = torch.zeros((H, W, 4), dtype=torch.uint8, device=f"cuda:{local}")
    total = torch.zeros(1, dtype=torch.int64, device=f"cuda:{local}")
    K, Wm = args.steps, args.warmup

    def frame(i, counters=None):
        ctx.raycast(orbit_params(rb, lut, i, bm), W, H, out=img, total=total,
                    counters=counters, stream=ctx.stream)

    # untimed counting pass over the same frames: algorithmic work per frame,
    # and the slots each frame reads (compulsory bytes)
    cnt = torch.zeros(4, dtype=torch.int64, device=f"cuda:{local}")
    bits = torch.zeros((info["nslots"] + 31) // 32, dtype=torch.int32, device=f"cuda:{local}")
    ctx.set_slot_trace(bits)
    touched = []
    for i in range(Wm, Wm + K):
        bits.zero_()
        torch.cuda.synchronize()  # the frame runs on the context's stream
        frame(i, counters=cnt)
        torch.cuda.synchronize()
        touched.append(int(np.unpackbits(bits.cpu().numpy().view(np.uint8)).sum()))
    ctx.set_slot_trace(None)
    torch.cuda.synchronize()
    counts = cnt.cpu().numpy().astype(np.float64)
    slots_read = float(np.mean(touched))
    l2_gbs = ctx.l2_read_probe(48 << 20, 40)

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # clocks are sampled across the warm-up and the timed frames
    with ClockSampler(local) as clk:
        for i in range(Wm):
            frame(i)
        torch.cuda.synchronize()  # the frames run on the context's own stream
        total.zero_()
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        e0.record(stream)
        for i in range(Wm, Wm + K):
            frame(i)
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    samples = float(total.item())
    if abs(samples - counts[0]) > 0.5:
        print(f"warning: counting pass {counts[0]:.0f} samples, timed pass {samples:.0f}",
              file=sys.stderr)
    samples_all, ms_max = reduce_replicas(dist, samples, ms, torch.device(f"cuda:{local}"))
    value = samples_all / (ms_max * 1e-3) / 1e9
    fps = K * world / (ms_max * 1e-3)

    # end to end through the render3d-facing API: r3d_frame + r3d_read_frame
    modes = mode_stats(rb, ctx, lut, torch, stream, total, img, ORBIT_FRAMES * 2)

    r = rb.Renderer(W, H)
    r.set_transfer(lut)
    r.set_alpha_cutoff(CUTOFF)
    r.bricks_begin_volume(vol, NLEV)
    host = torch.empty((H, W, 4), dtype=torch.uint8, pin_memory=True).numpy()
    # the frames' parameter blocks are the inputs: built before the timed
    # loop, handed to r3d_frame (248 B each, host to device) inside it
    params = []
    for i in range(Wm + K):
        p = orbit_params(rb, lut, i, 0)
        r.bricks_params(p)
        params.append(p)
    for i in range(Wm):
        r.frame(params[i])
        r.read_frame(host)
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for i in range(Wm, Wm + K):
        r.frame(params[i])
        r.read_frame(host)
    e2e_s = time.perf_counter() - t0
    te = torch.tensor([e2e_s], device=f"cuda:{local}")
    if dist:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_value = samples_all / float(te.item()) / 1e9
    r.close()

    shard = shard_bench(rb, torch, local, vol, lut, ORBIT_FRAMES * 2)
    overlays = overlay_bench(rb, ctx, lut, torch, stream, total, img, ORBIT_FRAMES * 2)

    noalloc = noalloc_bench(rb, torch, ctx, lut, img, ORBIT_FRAMES)
    split = split_views_bench(rb, torch, ctx, lut, ORBIT_FRAMES)

    bt = None
    if not args.no_batch:
        bt = batch_bench(rb, torch, local, ctx, reps=5)

    fb = None
    if not args.no_fwd_bwd:
        fb = fwd_bwd_bench(rb, ctx, torch, local, steps=20, adam_steps=100)
        fb["ratio_vs_plain"] = fb["value"] / value
        fb["ratio_vs_plain_same_views"] = fb["value"] / fb["plain_same_views"]["gsamples_per_s"]

    peak, peak_kind = measured_peaks()
    alg = algorithmic_bytes(counts, W * H * K)
    sms = torch.cuda.get_device_properties(local).multi_processor_count
    clk_sum = clk.summary()
    sm_hz = (clk_sum["sm_mhz"] or 1965.0) * 1e6
    achieved = alg / (ms * 1e-3) / 1e9
    out = None
    if rank == 0:
        cpu = parity = None
        if world == 1 and not args.no_cpu_baseline:
            import oracle as orc
            page, pool = ctx.bricks_read()
            ctx.set_alpha_cutoff(CUTOFF)  # the adjoint workload left it at 0.98
            cpu = cpu_baseline(rb, orc, ctx, (page, pool, bm), lut,
                               list(range(0, ORBIT_FRAMES, 4)), os.cpu_count() or 1)
            del pool
            parity = cpu.pop("parity")
        out = {"metric": METRIC, "value": value,
               "unit": "Gsamples/s", "n_gpus": world, "steps": K, "warmup": Wm,
               "ms_per_step": ms_max / K, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f32", "data": "synthetic",
               "config": {"workload": WORKLOAD, "frames_per_step": 1, "cutoff": CUTOFF,
                          "step_voxels": STEP_VOXELS, "lod_bias": 0.0,
                          "slots": info["nslots"], "l2": "inputs larger than L2 "
                          f"(brick pool {info['nslots'] * 2} MiB)",
                          "parallelism": f"replicas x{world}"},
               "fps": fps, "mrays_per_s": W * H * K * world / (ms_max * 1e-3) / 1e6,
               "samples_per_frame": counts[0] / K,
               "work_per_frame": {"samples": counts[0] / K, "tf_lookups": counts[1] / K,
                                  "shaded": counts[2] / K, "page_walks": counts[3] / K},
               "e2e": {"value": e2e_value, "unit": "Gsamples/s", "h2d_bytes_per_step": 248,
                       "d2h_bytes_per_step": W * H * 4, "fps": K * world / float(te.item())},
               "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak,
                            "unit": "GB/s", "frac": achieved / peak,
                            "traffic": FWD_DRAM_TRAFFIC_BYTES,
                            "peak_kind": peak_kind,
                            "algorithmic_bytes_per_frame": alg / K,
                            # the same algorithmic bytes against the L2 read
                            # bandwidth measured by this run's L2-resident probe
                            "l2_peak_gbs": l2_gbs, "l2_frac": achieved / l2_gbs,
                            # unique slots a frame reads (counting pass), as
                            # 2 MiB u8 bricks and as this layout's bytes (8 MiB
                            # quad words + 4 KiB block maxima per slot)
                            "slots_read_per_frame": slots_read,
                            "compulsory_hbm_bytes": slots_read * (2 << 20),
                            "compulsory_frac": slots_read * (2 << 20) / (ms_max / K * 1e-3)
                            / 1e9 / peak,
                            "compulsory_layout_bytes": slots_read * ((8 << 20) + 4096),
                            # the captured launches' warp instructions per
                            # sample, times this run's samples per frame,
                            # over the issue slots of its frame time (148
                            # SMs x 4 schedulers x the median SM clock); and
                            # the captured thread instructions per sample
                            "issue_frac": FWD_WARP_INST / FWD_CAPTURED_SAMPLES * (counts[0] / K)
                            / (sms * 4 * sm_hz * ms_max / K * 1e-3),
                            "thread_inst_per_sample": FWD_THREAD_INST / FWD_CAPTURED_SAMPLES,
                            "simt_lanes_per_inst": FWD_THREAD_INST / FWD_WARP_INST},
               "modes": modes,
               "shard": shard,
               "overlays": overlays,
               "fwd_bwd": fb,
               "batch": bt,
               "noalloc": noalloc,
               "split_views": split,
               "gpu_launches": K,
               "clocks": clk_sum,
               "cpu_baseline": cpu,
               "parity": parity}
        print(json.dumps(out), flush=True)
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return out


def run_profile_sections(args) -> None:
    """Renders args.profile_sections frames (1920x1080, FULL) of each section
    mode over a 4096 x 4096 x 40 phantom -- tiled slab, clipmap, virtual
    slab -- and of a flattened segment over 512^3 bricks (a 1024 x 1024 x 64
    window, its bakes included); the command line that ncu captures."""
    import torch
    import render3d_b200 as rb
    lut = rb.scroll_ramp_tf()
    n = args.profile_sections
    img = torch.zeros((H, W, 4), dtype=torch.uint8, device="cuda")
    nx, ny, nz, d = 4096, 4096, 40, 16
    ctx = rb.Context(0)
    ctx.set_transfer(lut)
    ctx.set_alpha_cutoff(CUTOFF)
    vol = ctx.phantom((nx, ny, nz), seed=SEED)
    ext = (1.0, 1.0, d / nx)

    def view(i, setup):
        p = rb.camera_view(0.05 * math.sin(i * 0.05), 0.02, 0.25, W, H, lut,
                           target=(0.5, 0.5 * ext[1], 0.5 * ext[2]), step_voxels=STEP_VOXELS,
                           frame_index=i)
        setup(p)
        p.density = 6.0
        ctx.raycast(p, W, H, out=img, stream=ctx.stream)

    ctx.slab_build(vol, d + 2, 4)

    def slab_setup(p):
        ctx.slab_params(p)
        p.slab_depth = d
    ctx.clip_build(vol, d)
    ctx.clip_frame(nx / 2, ny / 2, 4)
    ctx.vslab_begin(vol, nx, ny, d)
    for _ in range(2):
        ctx.vslab_frame(nx / 2, ny / 2, 4, 64)
    for setup in (slab_setup, ctx.clip_params, ctx.vslab_params):
        for i in range(n):
            view(i, setup)
    torch.cuda.synchronize()
    ctx.close()
    del vol
    torch.cuda.empty_cache()
    s = surf_bench(rb, torch, lut, n, n=512, window=(1024, 1024, 64))
    print("profile section frames done:", n, "surf pitch 0.5 bake ms", s["pitch_0.5"]["bake_ms"])


def run_profile_filter(args) -> None:
    """The post-decode display filter: a streamed 512^3 cache with every
    brick resident (73 slots, 3 levels), re-filtered args.profile_filter
    times in each mode (the 72 non-coarsest slots copied in again from the
    host store, then filtered).  Prints CUDA-event times on the context's
    stream per refilter and the filter's share per slot (beyond the
    unfiltered re-upload); the command line that ncu captures."""
    import torch
    import render3d_b200 as rb
    lut = rb.scroll_ramp_tf()
    vol = rb.phantom(512, seed=SEED)
    ctx = rb.Context(0)
    ctx.stream_begin(vol, 3, 73)
    p = rb.camera_view(0.5, -0.4, 0.9, W, H, lut, step_voxels=STEP_VOXELS)
    for _ in range(30):
        st = ctx.stream_update(p, 64)
    assert st["resident"] == 73
    ev = torch.cuda.ExternalStream(ctx.stream)
    out = {}
    for mode in (0, 1, 2, 3, 4, 0x100, 0x101):
        ctx.bricks_postfilter(mode, 1.0)
        ctx.bricks_refilter()  # warm
        times = []
        for _ in range(args.profile_filter):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(ev)
            ctx.bricks_refilter()
            b.record(ev)
            b.synchronize()
            times.append(a.elapsed_time(b))
        out[mode] = min(times)
    base = out[0]
    res = {f"{m:#x}": {"ms_per_refilter": round(t, 4),
                       "filter_us_per_slot": round((t - base) * 1e3 / 72, 2)} for m, t in out.items()}
    print(json.dumps({"profile_filter": res, "slots": 72, "reps": args.profile_filter}))
    ctx.close()


def run_profile(args) -> None:
    """Renders args.profile frames of the workload with no timing: the
    command line that ncu captures."""
    import torch
    import render3d_b200 as rb
    lut = rb.scroll_ramp_tf()
    vol = rb.phantom(args.profile_size, seed=SEED)
    ctx = rb.Context(0)
    ctx.set_transfer(lut)
    ctx.set_alpha_cutoff(CUTOFF)
    ctx.bricks_build(vol, NLEV)
    img = torch.zeros((H, W, 4), dtype=torch.uint8, device="cuda")
    ctx.set_schedule(persistent=args.profile_persistent, staging=args.profile_staging)
    for i in range(args.profile):
        ctx.raycast(orbit_params(rb, lut, i, ctx.brick_mode, args.profile_mode), W, H, out=img,
                    stream=ctx.stream)
    torch.cuda.synchronize()
    # the work counters of the same frames, from launches after the profiled
    # ones (samples, TF lookups, shaded samples, page walks per frame)
    counts = []
    for i in range(args.profile):
        cnt = torch.zeros(4, dtype=torch.int64, device="cuda")
        ctx.raycast(orbit_params(rb, lut, i, ctx.brick_mode, args.profile_mode), W, H, out=img,
                    counters=cnt, stream=ctx.stream)
        torch.cuda.synchronize()
        counts.append([int(x) for x in cnt.cpu()])
    print(json.dumps({"profile_frames": args.profile, "mode": args.profile_mode,
                      "counters_per_frame": counts}))
    ctx.close()


def run_sparse(args) -> None:
    """The large-volume workload: a 2048^3 phantom (8 GiB, generated on the
    device) with only the bricks whose maximum exceeds 40 resident, rendered
    at 3840x2160 with LOD bias 0 and 1; and the adjoint at 512^3 FP32, 16
    views of 512x512, step 0.25, checkpoints every 32 / 64 / 128 samples,
    deterministic and atomic accumulation."""
    import torch
    import render3d_b200 as rb
    lut = rb.scroll_ramp_tf()
    ctx = rb.Context(0)
    ctx.set_transfer(lut)
    ctx.set_alpha_cutoff(CUTOFF)
    t0 = time.perf_counter()
    vol = ctx.phantom(2048, seed=SEED)
    ctx.bricks_build(vol, NLEV, min_max=41)
    del vol
    torch.cuda.empty_cache()
    build_s = time.perf_counter() - t0
    info = ctx.bricks_info()
    total_bricks = sum(((2048 >> l) // 128) ** 3 for l in range(NLEV))
    img = torch.zeros((2160, 3840, 4), dtype=torch.uint8, device="cuda")
    tot = torch.zeros(1, dtype=torch.int64, device="cuda")
    st = torch.cuda.ExternalStream(ctx.stream)
    out = {"workload": "sparse 2048^3 (bricks with max > 40 resident), 3840x2160, full shading",
           "resident_bricks": info["nslots"], "total_bricks": total_bricks,
           "resident_fraction": info["nslots"] / total_bricks, "build_s": build_s}
    K = max(args.steps // 10, 20)
    for bias in (0.0, 1.0):
        def frame(i):
            p = rb.orbit_view((i % ORBIT_FRAMES) / ORBIT_FRAMES, 3840, 2160, lut,
                              step_voxels=STEP_VOXELS, lod_bias=bias, frame_index=i)
            p.brick_mode = ctx.brick_mode
            ctx.raycast(p, 3840, 2160, out=img, total=tot, stream=ctx.stream)
        for i in range(10):
            frame(i)
        torch.cuda.synchronize()
        tot.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for i in range(K):
            frame(i)
        e1.record(st)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / K
        out[f"lod_bias_{int(bias)}"] = {"ms_per_frame": ms, "fps": 1000.0 / ms,
                                        "gsamples_per_s": tot.item() / K / (ms * 1e-3) / 1e9}
    ctx.close()
    # adjoint at 512^3
    ctx = rb.Context(0)
    ctx.set_alpha_cutoff(0.98)
    n, nv, w = 512, 16, 512
    dens = ctx.phantom(n, seed=SEED).float().div_(255.0)
    g = torch.Generator(device="cuda").manual_seed(SEED)
    dens.add_(torch.randn(dens.shape, device="cuda", generator=g) * (10.0 / 255.0))
    flut = torch.tensor(lut.astype(np.float32) / 255.0, device="cuda")
    views = [rb.orbit_view(i / nv, w, w, lut, step_voxels=0.25, frame_index=i) for i in range(nv)]
    for v in views:
        v.max_mip = 0.0
    nf = nv * w * w * 3
    rgb = torch.empty(nf, device="cuda")
    tot.zero_()
    st = torch.cuda.ExternalStream(ctx.stream)
    ctx.diff_forward(dens, flut, views, rgb, total=tot, stream=ctx.stream)
    torch.cuda.synchronize()
    samples = tot.item()
    grad = torch.randn(nf, device="cuda", generator=g)
    gd = torch.empty_like(dens)
    gl = torch.empty_like(flut)
    gs = torch.empty(1, device="cuda")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(3):
        ctx.diff_forward(dens, flut, views, rgb, stream=ctx.stream)
    e1.record(st)
    torch.cuda.synchronize()
    bwd = {"samples_per_pass": samples, "max_steps_per_ray": None,
           "fwd_ms": e0.elapsed_time(e1) / 3}
    for k in (32, 64, 128):
        for det in (False, True):
            ctx.raycast_bwd(dens, flut, views, grad, gd, gl, gs, k, det, stream=ctx.stream)
            e0.record(st)
            for _ in range(3):
                ctx.raycast_bwd(dens, flut, views, grad, gd, gl, gs, k, det, stream=ctx.stream)
            e1.record(st)
            torch.cuda.synchronize()
            bwd[f"bwd_k{k}_{'det' if det else 'atomic'}_ms"] = e0.elapsed_time(e1) / 3
            ctx.diff_forward(dens, flut, views, rgb, stream=ctx.stream, tape=True)
            e0.record(st)
            for _ in range(3):
                ctx.raycast_bwd(dens, flut, views, grad, gd, gl, gs, k, det, stream=ctx.stream,
                                tape=True)
            e1.record(st)
            torch.cuda.synchronize()
            bwd[f"bwd_k{k}_{'det' if det else 'atomic'}_tape_ms"] = e0.elapsed_time(e1) / 3
    out["adjoint_512"] = bwd
    ctx.close()
    torch.cuda.empty_cache()
    out["stream"] = stream_bench(rb, torch, lut)
    out["stream_small_pool"] = stream_bench(rb, torch, lut, nslots=80)
    # the cache at 35 % residency: 1638 of the pyramid's 4680 bricks resident,
    # which ones chosen by the pump's view-cone request set (the reference's
    # residency rule for a pool smaller than the volume), at 3840x2160
    out["stream_35pct_4k"] = stream_bench(rb, torch, lut, nslots=1638, budget=64, frames=120,
                                          w=3840, h=2160)
    out["fixed_35pct_4k"] = stream_bench(rb, torch, lut, nslots=1638, budget=1638, frames=120,
                                         w=3840, h=2160, pump_timed=False)
    print(json.dumps(out), flush=True)


def stream_bench(rb, torch, lut, nslots: int = 1024, budget: int = 16,
                 frames: int = 240, w: int = W, h: int = H, pump_timed: bool = True) -> dict:
    """The 2048^3 phantom as a streaming cache: the whole 4-level pyramid in
    pinned host memory and nslots device slots (1024: 2 GiB); every frame of
    a w x h orbit runs one pump update (at most `budget` bricks copied in) and
    renders; wall-clock fps with one synchronize at the end.  pump_timed
    False: the pump runs over the warm-up frames only, and the timed frames
    render the cache as it was left (a fixed partial residency, the absent
    bricks drawn from coarser levels)."""
    ctx = rb.Context(0)
    try:
        ctx.set_transfer(lut)
        ctx.set_alpha_cutoff(CUTOFF)
        vol = ctx.phantom(2048, seed=SEED)
        t0 = time.perf_counter()
        ctx.stream_begin(vol, NLEV, nslots)
        begin_s = time.perf_counter() - t0
        del vol
        torch.cuda.empty_cache()
        img = torch.zeros((h, w, 4), dtype=torch.uint8, device="cuda")

        def frame(i, stats, pump=True):
            p = rb.orbit_view((i % ORBIT_FRAMES) / ORBIT_FRAMES, w, h, lut,
                              step_voxels=STEP_VOXELS, frame_index=i)
            p.brick_mode = ctx.brick_mode
            if pump:
                st = ctx.stream_update(p, budget)
                for k in stats:
                    stats[k] += st[k]
            ctx.raycast(p, w, h, out=img, stream=ctx.stream)
        warm = {k: 0 for k in ("desired", "requested", "uploaded", "evicted")}
        for i in range(20):
            frame(i, warm)
        torch.cuda.synchronize()
        stats = {k: 0 for k in ("desired", "requested", "uploaded", "evicted")}
        t0 = time.perf_counter()
        for i in range(20, 20 + frames):
            frame(i, stats, pump_timed)
        torch.cuda.synchronize()
        s = time.perf_counter() - t0
        return {"workload": f"2048^3 streamed: 4680 bricks in pinned host memory, {nslots} device "
                            f"slots, {w}x{h} orbit, pump budget {budget} bricks per frame"
                            + ("" if pump_timed else " over the warm-up only (fixed residency)"),
                "resident_fraction": nslots / 4680,
                "begin_s": begin_s, "fps": frames / s, "ms_per_frame": 1e3 * s / frames,
                "bricks_copied_per_frame": stats["uploaded"] / frames,
                "evicted_per_frame": stats["evicted"] / frames,
                "h2d_gb_per_s": stats["uploaded"] * 2 * 1024 ** 2 / s / 1e9,
                "requested_per_frame": stats["requested"] / frames}
    finally:
        ctx.close()


def sections_bench(rb, torch, lut, frames: int) -> dict:
    """Whole cross-sections of an 8192 x 8192 x 64 phantom (4 GiB, generated
    on the device) in the three modes built for them: the tiled slab (ring
    of 32 slices), the XY clipmap (window depth 32) and the virtual slab
    (vslab_bench).  A 1920x1080 camera
    faces the section and pans across it; each mode is timed rendering a
    fixed window, and with a per-frame update (slab: the window scrolls one
    slice; clip: the focus follows the pan and the window scrolls one slice,
    so levels recentre and ring layers refill).  Device time of the frames
    with CUDA events on the context stream."""
    nx, ny, nz, wz = 8192, 8192, 64, 32
    out = {"workload": f"cross-sections of {nx}x{ny}x{nz}, 1920x1080 face-on pan, full shading"}
    ctx = rb.Context(0)
    try:
        ctx.set_transfer(lut)
        ctx.set_alpha_cutoff(CUTOFF)
        vol = ctx.phantom((nx, ny, nz), seed=SEED)
        out["vslab"] = vslab_bench(rb, torch, lut, vol, frames)
        t0 = time.perf_counter()
        ctx.slab_build(vol, wz, 0)
        torch.cuda.synchronize()
        slab_s = time.perf_counter() - t0
        t0 = time.perf_counter()
        ctx.clip_build(vol, wz)
        ctx.clip_frame(0.3 * nx, 0.5 * ny, 0)
        torch.cuda.synchronize()
        clip_s = time.perf_counter() - t0
        del vol
        torch.cuda.empty_cache()
        img = torch.zeros((H, W, 4), dtype=torch.uint8, device="cuda")
        tot = torch.zeros(1, dtype=torch.int64, device="cuda")
        st = torch.cuda.ExternalStream(ctx.stream)
        ext = (1.0, ny / nx, (wz - 2) / nx)

        def view(i):
            u = 0.3 + 0.4 * (i % 240) / 240.0
            p = rb.camera_view(0.05 * math.sin(i * 0.05), 0.02, 0.12, W, H, lut,
                               target=(u, 0.5 * ext[1], 0.5 * ext[2]), step_voxels=STEP_VOXELS,
                               frame_index=i)
            return p, u

        def run(kind, update):
            def frame(i):
                p, u = view(i)
                if kind == "slab":
                    if update:
                        ctx.slab_window((i // 4) % (nz - wz))
                    ctx.slab_params(p)
                    p.slab_depth = wz - 2
                else:
                    if update:
                        ctx.clip_frame(u * nx, 0.5 * ny, (i // 4) % (nz - wz))
                    ctx.clip_params(p)
                p.density = 6.0
                ctx.raycast(p, W, H, out=img, total=tot, stream=ctx.stream)
            for i in range(10):
                frame(i)
            torch.cuda.synchronize()
            tot.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0 = time.perf_counter()
            e0.record(st)
            for i in range(10, 10 + frames):
                frame(i)
            e1.record(st)
            torch.cuda.synchronize()
            wall = time.perf_counter() - t0
            ms = e0.elapsed_time(e1) / frames
            return {"ms_per_frame": ms, "fps": 1000.0 / ms, "wall_fps": frames / wall,
                    "gsamples_per_s": tot.item() / frames / (ms * 1e-3) / 1e9}
        out["slab"] = {"build_s": slab_s, "fixed_window": run("slab", False),
                       "window_scroll_every_4_frames": run("slab", True)}
        out["clip"] = {"build_s": clip_s, "fixed_window": run("clip", False),
                       "focus_pan_and_scroll": run("clip", True)}
    finally:
        ctx.close()
    return out


def vslab_bench(rb, torch, lut, vol, frames: int) -> dict:
    """The virtual slab over the same volume: the whole 8192^2 x 30 section
    (fixed, then scrolling one slice every 4 frames with 64 cell fills a
    frame), and a 4096^2 x 30 window with a 16-slice z margin panning across
    the volume (16 fills a frame).  Device time of fills and frames with
    CUDA events on the context stream; fills are counted per frame."""
    nz, ny, nx = vol.shape
    out = {}
    for name, (Wn, Hn, zm, budget, pan) in {
            "whole_section": (nx, ny, 0, 64, False),
            "window_4096_pan": (4096, 4096, 16, 16, True)}.items():
        ctx = rb.Context(0)
        try:
            ctx.set_transfer(lut)
            ctx.set_alpha_cutoff(CUTOFF)
            D = 30
            ctx.vslab_begin(vol, Wn, Hn, D, zm)
            img = torch.zeros((H, W, 4), dtype=torch.uint8, device="cuda")
            tot = torch.zeros(1, dtype=torch.int64, device="cuda")
            st = torch.cuda.ExternalStream(ctx.stream)
            ext = (1.0, Hn / Wn, D / Wn)

            def frame(i, update):
                fx = (0.3 + 0.4 * (i % 240) / 240.0) * nx if pan else nx / 2
                z0 = (i // 4) % (nz - D - 2) if update else 8
                s = ctx.vslab_frame(fx, ny / 2, z0, budget)
                p = rb.camera_view(0.05 * math.sin(i * 0.05), 0.02, 0.12 * Wn / nx, W, H, lut,
                                   target=(0.5, 0.5 * ext[1], 0.5 * ext[2]),
                                   step_voxels=STEP_VOXELS, frame_index=i)
                ctx.vslab_params(p)
                p.density = 6.0
                ctx.raycast(p, W, H, out=img, total=tot, stream=ctx.stream)
                return s["jobs"]
            for i in range(12):  # fill the window
                frame(i, False)
            res = {}
            for mode, update in (("fixed", False), ("moving", True)):
                torch.cuda.synchronize()
                tot.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                jobs = 0
                e0.record(st)
                for i in range(12, 12 + frames):
                    jobs += frame(i, update)
                e1.record(st)
                torch.cuda.synchronize()
                ms = e0.elapsed_time(e1) / frames
                res[mode] = {"ms_per_frame": ms, "fps": 1000.0 / ms,
                             "fills_per_frame": jobs / frames,
                             "gsamples_per_s": tot.item() / frames / (ms * 1e-3) / 1e9}
            lay = ctx.vslab_layout()
            res["tiles"] = lay.ntiles
            res["tile_gb"] = lay.ntiles * (lay.px + 2) ** 2 * lay.wz / 1e9
            out[name] = res
        finally:
            ctx.close()
    return out


def surf_bench(rb, torch, lut, frames: int, n: int = N_EDGE, window=(2048, 2048, 96)) -> dict:
    """Flattened-segment views over the n^3 (default 1024^3) LOD brick
    cache: a wavy sheet (513 x 513 grid of 2-voxel cells around the centre)
    baked into a 2048 x 2048 x 96 flattened volume at pitch 0.5 and 2
    voxels, then 1920x1080 surf views in FULL at two zooms.  Bake and frame
    times with CUDA events."""
    ctx = rb.Context(0)
    try:
        ctx.set_transfer(lut)
        ctx.set_alpha_cutoff(CUTOFF)
        vol = ctx.phantom(n, seed=SEED)
        ctx.bricks_build(vol, NLEV)
        del vol
        g = 513
        j, i = np.mgrid[0:g, 0:g].astype(np.float64)
        x, y = 0.5 * n - 512.0 + 2.0 * i, 0.5 * n - 512.0 + 2.0 * j
        z = 0.5 * n + 60.0 * n / 1024.0 * np.sin(x / 90.0) + 40.0 * n / 1024.0 * np.cos(y / 130.0)
        nrm = np.stack([-60.0 / 90.0 * np.cos(x / 90.0), 40.0 / 130.0 * np.sin(y / 130.0),
                        np.ones_like(x)], -1)
        nrm /= np.linalg.norm(nrm, axis=-1, keepdims=True)
        coords = np.zeros((g, g, 4), np.float32)
        coords[..., 0], coords[..., 1], coords[..., 2], coords[..., 3] = x, y, z, 1.0
        normals = np.zeros((g, g, 4), np.float32)
        normals[..., :3] = nrm
        ctx.surf_begin(coords, normals)
        Wv, Hv, Lv = window
        ctx.surfvol_begin(Wv, Hv, Lv, Lv // 2, 0.5, 0.5)
        st = torch.cuda.ExternalStream(ctx.stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        out = {"workload": f"{n}^3 LOD bricks, 513^2 segment grid, {Wv}x{Hv}x{Lv} flattened "
                           "volume, 1920x1080 surf views"}
        img = torch.zeros((H, W, 4), dtype=torch.uint8, device="cuda")
        for step in (0.5, 2.0):
            ctx.surfvol_window(0.0, 0.0, step, 0.0)  # warm
            torch.cuda.synchronize()
            e0.record(st)
            for k in range(5):
                ctx.surfvol_window(float(k), 0.0, step, 0.0)
            e1.record(st)
            torch.cuda.synchronize()
            bake_ms = e0.elapsed_time(e1) / 5
            span = Wv * step
            res = {"bake_ms": bake_ms,
                   "bake_gtexels_per_s": Wv * Hv * Lv / (bake_ms * 1e-3) / 1e9}
            for zoom, half_w in (("whole_window", 0.5 * span), ("quarter", 0.125 * span)):
                def frame(i):
                    p = rb.FrameParams()
                    p.viewport[0], p.viewport[1] = W, H
                    p.mode = 0
                    p.cam_origin[:] = (0.5 * span + 4.0 * math.sin(i * 0.1), 0.5 * span, 0.0)
                    p.cam_right[:] = (half_w, 0.0, 0.0)
                    p.cam_up[:] = (0.0, half_w * H / W, 0.0)
                    p.step_voxels, p.density, p.threshold = 0.5, 1.5, 0.02
                    p.slab_z0, p.slab_depth, p.frame_index = 0.0, 64, i
                    ctx.surfvol_params(p)
                    ctx.raycast(p, W, H, out=img, stream=ctx.stream)
                for i in range(5):
                    frame(i)
                torch.cuda.synchronize()
                e0.record(st)
                for i in range(frames):
                    frame(i)
                e1.record(st)
                torch.cuda.synchronize()
                ms = e0.elapsed_time(e1) / frames
                res[zoom] = {"ms_per_frame": ms, "fps": 1000.0 / ms}
            out[f"pitch_{step}"] = res
        return out
    finally:
        ctx.close()


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    # render3d's perf protocol: 400 warm-up frames, 1200 measured
    # (tools/perf.sh:18-19)
    ap.add_argument("--steps", type=int, default=1200)
    ap.add_argument("--warmup", type=int, default=400)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fwd-bwd", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--workload", default="orbit1024",
                    choices=["orbit1024", "sparse2048", "sections8192", "surf1024"],
                    help="sparse2048: the large sparse volume and 512^3 adjoint (extra line)")
    ap.add_argument("--profile", type=int, default=0, metavar="N",
                    help="only build the workload and render N orbit frames (for ncu)")
    ap.add_argument("--profile-mode", type=int, default=0)
    ap.add_argument("--profile-persistent", type=int, default=0,
                    help="schedule of the --profile frames: 0 grid, 1 lane refill, 2 whole tiles")
    ap.add_argument("--profile-staging", type=int, default=0,
                    help="1: the --profile frames run the TMA-staged kernel")
    ap.add_argument("--profile-sections", type=int, default=0, metavar="N",
                    help="only render N frames of each section mode and of flattened views")
    ap.add_argument("--profile-diff", type=int, default=0, metavar="N",
                    help="only run N forward+backward steps of the differentiable workload")
    ap.add_argument("--profile-filter", type=int, default=0, metavar="N",
                    help="only re-filter a streamed 512^3 cache N times in each display filter")
    ap.add_argument("--profile-size", type=int, default=N_EDGE)
    args = ap.parse_args()
    if args.profile:
        run_profile(args)
        return
    if args.profile_sections:
        run_profile_sections(args)
        return
    if args.profile_filter:
        run_profile_filter(args)
        return
    if args.profile_diff:
        import torch
        import render3d_b200 as rb
        ctx = rb.Context(0)
        fb = fwd_bwd_bench(rb, ctx, torch, 0, steps=args.profile_diff, adam_steps=1)
        print("profile fwd+bwd steps done:", fb["steps"])
        ctx.close()
        return
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "sparse2048":
        run_sparse(args)
    elif args.workload == "surf1024":
        import torch
        import render3d_b200 as rb
        print(json.dumps(surf_bench(rb, torch, rb.scroll_ramp_tf(), max(args.steps // 5, 60))),
              flush=True)
    elif args.workload == "sections8192":
        import torch
        import render3d_b200 as rb
        print(json.dumps(sections_bench(rb, torch, rb.scroll_ramp_tf(),
                                        max(args.steps // 5, 60))), flush=True)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
