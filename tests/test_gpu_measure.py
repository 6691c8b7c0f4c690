"""The measurement helpers the benchmark's roofline terms come from: the
L2-resident read probe (r3d_cuda_l2_read_probe) and the slot trace of
counting launches (r3d_cuda_set_slot_trace)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_l2_read_probe(ctx):
    gbs = ctx.l2_read_probe(48 << 20, 20)
    # an L2-resident sweep runs well above the HBM copy rate (~6.5 TB/s) and
    # below any plausible L2 ceiling
    assert 6000.0 < gbs < 60000.0, gbs


def test_slot_trace_counts_read_slots(rb, ctx, phantom256, scroll_tf):
    import torch
    ctx.set_transfer(scroll_tf)
    ctx.bricks_build(phantom256, nlev=2)
    info = ctx.bricks_info()
    bits = torch.zeros((info["nslots"] + 31) // 32, dtype=torch.int32, device="cuda")
    p = rb.camera_view(0.7, -0.3, 1.5, 256, 192, scroll_tf, step_voxels=0.5)
    p.brick_mode = ctx.brick_mode
    ctx.set_slot_trace(bits)
    try:
        ctx.raycast(p, 256, 192)  # plain launch: the trace is not touched
        torch.cuda.synchronize()
        assert int(bits.abs().sum().item()) == 0
        cnt = np.zeros(4, np.uint64)
        ctx.raycast(p, 256, 192, counters=cnt)
        torch.cuda.synchronize()
        flags = np.unpackbits(bits.cpu().numpy().view(np.uint8), bitorder="little")
        n = int(flags.sum())
        assert 0 < n <= info["nslots"]
        assert not flags[info["nslots"]:].any()  # no bit past the pool
    finally:
        ctx.set_slot_trace(None)
