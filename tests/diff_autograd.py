"""Test-only torch.autograd.Function over the library's differentiable
raycast (r3d_cuda_diff_forward / r3d_cuda_raycast_bwd through ctypes)."""
import torch


class RaycastFn(torch.autograd.Function):
    """rgb = render(density, lut, density_scale) for a list of views.

    density: (nz, ny, nx) f32 CUDA, lut: (256, 4) f32 CUDA, scale: () f32
    (density scale, written into every view's params).  Returns the packed
    f32 RGB of all views (sum of w*h*3)."""

    @staticmethod
    def forward(ctx, density, lut, scale, rctx, views, ckpt_k, deterministic):
        vs = []
        for v in views:
            q = v.copy()
            q.density = float(scale)
            vs.append(q)
        n = sum(v.viewport[0] * v.viewport[1] * 3 for v in vs)
        rgb = torch.empty(n, dtype=torch.float32, device=density.device)
        torch.cuda.synchronize()
        rctx.diff_forward(density, lut, vs, rgb, stream=rctx.stream)
        torch.cuda.synchronize()
        ctx.save_for_backward(density, lut)
        ctx.rctx, ctx.views, ctx.k, ctx.det = rctx, vs, ckpt_k, deterministic
        return rgb

    @staticmethod
    def backward(ctx, grad_rgb):
        density, lut = ctx.saved_tensors
        gd = torch.empty_like(density)
        gl = torch.empty_like(lut)
        gs = torch.empty(1, dtype=torch.float32, device=density.device)
        g = grad_rgb.contiguous()
        torch.cuda.synchronize()
        ctx.rctx.raycast_bwd(density, lut, ctx.views, g, gd, gl, gs, ctx.k, ctx.det,
                             stream=ctx.rctx.stream)
        torch.cuda.synchronize()
        return gd, gl, gs[0], None, None, None, None


def render(rctx, density, lut, scale, views, ckpt_k=32, deterministic=False):
    return RaycastFn.apply(density, lut, scale, rctx, views, ckpt_k, deterministic)
