"""torch.autograd.Function wrapper of the path tracer — test harness only.

forward(albedo, sky) renders passes [pass0, pass0 + spp) of a prt.Context with
per-triangle albedo and sky radiance and returns the mean image (H, W, 3);
backward calls prt_render_backward (path replay, nothing stored between the
two passes) with dL/dsum = dL/dimage / spp."""

import torch


class PathTrace(torch.autograd.Function):
    @staticmethod
    def forward(fctx, albedo, sky, ctx, spp, max_depth, pass0=0):
        ctx.set_albedo(albedo.detach().contiguous())
        ctx.set_sky(float(sky.item()))
        ctx.clear()
        ctx.set_pass(pass0)
        ctx.render(spp, max_depth, accumulate=True)
        acc = torch.empty((ctx.height, ctx.width, 4), dtype=torch.float32, device=albedo.device)
        ctx.read_accum(acc)
        torch.cuda.synchronize()
        fctx.prt = (ctx, spp, max_depth, pass0)
        fctx.save_for_backward(albedo, sky)
        return acc[..., :3] / spp

    @staticmethod
    def backward(fctx, grad):
        ctx, spp, max_depth, pass0 = fctx.prt
        albedo, sky = fctx.saved_tensors
        dsum = (grad / spp).contiguous().float()
        d_alb = torch.zeros_like(albedo)
        d_sky = torch.zeros(1, dtype=torch.float32, device=albedo.device)
        ctx.render_backward(pass0, spp, max_depth, dsum, d_alb, d_sky)
        torch.cuda.synchronize()
        return d_alb, d_sky.reshape(sky.shape), None, None, None, None
