"""A thin torch.autograd.Function over the tracer's primal render and its path-replay adjoint
(rtpg_tracer_render / rtpg_tracer_render_adjoint).  It exists for tests and examples: the
parameters are the albedo texture of one material and the emitter radiances; the output is
the mean image of `spp` samples drawn from the tracer's seed (the streams are restarted before
the primal and before the adjoint, so both see the same random numbers)."""
from __future__ import annotations

import torch

from .tracer import FLAG_NEE


class RenderFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, texture, light_rgb, tracer, spp, texture_index, flags=FLAG_NEE):
        tracer.set_light_emission(light_rgb.detach().cpu().numpy())
        if tracer.textures.get(texture_index) is not texture:
            tracer.set_texture(texture_index, texture)
        tracer.clear()
        tracer.render(spp, flags)
        img = tracer.image()
        ctx.tracer, ctx.spp, ctx.texture_index, ctx.flags = tracer, spp, texture_index, flags
        ctx.tex_shape, ctx.n_lights = texture.shape, light_rgb.shape[0]
        ctx.light_device = light_rgb.device
        return img

    @staticmethod
    def backward(ctx, grad_img):
        tr = ctx.tracer
        g_tex = torch.zeros(ctx.tex_shape, dtype=torch.float32, device=grad_img.device)
        g_light = torch.zeros((ctx.n_lights, 3), dtype=torch.float32, device=grad_img.device)
        tr.clear()
        tr.render_adjoint(ctx.spp, grad_img.contiguous().float(), ctx.flags, ctx.texture_index, g_tex, g_light)
        return g_tex, g_light.to(ctx.light_device), None, None, None, None


def render(texture, light_rgb, tracer, spp, texture_index=0, flags=FLAG_NEE):
    """Mean image (h, w, 3) of spp samples, differentiable w.r.t. texture and light_rgb."""
    return RenderFunction.apply(texture, light_rgb, tracer, spp, texture_index, flags)
