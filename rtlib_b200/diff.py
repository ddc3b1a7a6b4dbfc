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


def config4_gradients(device, n_texels=512, width=512, height=512, tex_size=256, spp=64, seed=4, eps=1e-3):
    """The differentiable-rendering configuration and its gradient check: the Cornell box at
    width x height with a tex_size^2 RGB albedo texture on the back wall (U[0.2, 0.9]) and its
    ceiling light split into 4 x 4 emitters; the target is rendered (4 x spp, another seed)
    with the texture perturbed by N(0, 0.05) per texel and clamped to [0, 1]; the loss is the L2
    image difference.  Forward and adjoint use spp samples, max depth 8, NEE, replaying the same
    per-pixel streams.  Returns the adjoint gradients and the central differences (eps, common
    random numbers: every render restarts the same streams) of n_texels random texels (3
    channels each) and of all emitters as flat arrays, and the device milliseconds of the
    forward render and of the adjoint."""
    import numpy as np

    from . import scenes
    from .tracer import Tracer
    sc = scenes.cornell_box(width, height, light_grid=4, back_texture=True)
    rng = np.random.default_rng(seed)
    tex0 = rng.uniform(0.2, 0.9, (tex_size, tex_size, 3)).astype(np.float32)
    target_tex = np.clip(tex0 + rng.normal(0.0, 0.05, tex0.shape), 0.0, 1.0).astype(np.float32)
    light0 = np.asarray(sc["light_emission"], np.float32).reshape(-1, 3).copy()
    tex = torch.from_numpy(tex0).to(device)
    tr = Tracer(sc, device, max_depth=8, width=width, height=height, textures={0: tex}, seed=seed + 100)
    tr.set_texture(0, torch.from_numpy(target_tex).to(device))
    tr.clear()
    tr.render(4 * spp, FLAG_NEE)
    target = tr.image64()
    tr.set_texture(0, tex)
    tr.set_seed(seed)
    npx = 3.0 * width * height

    def loss():
        tr.clear()
        tr.render(spp, FLAG_NEE)
        img = tr.image64()
        return ((img - target) ** 2).sum(dim=(0, 1)) / npx, img

    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    ev[0].record()
    _, img = loss()
    ev[1].record()
    d_img = (2.0 * (img - target) / npx).float().contiguous()
    g_tex = torch.zeros_like(tex)
    g_light = torch.zeros((light0.shape[0], 3), dtype=torch.float32, device=device)
    tr.clear()
    tr.render_adjoint(spp, d_img, FLAG_NEE, 0, g_tex, g_light)
    ev[2].record()
    torch.cuda.synchronize()
    texels = rng.choice(tex_size * tex_size, n_texels, replace=False)
    fd_tex = np.zeros((n_texels, 3))
    for k, t in enumerate(texels):
        y, x = divmod(int(t), tex_size)
        base = tex[y, x].clone()
        tex[y, x] = base + eps
        lp, _ = loss()
        tex[y, x] = base - eps
        lm, _ = loss()
        tex[y, x] = base
        fd_tex[k] = ((lp - lm) / (2 * eps)).cpu().numpy()
    fd_light = np.zeros_like(light0, dtype=np.float64)
    for i in range(light0.shape[0]):
        lt = light0.copy()
        lt[i] += eps
        tr.set_light_emission(lt)
        lp, _ = loss()
        lt[i] -= 2 * eps
        tr.set_light_emission(lt)
        lm, _ = loss()
        fd_light[i] = ((lp - lm) / (2 * eps)).cpu().numpy()
    tr.set_light_emission(light0)
    adj_tex = g_tex.reshape(-1, 3)[torch.from_numpy(texels).to(device)].cpu().numpy()
    return {"adj_texels": adj_tex.ravel(), "fd_texels": fd_tex.ravel(), "adj_lights": g_light.cpu().numpy().ravel(),
            "fd_lights": fd_light.ravel(), "forward_ms": ev[0].elapsed_time(ev[1]),
            "adjoint_ms": ev[1].elapsed_time(ev[2]), "paths_per_render": width * height * spp}
