"""Path-replay adjoint (rtpg_tracer_render_adjoint) against common-random-number central
finite differences of the same estimator.

The parameters are the back-wall albedo texture and the emitter radiances of the Cornell box
with its ceiling light split into 4 x 4 emitters; the loss is the mean squared difference to a
target rendered with a perturbed texture.  With the same per-pixel streams, a change of a
parameter changes no sampling decision (cosine sampling, light selection and RIS-free NEE do
not depend on albedo or radiance), so the estimator is a smooth function of the parameters
and its central difference at eps = 1e-3 must match the adjoint within 2%."""
import numpy as np
import pytest

from rtlib_b200 import scenes

pytestmark = pytest.mark.gpu

W = H = 64
SPP = 16
TEX = 32
EPS = 1e-3


def _setup(cuda, seed=7):
    import torch
    from rtlib_b200.tracer import Tracer
    sc = scenes.cornell_box(W, H, light_grid=4, back_texture=True)
    rng = np.random.default_rng(seed)
    tex0 = rng.uniform(0.2, 0.9, (TEX, TEX, 3)).astype(np.float32)
    target_tex = np.clip(tex0 + rng.normal(0.0, 0.05, tex0.shape), 0.0, 1.0).astype(np.float32)
    light0 = np.asarray(sc["light_emission"], np.float32).reshape(-1, 3).copy()
    tex = torch.from_numpy(tex0).to(cuda)
    tr = Tracer(sc, cuda, max_depth=8, width=W, height=H, textures={0: tex})
    # target image: perturbed texture, more samples
    ttex = torch.from_numpy(target_tex).to(cuda)
    tr.set_texture(0, ttex)
    tr.clear()
    tr.render(4 * SPP, 1)
    target = tr.image64()
    tr.set_texture(0, tex)
    return sc, tr, tex, light0, target


def _per_channel_loss(tr, target):
    import torch
    tr.clear()
    tr.render(SPP, 1)
    img = tr.image64()
    return ((img - target) ** 2).sum(dim=(0, 1)) / (3.0 * W * H), img


def _adjoint(cuda, tr, target, light0):
    import torch
    _, img = _per_channel_loss(tr, target)
    d_img = (2.0 * (img - target) / (3.0 * W * H)).float().contiguous()
    g_tex = torch.zeros((TEX, TEX, 3), dtype=torch.float32, device=cuda)
    g_light = torch.zeros((light0.shape[0], 3), dtype=torch.float32, device=cuda)
    tr.clear()
    tr.render_adjoint(SPP, d_img, 1, 0, g_tex, g_light)
    return g_tex.cpu().numpy(), g_light.cpu().numpy()


def _check(adj, fd, tol=0.02):
    adj, fd = np.asarray(adj, np.float64).ravel(), np.asarray(fd, np.float64).ravel()
    assert np.abs(fd).max() > 0
    big = np.abs(fd) > 1e-2 * np.abs(fd).max()
    rel = np.abs(adj[big] - fd[big]) / np.abs(fd[big])
    assert rel.max() < tol, (rel.max(), np.argmax(rel))
    assert np.linalg.norm(adj - fd) < tol * np.linalg.norm(fd)
    return rel


def test_adjoint_matches_central_differences(cuda):
    import torch
    sc, tr, tex, light0, target = _setup(cuda)
    g_tex, g_light = _adjoint(cuda, tr, target, light0)
    rng = np.random.default_rng(11)
    texels = rng.choice(TEX * TEX, 48, replace=False)
    fd_tex = np.zeros((len(texels), 3))
    for k, t in enumerate(texels):
        y, x = divmod(int(t), TEX)
        base = tex[y, x].clone()
        tex[y, x] = base + EPS
        lp, _ = _per_channel_loss(tr, target)
        tex[y, x] = base - EPS
        lm, _ = _per_channel_loss(tr, target)
        tex[y, x] = base
        fd_tex[k] = ((lp - lm) / (2 * EPS)).cpu().numpy()
    adj_tex = g_tex.reshape(-1, 3)[texels]
    _check(adj_tex, fd_tex)
    fd_light = np.zeros_like(light0, dtype=np.float64)
    for i in range(light0.shape[0]):
        l = light0.copy()
        l[i] += EPS
        tr.set_light_emission(l)
        lp, _ = _per_channel_loss(tr, target)
        l[i] -= 2 * EPS
        tr.set_light_emission(l)
        lm, _ = _per_channel_loss(tr, target)
        fd_light[i] = ((lp - lm) / (2 * EPS)).cpu().numpy()
    tr.set_light_emission(light0)
    _check(g_light, fd_light)


def test_autograd_wrapper(cuda):
    """rtlib_b200.diff.render gives the same gradients through torch.autograd."""
    import torch
    from rtlib_b200 import diff
    sc, tr, tex, light0, target = _setup(cuda)
    g_tex, g_light = _adjoint(cuda, tr, target, light0)
    p_tex = tex.clone().requires_grad_(True)
    p_light = torch.from_numpy(light0.copy()).requires_grad_(True)
    img = diff.render(p_tex, p_light, tr, SPP, 0)
    loss = ((img.double() - target.float().double()) ** 2).mean()
    loss.backward()
    np.testing.assert_allclose(p_tex.grad.cpu().numpy(), g_tex, rtol=1e-3, atol=1e-9)
    np.testing.assert_allclose(p_light.grad.numpy(), g_light, rtol=1e-3, atol=1e-9)


def test_adjoint_against_cpu_oracle_differences(cuda, oracle):
    """The same gradients against central differences of the CPU restatement of the
    integrator (oracle), on a few texels and all emitters.  CPU and GPU follow the same random
    numbers; the few paths that separate on float differences of sin/cos widen the bound."""
    from oracle.oracle import OracleRenderer
    sc, tr, tex, light0, target = _setup(cuda)
    g_tex, g_light = _adjoint(cuda, tr, target, light0)
    tnp = target.cpu().numpy()
    texture = tex.cpu().numpy().copy()
    r = OracleRenderer(oracle, sc, width=W, height=H, texture=texture)
    lmf = sc["light_material_first"]

    def loss():
        r.restart()
        r.render(SPP, 1)
        img = r.accum.reshape(H, W, 3) / r.samples
        return ((img - tnp) ** 2).sum(axis=(0, 1)) / (3.0 * W * H)

    rng = np.random.default_rng(11)
    texels = rng.choice(TEX * TEX, 8, replace=False)
    fd_tex = np.zeros((len(texels), 3))
    for k, t in enumerate(texels):
        y, x = divmod(int(t), TEX)
        base = r.tex[y, x].copy()
        r.tex[y, x] = base + EPS
        lp = loss()
        r.tex[y, x] = base - EPS
        lm = loss()
        r.tex[y, x] = base
        fd_tex[k] = (lp - lm) / (2 * EPS)
    fd_light = np.zeros_like(light0, dtype=np.float64)
    for i in range(light0.shape[0]):
        l = light0.copy()
        l[i] += EPS
        r.set_light_emission(l, lmf)
        lp = loss()
        l[i] -= 2 * EPS
        r.set_light_emission(l, lmf)
        lm = loss()
        fd_light[i] = (lp - lm) / (2 * EPS)
    adj = np.concatenate([g_tex.reshape(-1, 3)[texels].ravel(), g_light.ravel()])
    fd = np.concatenate([fd_tex.ravel(), fd_light.ravel()])
    assert np.linalg.norm(adj - fd) < 0.05 * np.linalg.norm(fd)


def test_config4_adjoint_matches_central_differences(cuda):
    """512 texels of the 256 x 256 texture and all 16 emitters at 512 x 512, 64 spp: every
    checked gradient within 2 % of its central difference (gradients below 1 % of the largest
    one are float noise in the difference and enter only the norm check)."""
    from rtlib_b200 import diff
    r = diff.config4_gradients(cuda)
    _check(r["adj_texels"], r["fd_texels"])
    _check(r["adj_lights"], r["fd_lights"])
