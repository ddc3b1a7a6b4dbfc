"""CPU restatement of the learned guide's network (TEST INFRASTRUCTURE ONLY: the checker of
rtlib_b200/csrc/mlp.cu; nothing in the product imports it).

numpy, float64 arithmetic with the roundings the GPU path makes: features, weights and hidden
activations rounded to bfloat16 (round to nearest even), output-layer gradients and the
backward activations' gradients rounded to bfloat16 before they enter the next product, fp32
network outputs.  Layouts and formulas follow rtlib_b200/csrc/mlp_dev.cuh and mlp.cu."""
from __future__ import annotations

import numpy as np

N_IN, N_H, N_OUT, LOBES, FREQS = 80, 64, 48, 8, 12
OFF = (0, 80 * 64, 80 * 64 + 64 * 64, 80 * 64 + 2 * 64 * 64)
SHAPES = ((80, 64), (64, 64), (64, 64), (64, 48))
LK_MIN, LK_MAX = -2.3, 6.9
W_CLAMP = 20.0


def bf16(x):
    """Round float32 values to bfloat16 (nearest even), returned as float32."""
    a = np.ascontiguousarray(x, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).reshape(a.shape)


def unpack(w):
    return [np.asarray(w[o:o + a * b], np.float32).reshape(a, b) for o, (a, b) in zip(OFF, SHAPES)]


def features(pos, nrm, wo, mn, mx):
    pos = np.asarray(pos, np.float32)
    u = ((pos - np.asarray(mn, np.float32)) * (np.float32(1.0) / (np.asarray(mx, np.float32) - np.asarray(mn, np.float32)))).astype(np.float32)
    n = pos.shape[0]
    f = np.zeros((n, N_IN), np.float32)
    for c in range(3):
        a = u[:, c].astype(np.float64)
        for j in range(FREQS):
            f[:, c * 24 + 2 * j] = np.sin(np.pi * a)
            f[:, c * 24 + 2 * j + 1] = np.cos(np.pi * a)
            a = a * 2.0
    f[:, 72:75] = nrm
    f[:, 75:78] = wo
    f[:, 78] = 1.0
    return f


def forward(w, x):
    """Raw outputs (n, 48) and the bf16 activations [X0, H1, H2, H3]."""
    W = [bf16(m).astype(np.float64) for m in unpack(w)]
    acts = [bf16(x)]
    h = acts[0].astype(np.float64)
    for l in range(3):
        h = bf16(np.maximum(h @ W[l], 0.0).astype(np.float32)).astype(np.float64)
        acts.append(h.astype(np.float32))
    o = (h @ W[3]).astype(np.float32)
    return o, acts


def head(o):
    o = np.asarray(o, np.float64)
    n = o.shape[0]
    m = o[:, :40].reshape(n, LOBES, 5)
    mu_raw = m[:, :, :3]
    ln = np.maximum(np.linalg.norm(mu_raw, axis=2, keepdims=True), 1e-12)
    mu = mu_raw / ln
    s = m[:, :, 3]
    kappa = np.exp(np.clip(s, LK_MIN, LK_MAX))
    a = m[:, :, 4]
    e = np.exp(a - a.max(axis=1, keepdims=True))
    wgt = e / e.sum(axis=1, keepdims=True)
    return mu, kappa, wgt, ln[..., 0], s


def vmf_pdf(mu, kappa, w):
    return kappa / (2 * np.pi * (1 - np.exp(-2 * kappa))) * np.exp(kappa * ((mu * w[:, None, :]).sum(-1) - 1))


def mixture_pdf(o, w):
    mu, kappa, wgt, _, _ = head(o)
    return (wgt * vmf_pdf(mu, kappa, np.asarray(w, np.float64))).sum(1)


def loss_grad(w, x, wi, weight):
    """Loss -sum w log q / sum w and its gradient (16384,) as the GPU computes them."""
    W = [bf16(m).astype(np.float64) for m in unpack(w)]
    o, acts = forward(w, x)
    wi = np.asarray(wi, np.float64)
    weight = np.maximum(np.asarray(weight, np.float32), 0.0)
    sw = float(weight.astype(np.float64).sum())
    scale = 1.0 / sw if sw > 0 else 0.0
    # the weight clamp of the training kernel: 20 x the mean weight of the call
    weight = np.minimum(weight, np.float32(20.0) * np.float32(sw / weight.shape[0])).astype(np.float64)
    mu, kappa, wgt, ln, s = head(o)
    fk = vmf_pdf(mu, kappa, wi)
    q = np.maximum((wgt * fk).sum(1), 1e-30)
    loss = float((weight * -np.log(q)).sum() * scale)
    r = wgt * fk / q[:, None]
    mw = (mu * wi[:, None, :]).sum(-1)
    gm = (wi[:, None, :] - mu * mw[..., None]) * (r * kappa / ln)[..., None]
    e = np.exp(-2 * kappa)
    dlk = 1 / kappa - 2 * e / (1 - e) + (mw - 1)
    gs = np.where((s > LK_MIN) & (s < LK_MAX), r * kappa * dlk, 0.0)
    ga = r - wgt
    sc = -(weight * scale)[:, None]
    g = np.zeros((o.shape[0], N_H))
    gl = np.concatenate([gm, gs[..., None], ga[..., None]], axis=2).reshape(-1, 40)
    g[:, :40] = gl * sc
    dy = bf16(g.astype(np.float32)).astype(np.float64)
    grads = [None] * 4
    for l in (3, 2, 1, 0):
        xin = acts[l].astype(np.float64)
        grads[l] = xin.T @ dy[:, :SHAPES[l][1]]
        if l > 0:
            dx = dy[:, :SHAPES[l][1]] @ W[l].T
            dx = np.where(acts[l] > 0, dx, 0.0)
            dy = bf16(dx.astype(np.float32)).astype(np.float64)
    return loss, np.concatenate([gr.ravel() for gr in grads]).astype(np.float64)
