"""The CPU restatement of the learned guide (oracle/mlp_oracle.py): bf16 rounding and the
analytic output-layer gradient against central differences (CPU only)."""
import numpy as np

from oracle import mlp_oracle as M


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.01171875, -2.5, 3.1415927, 0.0], np.float32)
    assert M.bf16(x).tolist() == [1.0, 1.0, 1.015625, -2.5, 3.140625, 0.0]


def test_head_gradient_central_differences():
    rng = np.random.default_rng(1)
    n = 4
    o = rng.normal(size=(n, 48)) * 0.8
    wi = rng.normal(size=(n, 3))
    wi /= np.linalg.norm(wi, axis=1, keepdims=True)
    wt = rng.uniform(0.5, 2, n)

    def loss(o):
        return float((wt * -np.log(M.mixture_pdf(o, wi))).sum() / wt.sum())

    # the oracle's analytic gradient of the raw outputs, without the bf16 rounding of the
    # backward pass: a one-layer network whose output is o (identity input, identity weights)
    mu, kappa, wgt, ln, s = M.head(o)
    fk = M.vmf_pdf(mu, kappa, wi)
    q = (wgt * fk).sum(1)
    r = wgt * fk / q[:, None]
    mw = (mu * wi[:, None, :]).sum(-1)
    gm = (wi[:, None, :] - mu * mw[..., None]) * (r * kappa / ln)[..., None]
    e = np.exp(-2 * kappa)
    gs = r * kappa * (1 / kappa - 2 * e / (1 - e) + (mw - 1))
    g = np.concatenate([gm, gs[..., None], (r - wgt)[..., None]], axis=2).reshape(n, 40)
    g *= -(wt / wt.sum())[:, None]
    fd = np.zeros_like(g)
    for i in range(n):
        for j in range(40):
            a, b = o.copy(), o.copy()
            a[i, j] += 1e-6
            b[i, j] -= 1e-6
            fd[i, j] = (loss(a) - loss(b)) / 2e-6
    assert np.abs(g - fd).max() < 1e-7 * max(1.0, np.abs(fd).max())


def test_mixture_is_normalised():
    rng = np.random.default_rng(2)
    o = rng.normal(size=(1, 48))
    # Monte Carlo over the sphere: E[q] * 4 pi = 1
    d = rng.normal(size=(200000, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    q = M.mixture_pdf(np.repeat(o, d.shape[0], 0), d)
    assert abs(q.mean() * 4 * np.pi - 1.0) < 0.02
