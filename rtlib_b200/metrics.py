"""Image error metrics and the result-image format of the test application.

``rmae`` / ``smape`` restate the comparison tool RTLibExtOPX7Comp.cpp:124-145 (all-range
branch); ``relmse`` is the relative mean squared error used for equal-time comparisons:
mean over pixels and channels of (img - ref)^2 / (ref^2 + eps), optionally after scaling both
images by the reference's mean.  ``save_result_bin`` writes
what SaveResultImage writes (RTLibExtOPX7TestApplication.cpp:2590-2610): float RGB mean
radiance with the pixel order reversed."""
from __future__ import annotations

import numpy as np


def relmse(img, ref, eps=1e-2, normalize=False):
    """normalize: divide both images by the reference's mean first, so that eps = 1e-2 means
    1% of the mean brightness (dark scenes otherwise compare only in their brightest pixels)."""
    img = np.asarray(img, np.float64)
    ref = np.asarray(ref, np.float64)
    if normalize:
        m = float(np.mean(ref[np.isfinite(ref)]))
        if m > 0:
            img, ref = img / m, ref / m
    ok = np.isfinite(img).all(axis=-1) & np.isfinite(ref).all(axis=-1)
    return float(np.mean(((img - ref) ** 2 / (ref ** 2 + eps))[ok]))


def relmse_denoised(img, ref_a, ref_b, n_a, n_b, eps=1e-2, normalize=False):
    """relMSE of img against the converged image, estimated from two independent reference
    renders of n_a and n_b samples per pixel.  Against their weighted mean r, the error of img
    is E[(img - t)^2] + Var(r) (t the converged image, img independent of r); with per-sample
    variance s^2, Var(r) = s^2 / (n_a + n_b) and E[(a - b)^2] = s^2 (1/n_a + 1/n_b), so
    Var(r) = E[(a - b)^2] * n_a n_b / (n_a + n_b)^2, which is subtracted per pixel with the
    same denominator.  Returns (relmse vs r, the estimate with r's variance removed)."""
    a = np.asarray(ref_a, np.float64)
    b = np.asarray(ref_b, np.float64)
    img = np.asarray(img, np.float64)
    r = (n_a * a + n_b * b) / float(n_a + n_b)
    if normalize:
        m = float(np.mean(r[np.isfinite(r)]))
        if m > 0:
            img, r, a, b = img / m, r / m, a / m, b / m
    ok = np.isfinite(img).all(axis=-1) & np.isfinite(a).all(axis=-1) & np.isfinite(b).all(axis=-1)
    den = r ** 2 + eps
    raw = (img - r) ** 2 / den
    c = float(n_a) * float(n_b) / float(n_a + n_b) ** 2
    noise = c * (a - b) ** 2 / den
    return float(np.mean(raw[ok])), float(np.mean((raw - noise)[ok]))


def rmae(img, ref):
    """sum |img - ref| (Euclidean RGB distance) / sum (|ref| + |img|) / 2 over pixels with ref != 0."""
    b = np.asarray(ref, np.float32).reshape(-1, 3)
    c = np.asarray(img, np.float32).reshape(-1, 3)
    ok = ~(np.isnan(b).any(1) | np.isnan(c).any(1))
    nb = np.sqrt((b ** 2).sum(1))
    m = ok & (nb > 0)
    d = np.sqrt(((b - c) ** 2).sum(1))
    mean = ((nb + np.sqrt((c ** 2).sum(1))) * 0.5)[m].sum()
    return float(d[m].sum() / mean) if mean > 0 else 0.0


def smape(img, ref):
    """mean over all pixels of |img - ref| / |ref| (Euclidean RGB), pixels with ref = 0 adding 0."""
    b = np.asarray(ref, np.float32).reshape(-1, 3)
    c = np.asarray(img, np.float32).reshape(-1, 3)
    ok = ~(np.isnan(b).any(1) | np.isnan(c).any(1))
    nb = np.sqrt((b ** 2).sum(1))
    m = ok & (nb > 0)
    d = np.sqrt(((b - c) ** 2).sum(1))
    return float((d[m] / nb[m]).sum() / b.shape[0])


def save_result_bin(path, mean_rgb):
    """mean_rgb: (h, w, 3) float; written with the pixel order reversed, float32."""
    a = np.asarray(mean_rgb, np.float32).reshape(-1, 3)[::-1]
    a.tofile(path)


def load_result_bin(path, width, height):
    a = np.fromfile(path, np.float32).reshape(-1, 3)[::-1]
    return a.reshape(height, width, 3)
