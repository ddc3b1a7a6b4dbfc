"""Error metrics and the result-image format (CPU)."""
import numpy as np

from rtlib_b200 import metrics


def test_relmse_rmae_smape_small_cases(tmp_path):
    ref = np.array([[[1.0, 1.0, 1.0], [0.0, 0.0, 0.0]]], np.float32)
    img = np.array([[[1.1, 1.0, 0.9], [0.0, 0.0, 0.0]]], np.float32)
    # relMSE: (0.01 / 1.01 + 0 + 0.01 / 1.01) / 6
    assert abs(metrics.relmse(img, ref) - (0.02 / 1.01) / 6) < 1e-7
    d = np.sqrt(0.02)
    assert abs(metrics.smape(img, ref) - d / np.sqrt(3) / 2) < 1e-6
    mean = (np.sqrt(3) + np.sqrt(1.21 + 1 + 0.81)) / 2
    assert abs(metrics.rmae(img, ref) - d / mean) < 1e-6
    assert metrics.relmse(ref, ref) == 0.0
    # normalised: scale invariant
    a, b = metrics.relmse(img * 1e-3, ref * 1e-3, normalize=True), metrics.relmse(img, ref, normalize=True)
    assert b > 0 and abs(a - b) < 1e-5 * b
    p = tmp_path / "r.bin"
    metrics.save_result_bin(p, img)
    raw = np.fromfile(p, np.float32).reshape(-1, 3)
    assert np.array_equal(raw[0], img[0, 1]) and np.array_equal(raw[1], img[0, 0])
    assert np.array_equal(metrics.load_result_bin(p, 2, 1), img)


def test_relmse_denoised_removes_reference_noise():
    # truth t, image and two references with independent Gaussian noise of per-sample
    # variance s^2: the de-noised estimate recovers the image's own error
    rng = np.random.default_rng(0)
    t = rng.uniform(0.5, 2.0, (256, 256, 3))
    s, n_img, n_a, n_b = 0.5, 16, 40, 24
    img = t + rng.normal(0, s / np.sqrt(n_img), t.shape)
    a = t + rng.normal(0, s / np.sqrt(n_a), t.shape)
    b = t + rng.normal(0, s / np.sqrt(n_b), t.shape)
    raw, den = metrics.relmse_denoised(img, a, b, n_a, n_b)
    r = (n_a * a + n_b * b) / (n_a + n_b)
    assert abs(raw - metrics.relmse(img, r)) < 1e-12
    truth = metrics.relmse(img, t)
    assert raw > 1.15 * truth
    assert abs(den - truth) < 0.03 * truth
