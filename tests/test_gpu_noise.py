"""GPU parity of the ZOGY decorrelation (batched block FFT with the filter
fused between passes, Hann overlap-add), the whitened score PSF and the QA
helpers, against the FP64 NumPy oracle (reference src/noise.cpp)."""

from __future__ import annotations

import numpy as np
import pytest

from delta_b200 import _core
from oracle import numpy_ref as nr

pytestmark = pytest.mark.gpu


def _setup(h, w, seed=0, n_max=3, beta=1.3, nk=3):
    rng = np.random.default_rng(seed)
    knots = nr.grid_knots(0, 0, w - 1, h - 1, nk, nk)
    nc = (n_max + 1) * (n_max + 2) // 2
    k = knots.shape[0]
    theta = 0.05 * rng.standard_normal((nc + 1) * k)
    theta[k - 3] = 1.0
    theta[k + k - 2] = 0.2  # a spatial gradient in c_1
    diff = (rng.standard_normal((h, w)) * 10.0).astype(np.float32)
    diff[h // 3, w // 4] += 500.0
    vs = rng.uniform(80.0, 120.0, (h, w)).astype(np.float32)
    vr = rng.uniform(40.0, 60.0, (h, w)).astype(np.float32)
    vs[5, 5] = 1e30  # sentinel; the block median ignores it
    return knots, theta, beta, n_max, diff, vs, vr


@pytest.mark.parametrize("h,w,block,cells", [(300, 420, 64, 0), (300, 420, 64, 1), (257, 190, 128, 0),
                                             (40, 50, 64, 0), (200, 200, 32, 2), (600, 700, 256, 0),
                                             (530, 520, 256, 1)])
def test_decorrelate_matches_fp64_oracle(h, w, block, cells):
    knots, theta, beta, n_max, diff, vs, vr = _setup(h, w)
    got = _core.decorrelate(diff, knots, theta, beta, n_max, vs, vr, block=block, kernel_cell_blocks=cells)
    want = nr.decorrelate(diff, knots, theta, beta, n_max, vs, vr, block=block, kernel_cell_blocks=cells)
    np.testing.assert_allclose(got["variance"], want["variance"], rtol=2e-6)
    sigma = np.sqrt(want["variance"])
    assert np.max(np.abs(got["difference"] - want["difference"]) / sigma) < 1e-4


def test_decorrelate_preserves_variance_and_flattens_noise():
    # reference tests/test_noise.py:37-66 (white noise convolved with K -> whitened)
    rng = np.random.default_rng(3)
    h = w = 256
    knots = nr.grid_knots(0, 0, w - 1, h - 1, 3, 3)
    beta, n_max = 1.5, 0
    theta = np.zeros(2 * 9)
    theta[6] = 1.0
    ref_noise = rng.standard_normal((h, w)) * np.sqrt(50.0)
    bn = _core.basis_convolve(ref_noise.astype(np.float32), beta, n_max)[0]
    diff = (rng.standard_normal((h, w)) * 10.0 - bn).astype(np.float32)
    vs = np.full((h, w), 100.0, np.float32)
    vr = np.full((h, w), 50.0, np.float32)
    out = _core.decorrelate(diff, knots, theta, beta, n_max, vs, vr, block=64)
    d = out["difference"][16:-16, 16:-16].astype(np.float64)
    lag1 = np.mean(d[:, 1:] * d[:, :-1]) / np.var(d)
    assert abs(lag1) < 0.03
    np.testing.assert_allclose(np.var(d), np.median(out["variance"]), rtol=0.1)


def test_whiten_score_psf_matches_oracle():
    knots, theta, beta, n_max, diff, vs, vr = _setup(300, 420)
    r = 8
    yy, xx = np.mgrid[-r : r + 1, -r : r + 1]
    psf = np.exp(-(xx**2 + yy**2) / (2 * 2.0**2))
    psf = (psf / psf.sum()).astype(np.float32)
    got = _core.whiten_score_psf(psf, knots, theta, beta, n_max, vs, vr, 64)
    want = nr.whiten_score_psf(psf, knots, theta, beta, n_max, vs, vr, 64)
    np.testing.assert_allclose(got, want, rtol=1e-5, atol=1e-7)
    assert abs(got.astype(np.float64).sum() - 1.0) < 1e-5
    with pytest.raises(RuntimeError):
        _core.whiten_score_psf(psf, knots, theta, beta, n_max, vs, vr, 8)


def test_decorrelate_block_and_kernel_match_oracle():
    rng = np.random.default_rng(5)
    n = 64
    img = rng.standard_normal((n, n)).astype(np.float32)
    yy, xx = np.mgrid[-5:6, -5:6]
    kern = np.exp(-(xx**2 + yy**2) / 4.0)
    kern = (kern / kern.sum()).astype(np.float32)
    got = _core.decorrelate_block(img, kern, 100.0, 50.0)
    filt = nr.decorrelation_filter(kern, 100.0, 50.0, n)
    want = nr.apply_filter_fft(img, filt)
    np.testing.assert_allclose(got, want, atol=2e-5)
    gk = _core.decorrelation_kernel(kern, 100.0, 50.0, n)
    np.testing.assert_allclose(gk, nr.decorrelation_kernel_image(filt, n), atol=2e-6)


def test_decorrelate_rejects_bad_block():
    knots, theta, beta, n_max, diff, vs, vr = _setup(64, 64)
    with pytest.raises(RuntimeError):
        _core.decorrelate(diff, knots, theta, beta, n_max, vs, vr, block=48)
