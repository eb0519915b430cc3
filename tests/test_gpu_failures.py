"""Failure paths of the device library, made on purpose without faulting the
GPU: a bounded device loop that runs out, non-finite frames, and fits with no
usable stamps. Each failure must come back as the reference's error (or the
documented status) with the context still usable afterwards."""

from __future__ import annotations

import numpy as np
import pytest

import delta_b200 as delta
from delta_b200 import _core, _lib, validation
from oracle import cref, refbuild
from oracle import numpy_ref as nr

pytestmark = pytest.mark.gpu


def _snake(h=64, w=64):
    """One 8-connected component that winds through the frame: its union-find
    chains are long, so a loop cap of one step cannot resolve it."""
    score = np.zeros((h, w), np.float32)
    for y in range(1, h - 1, 4):
        score[y, 1 : w - 1] = 9.0
        x = w - 2 if (y // 4) % 2 == 0 else 1
        score[y : min(y + 4, h - 1), x] = 9.0
    return score


def test_label_loop_cap_reports_limit_and_the_context_recovers():
    score = _snake()
    ctx = _core.context()
    _lib.check(_lib.lib().dgpu_set_label_loop_cap(ctx.handle, 1), ctx.handle)
    try:
        with pytest.raises(_lib.DeviceLoopLimitError):
            _core.build_catalog(score, score, expected_fwhm=3.0)
    finally:
        _lib.check(_lib.lib().dgpu_set_label_loop_cap(ctx.handle, 0), ctx.handle)
    # the same context, default cap: labels equal the reference's CCL
    cat = _core.build_catalog(score, score, expected_fwhm=3.0)
    want, n = refbuild.label_components((score >= 5).astype(np.uint8)) if refbuild.available() else (None, 1)
    assert len(cat["x"]) == n == 1
    if want is not None:
        np.testing.assert_array_equal(_core.catalog_labels(score.shape), want)
    # and other work on it still runs
    img = np.random.default_rng(0).normal(0, 1, (64, 64)).astype(np.float32)
    psf = np.full((5, 5), 1 / 25, np.float32)
    var = np.ones_like(img)
    np.testing.assert_array_equal(_core.matched_filter(img, psf, var), cref.matched_filter(img, psf, var))


def test_non_finite_pixels_are_flagged_like_the_reference():
    """NaN / +-Inf pixels in either frame: the mask's non-finite bit and the
    exact-bad fill follow src/subtract.cpp:826-963 bit for bit."""
    p = validation.synthetic_pair(300, 260, 150, 5, mask_fraction=0.01)
    sci, ref = p.science.copy(), p.reference.copy()
    rng = np.random.default_rng(3)
    for img in (sci, ref):
        idx = rng.choice(img.size, 40, replace=False)
        img.flat[idx[:20]] = np.nan
        img.flat[idx[20:30]] = np.inf
        img.flat[idx[30:]] = -np.inf
    knots = nr.grid_knots(0, 0, 299, 259, 3, 3)
    theta = np.zeros(16 * 9)
    theta[15 * 9 : 16 * 9] = 0.0
    theta[0] = 1.0
    args = (sci, ref, knots, theta, 1.3, 4, 0, p.saturation, p.science_var, p.reference_var, p.science_mask,
            p.reference_mask)
    got = _core.subtract(*args)
    want = cref.subtract(*args)
    np.testing.assert_array_equal(got["mask"], want["mask"])
    assert np.any(got["mask"] & 8)
    np.testing.assert_array_equal(got["difference"], want["difference"])
    np.testing.assert_array_equal(got["variance"], want["variance"])


def test_all_nan_frame_and_background():
    """An all-NaN science frame has no finite sample: the background matches
    the reference's estimate_background, and subtract() stops at stamp
    selection with the reference's ValueError."""
    p = validation.synthetic_pair(256, 256, 120, 9)
    bad = np.full_like(p.science, np.nan)
    got = _core.estimate_background(bad)
    if refbuild.available():
        np.testing.assert_array_equal(np.array(got), np.array(refbuild.estimate_background(bad)))
    with pytest.raises(ValueError, match="no stamps selected"):
        delta.subtract(bad, p.reference, science_var=p.science_var, reference_var=p.reference_var)


def test_fit_without_usable_stamp_pixels_fails_like_the_reference():
    """No stamps, or stamps whose pixels are all masked: the reference raises
    runtime_error("fit_kernel: no usable stamp pixels") (src/fit.cpp:232)."""
    p = validation.synthetic_pair(200, 200, 60, 2, mask_fraction=0.0)
    knots = nr.grid_knots(0, 0, 199, 199, 3, 3)
    grid = np.logspace(-6, 6, 5)
    empty = np.zeros(0, np.int32)
    with pytest.raises(RuntimeError, match="no usable stamp pixels"):
        _core.fit_kernel(p.science, p.reference, knots, empty, empty, 10, 1.3, 2, grid)
    with pytest.raises(RuntimeError, match="no usable stamp pixels"):
        nr.fit_kernel(p.science, p.reference, knots, empty, empty, 10, 1.3, 2, grid)
    mask = np.full(p.science.shape, 1, np.uint8)
    xs, ys = np.array([50, 120], np.int32), np.array([60, 140], np.int32)
    with pytest.raises(RuntimeError, match="no usable stamp pixels"):
        _core.fit_kernel(p.science, p.reference, knots, xs, ys, 10, 1.3, 2, grid, science_mask=mask)
    # the context is still good for a real fit
    res = _core.fit_kernel(p.science, p.reference, knots, xs, ys, 10, 1.3, 2, grid)
    assert np.all(np.isfinite(res["theta"]))
