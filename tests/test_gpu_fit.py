"""GPU parity of the penalised GLS (GCV / CV / fixed lambda) and the stamp fit
(IRLS + clipping) against the FP64 oracle, plus the reference's analytic
solver checks (tests/test_solve.py:24-85 of tkillestein/delta)."""

from __future__ import annotations

import numpy as np
import pytest

from delta_b200 import _core, _lib
from oracle import numpy_ref as nr
from oracle import refbuild

pytestmark = pytest.mark.gpu

GRID = np.logspace(-6, 6, 25)


def _problem(seed=0, n=3000, nc=6, nk=4, noise=0.05):
    rng = np.random.default_rng(seed)
    knots = nr.grid_knots(0, 0, 499, 399, nk, nk)
    pts = np.column_stack([rng.uniform(0, 500, n), rng.uniform(0, 400, n)])
    bn = rng.standard_normal((n, nc)) * rng.uniform(0.5, 5.0, nc)
    k = knots.shape[0]
    theta_true = rng.standard_normal((nc + 1) * k) * 0.3
    tp = nr.ThinPlate(knots)
    d = tp.design(pts)
    c = theta_true.reshape(nc + 1, k).T
    f = d @ c
    target = f[:, nc] + np.sum(f[:, :nc] * bn, axis=1) + noise * rng.standard_normal(n)
    weights = rng.uniform(0.5, 2.0, n)
    return knots, pts, target, weights, bn, theta_true


def test_solve_gls_gcv_matches_oracle():
    knots, pts, t, w, bn, _ = _problem()
    got = _core.solve_gls_gcv(knots, pts, t, w, bn, GRID)
    want = nr.solve_gls_gcv(knots, pts, t, w, bn, GRID)
    assert got["lambda"] == want["lambda"]
    np.testing.assert_allclose(got["theta"], want["theta"], rtol=1e-7, atol=1e-9)
    np.testing.assert_allclose(got["gcv_curve"], want["gcv_curve"], rtol=1e-6)
    np.testing.assert_allclose(got["effective_dof"], want["effective_dof"], rtol=1e-8)
    np.testing.assert_allclose(got["rss"], want["rss"], rtol=1e-6)
    assert got["n_components"] == 6 and got["n_spatial"] == 16


def test_solve_gls_fixed_lambda_and_edf_limits():
    knots, pts, t, w, bn, _ = _problem(1, n=2000, nc=3, nk=3)
    for lam in (1e-8, 1e-2, 1e8):
        got = _core.solve_gls(knots, pts, t, w, bn, lam)
        want = nr.solve_gls(knots, pts, t, w, bn, lam)
        np.testing.assert_allclose(got["theta"], want["theta"], rtol=1e-7, atol=1e-9)
        np.testing.assert_allclose(got["effective_dof"], want["effective_dof"], rtol=1e-7, atol=1e-6)
        assert got["lambda_grid"].size == 0 and got["gcv_curve"].size == 0
    p = 4 * 9
    assert abs(_core.solve_gls(knots, pts, t, w, bn, 1e-10)["effective_dof"] - p) < 1e-3
    assert abs(_core.solve_gls(knots, pts, t, w, bn, 1e12)["effective_dof"] - 3 * 4) < 1e-2


def test_solve_gls_exact_recovery():
    knots, pts, t, w, bn, theta = _problem(2, n=2500, nc=3, nk=3, noise=0.0)
    got = _core.solve_gls(knots, pts, t, w, bn, 1e-10)
    np.testing.assert_allclose(got["theta"], theta, rtol=1e-5, atol=1e-6)


def test_solve_gls_cv_matches_oracle():
    knots, pts, t, w, bn, _ = _problem(3, n=2400, nc=4, nk=3)
    group = np.arange(t.size) % 4
    got = _core.solve_gls_cv(knots, pts, t, w, bn, GRID, group, 4)
    want = nr.solve_gls_cv(knots, pts, t, w, bn, GRID, group, 4)
    assert got["lambda"] == want["lambda"]
    fin = np.isfinite(want["gcv_curve"])
    assert np.array_equal(np.isfinite(got["gcv_curve"]), fin)
    np.testing.assert_allclose(got["gcv_curve"][fin], want["gcv_curve"][fin], rtol=1e-6)
    np.testing.assert_allclose(got["theta"], want["theta"], rtol=1e-7, atol=1e-9)
    # n_groups < 2 degrades to GCV; bad group ids raise like the reference.
    g1 = _core.solve_gls_cv(knots, pts, t, w, bn, GRID, group, 1)
    assert g1["lambda"] == nr.solve_gls_gcv(knots, pts, t, w, bn, GRID)["lambda"]
    with pytest.raises(RuntimeError):
        _core.solve_gls_cv(knots, pts, t, w, bn, GRID, group + 10, 4)
    with pytest.raises(RuntimeError):
        _core.solve_gls_gcv(knots, pts, t, w, bn, np.zeros(0))


def test_solve_gls_gcv_large_system_matches_oracle():
    """The shape of a full-frame fit (28 components, 5x5 knots: 725 unknowns,
    23 factor tiles) in FP64 against the oracle. Mixed precision: its GCV curve
    within 2e-4 of the oracle's over the grid points within two steps of the
    minimum (measured 2.8e-5: the rss excess of the unrefined BF16x3
    solutions, second order in their error) and within 2e-3 elsewhere
    (measured 3.3e-4, far from the anchor of the rss expansion); the curve is
    flat to 1.2e-5 between the grid points around this minimum, so the argmin
    may move one grid step. Theta at the oracle's lambda, after its FP64
    refinement step, within 2e-5 (measured 3.9e-6)."""
    knots, pts, t, w, bn, _ = _problem(5, n=30000, nc=28, nk=5, noise=0.05)
    got = _core.solve_gls_gcv(knots, pts, t, w, bn, GRID)
    want = nr.solve_gls_gcv(knots, pts, t, w, bn, GRID)
    assert got["lambda"] == want["lambda"]
    assert got["theta"].size == 29 * 25
    np.testing.assert_allclose(got["theta"], want["theta"], rtol=1e-6, atol=1e-8)
    np.testing.assert_allclose(got["gcv_curve"], want["gcv_curve"], rtol=1e-6)
    np.testing.assert_allclose(got["effective_dof"], want["effective_dof"], rtol=1e-7)
    mixed = _core.solve_gls_gcv(knots, pts, t, w, bn, GRID, precision="mixed")
    # a refinement correction of 2.5e-3 keeps the mixed solve (fallback above 1e-2)
    assert mixed["precision_used"] == "mixed" and 0.0 < mixed["refine_correction"] < 1e-2
    i = int(np.argmin(want["gcv_curve"]))
    near = slice(max(0, i - 2), i + 3)
    np.testing.assert_allclose(mixed["gcv_curve"][near], want["gcv_curve"][near], rtol=2e-4)
    np.testing.assert_allclose(mixed["gcv_curve"], want["gcv_curve"], rtol=2e-3)
    assert abs(np.log10(mixed["lambda"] / want["lambda"])) <= 0.5 + 1e-9
    fixed = _core.solve_gls(knots, pts, t, w, bn, want["lambda"], precision="mixed")
    err = np.linalg.norm(fixed["theta"] - want["theta"]) / np.linalg.norm(want["theta"])
    assert err < 2e-5, err


def test_solve_gls_cv_large_system_mixed_close_to_oracle():
    """Mixed-precision group CV at the 725-unknown shape: held-out errors within
    5e-4 of the oracle's wherever both searched a lambda (measured 9.5e-5), the
    choice within one grid step, theta within 2e-5 of the oracle's fit at the
    chosen lambda."""
    knots, pts, t, w, bn, _ = _problem(5, n=30000, nc=28, nk=5, noise=0.05)
    group = np.arange(t.size) % 4
    got = _core.solve_gls_cv(knots, pts, t, w, bn, GRID, group, 4, precision="mixed")
    want = nr.solve_gls_cv(knots, pts, t, w, bn, GRID, group, 4)
    both = np.isfinite(got["gcv_curve"]) & np.isfinite(want["gcv_curve"])
    assert both.sum() >= 5
    np.testing.assert_allclose(got["gcv_curve"][both], want["gcv_curve"][both], rtol=5e-4)
    assert abs(np.log10(got["lambda"] / want["lambda"])) <= 0.5 + 1e-9
    fit = nr.solve_gls(knots, pts, t, w, bn, got["lambda"])
    err = np.linalg.norm(got["theta"] - fit["theta"]) / np.linalg.norm(fit["theta"])
    assert err < 2e-5, err


@pytest.mark.parametrize("precision", ["fp32", "mixed", "tf32"])
def test_reduced_precision_modes_close_to_fp64(precision):
    """As a fit runs by default: FP32 SIMT within 1e-3; the tensor-core builds
    after their FP64 refinement step within 1e-6 (BF16x3 is kept; TF32, about
    11 significant bits per operand, is redone in FP64 when its refinement step
    shows it too coarse for the system, and TF32 kept or not, the result is
    within 1e-6)."""
    knots, pts, t, w, bn, _ = _problem(4, n=6000, nc=6, nk=4, noise=0.05)
    ref = _core.solve_gls_gcv(knots, pts, t, w, bn, GRID, precision="fp64")
    got = _core.solve_gls_gcv(knots, pts, t, w, bn, GRID, precision=precision)
    err = np.linalg.norm(got["theta"] - ref["theta"]) / np.linalg.norm(ref["theta"])
    assert err < {"fp32": 1e-3, "mixed": 1e-6, "tf32": 1e-6}[precision], err
    if precision == "mixed":
        assert got["precision_used"] == "mixed", got["precision_used"]
    if precision == "tf32":
        assert got["precision_used"] in ("tf32", "fp64"), got["precision_used"]


def test_tensor_core_builds_without_fallback():
    """The BF16x3 and TF32 builds measured as they are (the context's FP64
    fallback off): each runs in its own arithmetic, TF32's first solve is
    coarser than BF16x3's (its refinement correction is larger), and the
    refinement step leaves each with an error below its own correction."""
    knots, pts, t, w, bn, _ = _problem(4, n=6000, nc=6, nk=4, noise=0.05)
    lam = 1e-2
    ref = _core.solve_gls(knots, pts, t, w, bn, lam, precision="fp64")
    ctx = _lib.context()
    ctx.set_precision_fallback(False)
    try:
        got = {p: _core.solve_gls(knots, pts, t, w, bn, lam, precision=p) for p in ("mixed", "tf32")}
    finally:
        ctx.set_precision_fallback(True)
    corr, err = {}, {}
    for p, g in got.items():
        assert g["precision_used"] == p, (p, g["precision_used"])
        corr[p] = g["refine_correction"]
        err[p] = np.linalg.norm(g["theta"] - ref["theta"]) / np.linalg.norm(ref["theta"])
        assert np.isfinite(corr[p]) and err[p] < max(corr[p], 1e-9), (p, corr[p], err[p])
    print("refinement corrections", corr, "errors after refinement", err)
    assert corr["tf32"] > corr["mixed"], corr


# ---------------------------------------------------------------------------- fit


def _fit_frame(seed=0, h=220, w=240, n_star=30, stamp_radius=7):
    rng = np.random.default_rng(seed)
    ys, xs = np.mgrid[0:h, 0:w]
    ref = np.full((h, w), 100.0)
    sci = np.full((h, w), 100.0)
    pos = []
    while len(pos) < n_star:
        x, y = rng.uniform(12, w - 12), rng.uniform(12, h - 12)
        if all((x - a) ** 2 + (y - b) ** 2 > 20**2 for a, b in pos):
            pos.append((x, y))
    for x, y in pos:
        f = rng.uniform(5e3, 5e4)
        ref += f / (2 * np.pi * 1.4**2) * np.exp(-((xs - x) ** 2 + (ys - y) ** 2) / (2 * 1.4**2))
        sg = 2.0 + 0.3 * x / w
        sci += f / (2 * np.pi * sg**2) * np.exp(-((xs - x) ** 2 + (ys - y) ** 2) / (2 * sg**2))
    var_r = (ref / 1.5 + 9.0).astype(np.float32)
    var_s = (sci / 1.5 + 9.0).astype(np.float32)
    ref = (ref + rng.normal(0, 1, (h, w)) * np.sqrt(var_r)).astype(np.float32)
    sci = (sci + rng.normal(0, 1, (h, w)) * np.sqrt(var_s)).astype(np.float32)
    sm = np.zeros((h, w), np.uint8)
    rm = np.zeros((h, w), np.uint8)
    rm[:, 57] = 1
    sm[30:34, 100] = 1
    sx = np.array([int(round(x)) for x, _ in pos], np.int32)
    sy = np.array([int(round(y)) for _, y in pos], np.int32)
    sx[0], sy[0] = 3, 5  # a stamp clipped by the frame edge
    return sci, ref, var_s, var_r, sm, rm, sx, sy


def _oracle_bconv(beta, n_max, r):
    if refbuild.available():
        return lambda patch: refbuild.basis_convolve(patch, beta, n_max, r)
    return lambda patch: nr.basis_convolve(patch, beta, n_max, r).astype(np.float32)


@pytest.mark.parametrize("cv_folds,stamped", [(0, False), (3, False), (3, True)])
def test_fit_kernel_matches_oracle(cv_folds, stamped, monkeypatch):
    sci, ref, vs, vr, sm, rm, sx, sy = _fit_frame()
    h, w = sci.shape
    knots = nr.grid_knots(0, 0, w - 1, h - 1, 3, 3)
    beta, n_max, sr = 1.2, 3, 7
    r = nr.default_radius(beta, n_max)
    monkeypatch.setenv("DELTA_STAMP_APPROX", "1" if stamped else "0")
    kw = dict(clip_sigma=3.0, clip_iterations=3, min_stamps=5, cv_folds=cv_folds, science_var=vs,
              reference_var=vr, science_mask=sm, reference_mask=rm)
    got = _core.fit_kernel(sci, ref, knots, sx, sy, sr, beta, n_max, GRID, **kw)
    want = nr.fit_kernel(sci, ref, knots, sx, sy, sr, beta, n_max, GRID, basis_convolve_fn=_oracle_bconv(beta, n_max, r),
                         **kw)
    for key in ("n_pixels", "n_stamps_total", "n_stamps_used", "n_stamps_rejected", "cv_exact_design_bytes"):
        assert got[key] == want[key], key
    assert got["lambda"] == want["lambda"]
    np.testing.assert_array_equal(got["stamp_x"], want["stamp_x"])
    np.testing.assert_array_equal(got["stamp_accepted"], want["stamp_accepted"])
    np.testing.assert_allclose(got["theta"], want["theta"], rtol=1e-6, atol=1e-8 * np.abs(want["theta"]).max())
    np.testing.assert_allclose(got["stamp_chi2"], want["stamp_chi2"], rtol=1e-6)
    np.testing.assert_allclose(got["reduced_chi2"], want["reduced_chi2"], rtol=1e-6)
    np.testing.assert_allclose(got["component_sums"], want["component_sums"], rtol=1e-12, atol=1e-14)


def test_fit_kernel_errors():
    sci, ref, vs, vr, sm, rm, sx, sy = _fit_frame(1)
    h, w = sci.shape
    knots = nr.grid_knots(0, 0, w - 1, h - 1, 3, 3)
    with pytest.raises(RuntimeError):
        _core.fit_kernel(sci, ref, knots, sx, sy[:-1], 7, 1.2, 2, GRID)
    with pytest.raises(RuntimeError):
        _core.fit_kernel(sci, ref, knots, np.array([-100], np.int32), np.array([-100], np.int32), 7, 1.2, 2, GRID)


def _singular_problem(seed=7, n=2500, nc=4, nk=3):
    """A design whose component 2 is zero at every row: M's block for it is
    exactly zero, so A = M + lambda P0 keeps that field's three affine
    directions singular at every lambda (the penalty leaves them free). The
    Cholesky fails on the device as in Eigen; the reference then solves by its
    pivoted LDLT (src/solve.cpp:177-181, :328-333 in CV)."""
    knots, pts, t, w, bn, _ = _problem(seed, n=n, nc=nc, nk=nk)
    bn = bn.copy()
    bn[:, 2] = 0.0
    return knots, pts, t, w, bn


def test_ldlt_fallback_matches_oracle_on_a_singular_system():
    knots, pts, t, w, bn = _singular_problem()
    want = nr.solve_gls_gcv(knots, pts, t, w, bn, GRID)
    got = _core.solve_gls_gcv(knots, pts, t, w, bn, GRID)
    assert got["used_ldlt"]
    assert got["lambda"] == want["lambda"]
    np.testing.assert_allclose(got["gcv_curve"], want["gcv_curve"], rtol=1e-6)
    np.testing.assert_allclose(got["theta"], want["theta"], rtol=1e-7, atol=1e-9)
    np.testing.assert_allclose(got["effective_dof"], want["effective_dof"], rtol=1e-8)
    np.testing.assert_allclose(got["rss"], want["rss"], rtol=1e-6)
    k = knots.shape[0]
    # the dead field's coefficients: its bending part is zeroed by the penalty,
    # its affine part by the pseudo-inverse of the zero pivots
    np.testing.assert_allclose(got["theta"][2 * k : 3 * k], 0.0, atol=1e-12)
    for lam in (1e-6, 1.0, 1e6):
        g = _core.solve_gls(knots, pts, t, w, bn, lam)
        s = nr.solve_gls(knots, pts, t, w, bn, lam)
        assert g["used_ldlt"]
        np.testing.assert_allclose(g["theta"], s["theta"], rtol=1e-7, atol=1e-9)
        np.testing.assert_allclose(g["effective_dof"], s["effective_dof"], rtol=1e-8)


def test_ldlt_fallback_in_cv_and_mixed_precision():
    knots, pts, t, w, bn = _singular_problem(8, n=2400)
    group = np.arange(t.size) % 4
    got = _core.solve_gls_cv(knots, pts, t, w, bn, GRID, group, 4)
    want = nr.solve_gls_cv(knots, pts, t, w, bn, GRID, group, 4)
    assert got["lambda"] == want["lambda"] and got["used_ldlt"]
    fin = np.isfinite(want["gcv_curve"])  # coarse-to-fine search: unvisited lambdas stay inf
    assert np.array_equal(np.isfinite(got["gcv_curve"]), fin)
    np.testing.assert_allclose(got["gcv_curve"][fin], want["gcv_curve"][fin], rtol=1e-6)
    np.testing.assert_allclose(got["theta"], want["theta"], rtol=1e-7, atol=1e-9)
    # Mixed precision has no Cholesky factor to refine with: it redoes the fit in FP64.
    mixed = _core.solve_gls_gcv(knots, pts, t, w, bn, GRID, precision="mixed")
    assert mixed["precision_used"] == "fp64" and mixed["used_ldlt"]
    fp64 = _core.solve_gls_gcv(knots, pts, t, w, bn, GRID)
    np.testing.assert_array_equal(mixed["theta"], fp64["theta"])
    # an ordinary SPD system never takes the fallback
    knots, pts, t, w, bn, _ = _problem()
    assert not _core.solve_gls_gcv(knots, pts, t, w, bn, GRID)["used_ldlt"]
