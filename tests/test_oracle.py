"""CPU pins of the oracle: against the reference-built library / golden
fixtures, and against the analytic known answers of the reference's own test
suite (tests/test_basis.py, test_convolve.py, test_subtract.py, test_noise.py,
test_catalog.py of tkillestein/delta)."""

from __future__ import annotations

import numpy as np
import pytest
from conftest import load_golden

from oracle import cref, refbuild
from oracle import numpy_ref as nr

# ---------------------------------------------------------------- basis / convolve


def test_basis_matches_reference_golden():
    g = load_golden("basis")
    for i in range(4):
        beta, n_max, r = g[f"params_{i}"]
        b = nr.gauss_hermite_basis1d(float(beta), int(n_max), int(r))
        np.testing.assert_allclose(b, g[f"basis1d_{i}"], rtol=0, atol=1e-15)
        # float32 taps (what the convolutions use) are bit-identical
        assert np.array_equal(b.astype(np.float32), g[f"basis1d_{i}"].astype(np.float32))


def test_basis_convolve_matches_reference_golden():
    g = load_golden("basis")
    beta, n_max, r = g["conv_params"]
    out = nr.basis_convolve(g["conv_image"], float(beta), int(n_max), int(r))
    np.testing.assert_allclose(out, g["conv_out"], rtol=1e-5, atol=2e-6)


def test_impulse_response_is_kernel():
    # reference tests/test_convolve.py:26-52: impulse -> 180-degree flipped kernel
    img = np.zeros((41, 41), np.float32)
    img[20, 20] = 1.0
    out = nr.basis_convolve(img, 2.0, 2, 6)
    orders = nr.basis_orders(2)
    b1d = nr.gauss_hermite_basis1d(2.0, 2, 6)
    for c in range(len(orders)):
        k = nr.kernel2d(b1d, orders, c)
        np.testing.assert_allclose(out[c, 14:27, 14:27], k, atol=1e-6)
        assert np.all(out[c, :14] == 0) and np.all(out[c, 27:] == 0)


# --------------------------------------------------------------------- thin plate


def test_tps_penalty_symmetric_psd_and_affine_unpenalised():
    knots = nr.grid_knots(0, 0, 300, 200, 4, 3)
    tp = nr.ThinPlate(knots)
    p = tp.penalty
    np.testing.assert_allclose(p, p.T, atol=1e-12)
    assert np.linalg.eigvalsh(p).min() > -1e-9
    assert np.all(p[-3:, :] == 0) and np.all(p[:, -3:] == 0)


def test_householder_null_space_is_orthonormal_complement():
    knots = nr.grid_knots(0, 0, 1023, 1023, 5, 5)
    tp = nr.ThinPlate(knots)
    t = np.column_stack([np.ones(25), tp.kn])
    np.testing.assert_allclose(t.T @ tp.z, 0, atol=1e-13)
    np.testing.assert_allclose(tp.z.T @ tp.z, np.eye(22), atol=1e-13)


# --------------------------------------------------------------------- subtract


def test_c_oracle_matches_fp64_oracle():
    rng = np.random.default_rng(1)
    h, w = 200, 230
    sci = (100 + 5 * rng.standard_normal((h, w))).astype(np.float32)
    ref = (100 + 5 * rng.standard_normal((h, w))).astype(np.float32)
    knots = nr.grid_knots(0, 0, w - 1, h - 1, 3, 3)
    nc = 10
    theta = 0.1 * rng.standard_normal((nc + 1) * 9)
    vs = rng.uniform(1, 2, (h, w)).astype(np.float32)
    vr = rng.uniform(1, 2, (h, w)).astype(np.float32)
    sm = np.zeros((h, w), np.uint8)
    sm[50, 60] = 1
    rm = np.zeros((h, w), np.uint8)
    rm[100, 100] = 4
    a = nr.subtract(sci, ref, knots, theta, 1.5, 3, 0, 140.0, vs, vr, sm, rm)
    b = cref.subtract(sci, ref, knots, theta, 1.5, 3, 0, 140.0, vs, vr, sm, rm)
    np.testing.assert_allclose(b["difference"], a["difference"], atol=2e-4 * np.abs(a["difference"]).max())
    np.testing.assert_allclose(b["variance"], a["variance"], rtol=1e-5)
    assert np.array_equal(a["mask"], b["mask"])


def test_variance_constant_kernel_known_answer():
    # reference tests/test_subtract.py:128-154
    h = w = 50
    rng = np.random.default_rng(2)
    ref = rng.standard_normal((h, w)).astype(np.float32)
    sci = rng.standard_normal((h, w)).astype(np.float32)
    var_r = rng.uniform(0.5, 2.0, (h, w)).astype(np.float32)
    var_s = rng.uniform(0.5, 2.0, (h, w)).astype(np.float32)
    knots = nr.grid_knots(0.0, 0.0, w - 1.0, h - 1.0, 3, 3)
    k = knots.shape[0]
    theta = np.zeros(2 * k)
    theta[k - 3] = 1.3
    res = cref.subtract(sci, ref, knots, theta, 2.0, 0, science_var=var_s, reference_var=var_r)
    b1d = nr.gauss_hermite_basis1d(2.0, 0, nr.default_radius(2.0, 0))
    phi0 = nr.kernel2d(b1d, nr.basis_orders(0), 0).astype(np.float64)
    kf = (phi0**2)[::-1, ::-1]
    r = phi0.shape[0] // 2
    pad = np.zeros((h + 2 * r, w + 2 * r))
    pad[r : r + h, r : r + w] = var_r
    conv = sum(kf[i, j] * pad[i : i + h, j : j + w] for i in range(2 * r + 1) for j in range(2 * r + 1))
    np.testing.assert_allclose(res["variance"], var_s + 1.3**2 * conv, rtol=1e-3, atol=1e-3)


def test_mask_growth_box_and_edge_known_answer():
    # reference tests/test_subtract.py:173-215
    h = w = 41
    rng = np.random.default_rng(4)
    ref = rng.standard_normal((h, w)).astype(np.float32)
    sci = rng.standard_normal((h, w)).astype(np.float32)
    knots = nr.grid_knots(0.0, 0.0, w - 1.0, h - 1.0, 3, 3)
    theta = np.zeros(4 * 9)
    rm = np.zeros((h, w), np.uint8)
    rm[20, 20] = 1
    sm = np.zeros((h, w), np.uint8)
    sm[10, 30] = 1
    for impl in (nr, cref):
        mask = impl.subtract(sci, ref, knots, theta, 2.0, 1, science_mask=sm, reference_mask=rm)["mask"]
        r = nr.default_radius(2.0, 1)
        assert (mask[20 - r : 20 + r + 1, 20 - r : 20 + r + 1] & 1).all()
        assert mask[10, 30] & 1
        assert (mask[0, :] & 16).all() and (mask[:, 0] & 16).all()
        assert (mask[r:-r, r:-r] & 16 == 0).all()


# ---------------------------------------------------------------- matched filter


def test_matched_filter_peak_snr_known_answer():
    # reference tests/test_noise.py:163-181: peak S/N = amp sqrt(sum psf^2 / var), argmax exact
    h = w = 64
    sig = 1.5
    r = 6
    yy, xx = np.mgrid[-r : r + 1, -r : r + 1]
    psf = np.exp(-(xx**2 + yy**2) / (2 * sig**2))
    psf = (psf / psf.sum()).astype(np.float32)
    img = np.zeros((h, w), np.float32)
    amp = 50.0
    img[30 - r : 30 + r + 1, 25 - r : 25 + r + 1] = amp * psf
    var = np.full((h, w), 4.0, np.float32)
    for impl in (nr, cref):
        score = impl.matched_filter(img, psf, var)
        iy, ix = np.unravel_index(np.argmax(score), score.shape)
        assert (iy, ix) == (30, 25)
        expect = amp * np.sqrt(float(np.sum(psf.astype(np.float64) ** 2)) / 4.0)
        assert abs(score[iy, ix] - expect) / expect < 1e-3


# ------------------------------------------------------------------------ catalog


@pytest.mark.parametrize("i", [0, 1, 2])
def test_label_numbering_matches_reference_golden(i):
    g = load_golden("catalog")
    score = g[f"score_{i}"]
    mask = g.get(f"mask_{i}")
    seed = nr.seed_mask(score, 5.0, +1, mask, True)
    labels, n = nr.label_components(seed)
    assert n == g[f"labels_{i}"].max()
    assert np.array_equal(labels, g[f"labels_{i}"])


def test_refbuild_label_numbering_is_raster_first():
    if not refbuild.available():
        pytest.skip("reference library not built")
    rng = np.random.default_rng(9)
    seed = (rng.random((300, 257)) < 0.3).astype(np.uint8)
    a, na = refbuild.label_components(seed)
    b, nb = nr.label_components(seed.astype(bool))
    assert na == nb and np.array_equal(a, b)


def test_reference_catalog_known_answers():
    # reference tests/test_catalog.py:75-86,142-152
    if not refbuild.available():
        pytest.skip("reference library not built")
    s = np.zeros((60, 60), np.float32)
    s[20:35, 20:35] = 6.0
    cat = refbuild.build_catalog(s, s, expected_fwhm=2.0)
    assert len(cat["x"]) == 1 and cat["n_pix"][0] == 225
    s = np.zeros((40, 40), np.float32)
    s[18:23, 18:23] = 8.0
    m = np.zeros((40, 40), np.uint8)
    m[18:23, 20] = 1
    cat = refbuild.build_catalog(s, s, mask=m, expected_fwhm=3.0)
    assert len(cat["x"]) == 2 and np.all(cat["mask_flags"] != 0)


def _gls_problem(seed, n=4000, nc=6, knots_side=3, rank_deficient=False):
    rng = np.random.default_rng(seed)
    knots = nr.grid_knots(0, 0, 500, 400, knots_side, knots_side)
    tp = nr.ThinPlate(knots)
    pts = np.column_stack([rng.uniform(0, 500, n), rng.uniform(0, 400, n)])
    des = tp.design(pts)
    bn = rng.normal(size=(n, nc))
    if rank_deficient:
        bn[:, 3] = bn[:, 1]  # two identical components: M is singular at lambda = 0
    target = bn @ rng.normal(size=nc) + 0.1 * rng.normal(size=n)
    weights = rng.uniform(0.5, 2.0, n)
    return des, target, weights, bn, tp.penalty


def test_c_gls_assembly_and_grid_match_numpy_oracle():
    """The C restatement of the GLS assembly and lambda-grid solve (the timed
    CPU chain's fit) equals the NumPy FP64 oracle (src/solve.cpp:70-262)."""
    if not cref.available():
        pytest.skip("oracle C library not built")
    des, t, w, bn, pen = _gls_problem(0)
    s = nr.System(des, t, w, bn, pen)
    m, rhs, ywy = cref.assemble(des, t, w, bn)
    np.testing.assert_allclose(m, s.m, rtol=1e-12, atol=1e-12 * np.abs(s.m).max())
    np.testing.assert_allclose(rhs, s.rhs, rtol=1e-12, atol=1e-12 * np.abs(s.rhs).max())
    assert ywy == pytest.approx(s.ywy, rel=1e-13)
    grid = np.logspace(-6, 6, 13)
    want = nr.solve_gls_gcv_system(s, grid)
    got = cref.gls_gcv(des, t, w, bn, pen, grid)
    assert got["lambda"] == want["lambda"]
    np.testing.assert_allclose(got["gcv_curve"], want["gcv_curve"], rtol=1e-9)
    np.testing.assert_allclose(got["theta"], want["theta"], rtol=1e-8, atol=1e-10)


def test_ldlt_fallback_on_a_rank_deficient_system():
    """A design with two identical components is singular: the Cholesky fails
    and the reference falls back to Eigen's pivoted LDLT (src/solve.cpp:177-181).
    Both restatements take that path, agree on the fit, give a minimum of the
    weighted residual, and report edf = tr(A^+ M) = rank at lambda = 0."""
    if not cref.available():
        pytest.skip("oracle C library not built")
    des, t, w, bn, pen = _gls_problem(1, rank_deficient=True)
    s = nr.System(des, t, w, bn, pen)
    with pytest.raises(np.linalg.LinAlgError):
        np.linalg.cholesky(s.m)
    got = cref.solve_grid(s, [0.0, 1.0])
    # the penalty leaves each field's affine part free, so the duplicate stays singular at any lambda
    assert got[0]["used_ldlt"] and got[1]["used_ldlt"]
    want = nr.solve_at(s, 0.0)
    # theta is not unique along M's null space (any LDLT's choice there rests on
    # rounding), so the fitted quantities are compared: M theta, rss and edf.
    np.testing.assert_allclose(s.m @ got[0]["theta"], s.m @ want["theta"], rtol=1e-7,
                               atol=1e-9 * np.abs(s.rhs).max())
    assert got[0]["rss"] == pytest.approx(want["rss"], rel=1e-8)
    assert got[0]["effective_dof"] == pytest.approx(want["effective_dof"], abs=1e-6)
    assert round(want["effective_dof"]) == np.linalg.matrix_rank(s.m)
    # normal equations hold: M theta = rhs (rhs lies in the range of M)
    np.testing.assert_allclose(s.m @ want["theta"], s.rhs, rtol=1e-7, atol=1e-7 * np.abs(s.rhs).max())
    # on an SPD matrix the LDLT solve is the ordinary solve
    a = s.m + np.eye(s.p)
    fac, perm = nr.ldlt_factor(a)
    np.testing.assert_allclose(nr.ldlt_solve(fac, perm, s.rhs), np.linalg.solve(a, s.rhs), rtol=1e-9)
    np.testing.assert_allclose(cref.ldlt_solve(a, s.rhs), np.linalg.solve(a, s.rhs), rtol=1e-9)
