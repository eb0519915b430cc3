"""The FP64 gradient oracle (oracle/grad_ref.py) against central finite
differences of its own FP64 forward -- host only. The reference has no
gradient code, so this is what pins the adjoint the device kernels are then
compared with."""

from __future__ import annotations

import numpy as np
import pytest

from delta_b200 import validation
from oracle import grad_ref
from oracle import numpy_ref as nr


def _model(size=(72, 88), n_max=2, knots_side=3, seed=0):
    h, w = size
    p = validation.synthetic_pair(w, h, 40, seed, mask_fraction=0.02)
    wt = np.where(p.science_mask == 0, 1.0 / (p.science_var + p.reference_var), 0.0).astype(np.float32)
    knots = nr.grid_knots(0, 0, w - 1, h - 1, knots_side, knots_side)
    m = grad_ref.KernelModel(p.science, p.reference, wt, knots, 1.4, n_max, reference_mask=p.reference_mask)
    rng = np.random.default_rng(seed + 1)
    theta = 0.05 * rng.standard_normal(m.nf * m.k)
    theta[0 : m.k] += 1.0  # mostly the first component, a unit kernel
    return m, theta


def test_shifted_basis_at_zero_is_the_basis_and_derivative_is_the_slope():
    g, dg = grad_ref.shifted_basis1d(1.7, 5, 6, 0.0)
    np.testing.assert_allclose(g, nr.gauss_hermite_basis1d(1.7, 5, 6), rtol=1e-13, atol=1e-16)
    h = 1e-6
    gp, _ = grad_ref.shifted_basis1d(1.7, 5, 6, 0.3 + h)
    gm, _ = grad_ref.shifted_basis1d(1.7, 5, 6, 0.3 - h)
    _, d3 = grad_ref.shifted_basis1d(1.7, 5, 6, 0.3)
    # d/dd g(u - d) = -g'(u - d)
    np.testing.assert_allclose((gp - gm) / (2 * h), -d3, rtol=1e-6, atol=1e-9)


@pytest.mark.parametrize("size,knots_side", [((72, 88), 3), ((300, 280), 4)])
def test_oracle_gradient_matches_central_differences(size, knots_side):
    m, theta = _model(size, knots_side=knots_side)
    dx, dy, s = 0.21, -0.33, 1.07
    g = m.grad(theta, dx, dy, s, reference=True)
    h = 1e-3
    fd = lambda f: (f(+h) - f(-h)) / (2 * h)  # noqa: E731
    assert fd(lambda e: m.chi2(theta, dx + e, dy, s)) == pytest.approx(g["grad_shift"][0], rel=1e-5)
    assert fd(lambda e: m.chi2(theta, dx, dy + e, s)) == pytest.approx(g["grad_shift"][1], rel=1e-5)
    assert fd(lambda e: m.chi2(theta, dx, dy, s + e)) == pytest.approx(g["grad_scale"], rel=1e-6)
    for i in (0, m.k + 2, (m.nf - 1) * m.k + 1):
        e_i = np.zeros_like(theta)
        e_i[i] = 1.0
        got = fd(lambda e: m.chi2(theta + e * e_i, dx, dy, s))
        assert got == pytest.approx(g["grad_theta"][i], rel=1e-6, abs=1e-6 * np.abs(g["grad_theta"]).max())
    # reference adjoint: directional derivative along a random perturbation of the used pixels
    rng = np.random.default_rng(5)
    v = np.where(m.replaced, 0.0, rng.standard_normal((m.h, m.w)))
    base = m.rs.copy()

    def chi_r(e):
        m.rs = base + e * v
        try:
            return m.chi2(theta, dx, dy, s)
        finally:
            m.rs = base

    assert fd(chi_r) == pytest.approx(float(np.sum(g["grad_reference"] * v)), rel=1e-6)


def test_stamp_gcv_adjoint_matches_central_differences():
    """The normal-equation-map adjoint of the FP64 oracle against central
    differences (h = 1e-3) of its own GCV / RSS."""
    p = validation.synthetic_pair(180, 160, 50, 4, mask_fraction=0.01)
    from oracle import refbuild

    if refbuild.available():
        sel = refbuild.select_stamps(p.science, p.reference, p.science_mask, p.reference_mask, stamp_radius=8,
                                     saturation=p.saturation, max_stamps=12)
        sx, sy = sel["x"], sel["y"]
    else:
        sx, sy = np.array([40, 90, 130, 60, 120]), np.array([40, 60, 110, 120, 30])
    knots = nr.grid_knots(0, 0, 179, 159, 3, 3)
    m = grad_ref.StampGCV(p.science, p.reference, p.science_var, p.reference_var, p.science_mask, p.reference_mask,
                          knots, sx, sy, 8, 1.5, 2)
    x0 = np.array([np.log(0.3), 0.17, -0.22, 1.05])
    g = m.grad(*x0)
    v = m.value(*x0)
    assert g["gcv"] == pytest.approx(v["gcv"], rel=1e-9)
    assert g["rss"] == pytest.approx(v["rss"], rel=1e-9)
    h = 1e-3
    for i in range(4):
        e = np.zeros(4)
        e[i] = h
        vp, vm = m.value(*(x0 + e)), m.value(*(x0 - e))
        fd_gcv = (vp["gcv_direct"] - vm["gcv_direct"]) / (2 * h)
        fd_rss = (vp["rss_direct"] - vm["rss_direct"]) / (2 * h)
        assert fd_gcv == pytest.approx(g["grad_gcv"][i], rel=1e-5, abs=1e-11), i
        assert fd_rss == pytest.approx(g["grad_rss"][i], rel=1e-5, abs=1e-9), i
