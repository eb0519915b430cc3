"""GPU parity of the frame kernels through the C ABI (``delta_b200._core``):
basis convolution, subtraction (difference / variance / mask), photometric
scale, matched filter and the connected-component catalog, against the
reference-built library (oracle/_ref), the C restatement with the reference's
float32 semantics (oracle/csrc) and the FP64 NumPy restatement."""

from __future__ import annotations

import numpy as np
import pytest
from conftest import load_golden

from delta_b200 import _core, validation
from oracle import cref, refbuild
from oracle import numpy_ref as nr

pytestmark = pytest.mark.gpu

# Difference / score tolerance: max |delta| <= 1e-3 of the local noise sigma
# (the drop-in bar); against the float32-semantics C restatement the kernels
# are expected to be bit-identical except where an FP64 lattice value rounds
# to a neighbouring float.
SIGMA_TOL = 1e-3


def _frame(rng, h, w, sky=100.0, noise=5.0, n_src=20):
    img = sky + noise * rng.standard_normal((h, w))
    ys, xs = np.mgrid[0:h, 0:w]
    for _ in range(n_src):
        x, y = rng.uniform(0, w), rng.uniform(0, h)
        img += rng.uniform(1e3, 5e4) / (2 * np.pi * 2.0**2) * np.exp(-((xs - x) ** 2 + (ys - y) ** 2) / 8.0)
    return img.astype(np.float32)


# ------------------------------------------------------------------ basis convolve


@pytest.mark.parametrize("shape,beta,n_max,r", [((24, 31), 1.5, 2, 5), ((70, 131), 1.1, 6, 8),
                                                ((128, 64), 2.0, 4, 10), ((5, 3), 0.8, 0, 3)])
def test_basis_convolve_bit_exact_vs_reference(shape, beta, n_max, r):
    rng = np.random.default_rng(0)
    img = rng.standard_normal(shape).astype(np.float32)
    got = _core.basis_convolve(img, beta, n_max, r)
    if refbuild.available():
        want = refbuild.basis_convolve(img, beta, n_max, r)
        assert np.array_equal(got, want), np.abs(got - want).max()
    want64 = nr.basis_convolve(img, beta, n_max, r)
    np.testing.assert_allclose(got, want64, atol=1e-5 * max(1.0, np.abs(want64).max()))


def test_basis_convolve_golden():
    g = load_golden("basis")
    beta, n_max, r = g["conv_params"]
    got = _core.basis_convolve(g["conv_image"], float(beta), int(n_max), int(r))
    assert np.array_equal(got, g["conv_out"])


# ------------------------------------------------------------------------ subtract


def _theta(rng, nc, k, amp0=1.0):
    th = 0.05 * rng.standard_normal((nc + 1) * k)
    th[k - 3] = amp0  # intercept of the c_0 field
    return th


CASES = [
    # (h, w, n_knots, beta, n_max, radius) -- exact-field and coarse-lattice paths,
    # ragged tile edges, single-component basis, large radius.
    (40, 48, 3, 2.0, 2, 0),
    (64, 64, 3, 1.2, 0, 4),
    (300, 280, 3, 1.5, 3, 0),
    (517, 389, 3, 1.0, 4, 10),
    (1024, 1024, 3, 0.95, 6, 8),
    (333, 1500, 4, 1.7, 5, 7),
]


@pytest.mark.parametrize("h,w,nk,beta,n_max,radius", CASES)
def test_subtract_parity(h, w, nk, beta, n_max, radius):
    rng = np.random.default_rng(h * 31 + w)
    sci = _frame(rng, h, w)
    ref = _frame(rng, h, w)
    knots = nr.grid_knots(0, 0, w - 1, h - 1, nk, nk)
    nc = (n_max + 1) * (n_max + 2) // 2
    theta = _theta(rng, nc, knots.shape[0])
    vs = (np.abs(sci) / 1.5 + 4.0).astype(np.float32)
    vr = (np.abs(ref) / 1.5 + 4.0).astype(np.float32)
    sm = np.zeros((h, w), np.uint8)
    rm = np.zeros((h, w), np.uint8)
    sm[rng.integers(0, h, 5), rng.integers(0, w, 5)] = 1
    rm[:, rng.integers(0, w)] = 1
    rm[rng.integers(0, h, 5), rng.integers(0, w, 5)] = 4
    ref[rng.integers(0, h), rng.integers(0, w)] = np.nan
    sat = float(np.percentile(sci, 99.9))
    got = _core.subtract(sci, ref, knots, theta, beta, n_max, radius, sat, vs, vr, sm, rm)
    c = cref.subtract(sci, ref, knots, theta, beta, n_max, radius, sat, vs, vr, sm, rm)
    f64 = nr.subtract(sci, ref, knots, theta, beta, n_max, radius, sat, vs, vr, sm, rm)
    # masks: bit-exact
    assert np.array_equal(got["mask"], c["mask"])
    assert np.array_equal(got["mask"], f64["mask"])
    sigma = np.sqrt(np.maximum(got["variance"], 1e-6))
    good = got["mask"] == 0
    d = got["difference"].astype(np.float64)
    # vs the float32-semantics restatement: (nearly) bit-identical
    dc = np.abs(d - c["difference"])
    assert np.max(dc[good] / sigma[good]) <= SIGMA_TOL
    assert np.mean(dc == 0) > 0.99
    # vs FP64: the drop-in tolerance wherever a noise level exists (masked
    # pixels keep their real values); filled pixels carry the same fill value.
    pos = got["variance"] > 0
    assert np.max(np.abs(d - f64["difference"])[pos] / sigma[pos]) <= SIGMA_TOL
    filled = ~pos
    np.testing.assert_allclose(d[filled], f64["difference"][filled], rtol=1e-5, atol=1e-4)
    # variance: same float arithmetic as the reference
    np.testing.assert_allclose(got["variance"], c["variance"], rtol=2e-6, atol=1e-6)
    np.testing.assert_allclose(got["variance"], f64["variance"], rtol=1e-4, atol=1e-4)


def test_subtract_layers_optional_and_self_subtraction():
    # reference tests/test_subtract.py:88-125
    h, w = 40, 40
    rng = np.random.default_rng(1)
    ref = (5.0 + rng.standard_normal((h, w))).astype(np.float32)
    knots = nr.grid_knots(0.0, 0.0, w - 1.0, h - 1.0, 3, 3)
    bn = _core.basis_convolve(ref, 1.8, 2)
    nc = bn.shape[0]
    theta = 0.05 * rng.standard_normal((nc + 1) * 9)
    fields = nr.Fields(knots, theta, nc, w, h)
    model = fields.field_full(nc).astype(np.float64)
    for n in range(nc):
        model += fields.field_full(n) * bn[n]
    res = _core.subtract(model.astype(np.float32), ref, knots, theta, 1.8, 2)
    assert res["variance"] is None and res["mask"] is None
    np.testing.assert_allclose(res["difference"], 0.0, atol=1e-3)


def test_subtract_science_variance_passthrough():
    h = w = 30
    rng = np.random.default_rng(3)
    ref = rng.standard_normal((h, w)).astype(np.float32)
    sci = rng.standard_normal((h, w)).astype(np.float32)
    var_s = rng.uniform(0.5, 2.0, (h, w)).astype(np.float32)
    knots = nr.grid_knots(0.0, 0.0, w - 1.0, h - 1.0, 3, 3)
    theta = np.zeros(4 * 9)
    res = _core.subtract(sci, ref, knots, theta, 1.5, 1, science_var=var_s)
    np.testing.assert_array_equal(res["variance"], var_s)


def test_subtract_rejects_bad_shapes():
    a = np.zeros((20, 20), np.float32)
    knots = nr.grid_knots(0, 0, 19, 19, 3, 3)
    with pytest.raises(RuntimeError):
        _core.subtract(a, np.zeros((20, 21), np.float32), knots, np.zeros(36), 1.5, 1)
    with pytest.raises(RuntimeError):
        _core.subtract(a, a, knots, np.zeros(35), 1.5, 1)


def test_subtract_all_masked_reference_fills_zero():
    h = w = 48
    rng = np.random.default_rng(5)
    sci = rng.standard_normal((h, w)).astype(np.float32)
    ref = rng.standard_normal((h, w)).astype(np.float32)
    rm = np.ones((h, w), np.uint8)
    knots = nr.grid_knots(0, 0, w - 1, h - 1, 3, 3)
    theta = _theta(rng, 3, 9)
    got = _core.subtract(sci, ref, knots, theta, 1.5, 1, reference_mask=rm)
    c = cref.subtract(sci, ref, knots, theta, 1.5, 1, reference_mask=rm)
    assert np.array_equal(got["mask"], c["mask"])
    np.testing.assert_allclose(got["difference"], c["difference"], atol=1e-5)


def test_photometric_scale_parity():
    h, w = 400, 400
    rng = np.random.default_rng(7)
    knots = nr.grid_knots(0.0, 0.0, w - 1.0, h - 1.0, 3, 3)
    theta = 0.1 * rng.standard_normal(7 * 9)
    sums = rng.standard_normal(6)
    got = _core.photometric_scale(knots, theta, sums, h, w)
    want = nr.photometric_scale(knots, theta, sums, h, w)
    np.testing.assert_allclose(got, want, rtol=1e-5, atol=1e-5)
    exact = _core.photometric_scale_at(knots, theta, sums, np.column_stack(
        [np.tile(np.arange(w), h), np.repeat(np.arange(h), w)]).astype(float)).reshape(h, w)
    err = np.max(np.abs(got - exact))
    assert 0 < err < 5e-3 * np.ptp(exact)


# ------------------------------------------------------------------ matched filter


@pytest.mark.parametrize("h,w,ps", [(64, 64, 13), (257, 190, 17), (1024, 1024, 17), (100, 80, 23), (31, 29, 5)])
def test_matched_filter_bit_exact(h, w, ps):
    rng = np.random.default_rng(h + ps)
    img = rng.standard_normal((h, w)).astype(np.float32) * 10
    var = rng.uniform(0.5, 3.0, (h, w)).astype(np.float32)
    var[rng.integers(0, h, 10), rng.integers(0, w, 10)] = 0.0
    r = ps // 2
    yy, xx = np.mgrid[-r : r + 1, -r : r + 1]
    psf = np.exp(-(xx**2 + yy**2) / (2 * 1.7**2))
    psf = np.clip(psf / psf.sum() - 1e-4, 0, None).astype(np.float32)  # exact zero wings
    got = _core.matched_filter(img, psf, var)
    want = cref.matched_filter(img, psf, var)
    assert np.array_equal(got, want), np.abs(got - want).max()
    np.testing.assert_allclose(got, nr.matched_filter(img, psf, var), atol=1e-4)


@pytest.mark.parametrize("ps", [17, 23])
def test_matched_filter_non_finite_tiles_bit_exact(ps):
    """Tiles holding NaN / Inf keep the reference's zero-tap skip (a zero tap
    never touches a non-finite pixel); all other tiles take the fast path."""
    h, w = 300, 270
    rng = np.random.default_rng(ps)
    img = rng.standard_normal((h, w)).astype(np.float32) * 10
    img[rng.integers(0, h, 25), rng.integers(0, w, 25)] = np.nan
    img[rng.integers(0, h, 5), rng.integers(0, w, 5)] = np.inf
    var = rng.uniform(0.5, 3.0, (h, w)).astype(np.float32)
    r = ps // 2
    yy, xx = np.mgrid[-r : r + 1, -r : r + 1]
    psf = np.exp(-(xx**2 + yy**2) / (2 * 1.7**2))
    psf = np.clip(psf / psf.sum() - 1e-4, 0, None).astype(np.float32)
    got = _core.matched_filter(img, psf, var)
    want = cref.matched_filter(img, psf, var)
    assert np.array_equal(got, want, equal_nan=True)
    assert np.isnan(got).any() and np.isfinite(got).any()


def test_matched_filter_peak_known_answer():
    h = w = 64
    r = 6
    yy, xx = np.mgrid[-r : r + 1, -r : r + 1]
    psf = np.exp(-(xx**2 + yy**2) / (2 * 1.5**2))
    psf = (psf / psf.sum()).astype(np.float32)
    img = np.zeros((h, w), np.float32)
    img[30 - r : 30 + r + 1, 25 - r : 25 + r + 1] = 50.0 * psf
    score = _core.matched_filter(img, psf, np.full((h, w), 4.0, np.float32))
    iy, ix = np.unravel_index(np.argmax(score), score.shape)
    assert (iy, ix) == (30, 25)
    expect = 50.0 * np.sqrt(float(np.sum(psf.astype(np.float64) ** 2)) / 4.0)
    assert abs(score[iy, ix] - expect) / expect < 1e-3


# -------------------------------------------------------------------------- catalog

INT_COLS = ["peak_x", "peak_y", "n_pix", "fwhm_consistent", "mask_flags", "is_dipole", "quality",
            "psf_chi2_dof", "shape_consistent", "near_bright_star"]
FLOAT_COLS = ["x", "y", "peak_snr", "flux", "expected_n_pix", "fwhm_ratio", "psf_chi2", "psf_amplitude",
              "psf_amplitude_err", "bright_star_dist"]


def _assert_catalog_equal(got, want):
    n = len(want["x"])
    assert len(got["x"]) == n
    for k in INT_COLS:
        assert np.array_equal(np.asarray(got[k]).astype(np.int64), np.asarray(want[k]).astype(np.int64)), k
    for k in FLOAT_COLS:
        np.testing.assert_allclose(got[k], want[k], rtol=1e-12, atol=1e-12, err_msg=k)


@pytest.mark.parametrize("i", [0, 1, 2])
@pytest.mark.parametrize("pol", [0, 1])
def test_catalog_matches_reference_golden(i, pol):
    g = load_golden("catalog")
    mask = g.get(f"mask_{i}")
    got = _core.build_catalog(g[f"score_{i}"], g[f"diff_{i}"], mask=mask, expected_fwhm=3.0,
                              return_negative=bool(pol))
    want = {k.split("_", 2)[2]: v for k, v in g.items() if k.startswith(f"cat{pol}_{i}_")}
    _assert_catalog_equal(got, want)
    if pol == 0:
        labels = _core.catalog_labels(g[f"score_{i}"].shape)
        assert np.array_equal(labels, g[f"labels_{i}"])


@pytest.mark.parametrize("seed,h,w,density", [(0, 300, 257, 0.3), (1, 1024, 1024, 0.05), (2, 64, 2000, 0.5),
                                              (3, 1, 500, 0.6), (4, 500, 1, 0.6)])
def test_labels_bit_exact_vs_reference(seed, h, w, density):
    if not refbuild.available():
        pytest.skip("reference library not built")
    rng = np.random.default_rng(seed)
    score = np.where(rng.random((h, w)) < density, 9.0, 0.0).astype(np.float32)
    _core.build_catalog(score, score, expected_fwhm=3.0)
    labels = _core.catalog_labels((h, w))
    want, n = refbuild.label_components((score >= 5).astype(np.uint8))
    assert labels.max() == n
    assert np.array_equal(labels, want)


def test_catalog_enrichment_matches_reference():
    if not refbuild.available():
        pytest.skip("reference library not built")
    rng = np.random.default_rng(8)
    h = w = 200
    score = rng.normal(0, 1, (h, w)).astype(np.float32)
    ys, xs = np.mgrid[0:h, 0:w]
    for x, y in [(40, 40), (120, 60), (70, 150), (180, 180)]:
        score += (12 * np.exp(-((xs - x) ** 2 + (ys - y) ** 2) / 6.0)).astype(np.float32)
    diff = score * 3.0
    var = np.full((h, w), 9.0, np.float32)
    r = 5
    yy, xx = np.mgrid[-r : r + 1, -r : r + 1]
    psf = np.exp(-(xx**2 + yy**2) / 6.0)
    psf = (psf / psf.sum()).astype(np.float32)
    bx = np.array([45.0, 10.0, 175.0])
    by = np.array([38.0, 190.0, 185.0])
    kw = dict(expected_fwhm=3.0, fit_psf_shape=True, variance=var, psf=psf, bright_x=bx, bright_y=by)
    got = _core.build_catalog(score, diff, **kw)
    want = refbuild.build_catalog(score, diff, **kw)
    _assert_catalog_equal(got, want)


def test_catalog_empty_and_all_seeded():
    z = np.zeros((50, 40), np.float32)
    got = _core.build_catalog(z, z)
    assert len(got["x"]) == 0
    o = np.full((50, 40), 7.0, np.float32)
    got = _core.build_catalog(o, o, expected_fwhm=3.0)
    assert len(got["x"]) == 1 and got["n_pix"][0] == 2000


def test_model_convolve_tile_heights_give_identical_bits_and_autotune_records():
    """Every tile height the autotuner may pick gives the same difference,
    variance and mask bits (the per-pixel order of each sum does not depend on
    the tiling), and the tuner records its timed choice."""
    import ctypes
    import os

    from delta_b200 import _lib

    p = validation.synthetic_pair(700, 530, 200, 8, mask_fraction=0.01)
    knots = nr.grid_knots(0, 0, 699, 529, 3, 3)
    theta = np.zeros(22 * 9)
    theta[0:9] = 1.0
    args = (p.science, p.reference, knots, theta, 1.3, 5, 0, p.saturation, p.science_var, p.reference_var,
            p.science_mask, p.reference_mask)
    outs = []
    try:
        for th in ("16", "32", "64"):
            os.environ["DELTA_MODEL_CONVOLVE_TH"] = th
            outs.append(_core.subtract(*args))
    finally:
        os.environ.pop("DELTA_MODEL_CONVOLVE_TH", None)
    for o in outs[1:]:
        for name in ("difference", "variance", "mask"):
            np.testing.assert_array_equal(o[name], outs[0][name], err_msg=name)
    tuned = _core.subtract(*args)
    np.testing.assert_array_equal(tuned["difference"], outs[0]["difference"])
    need = ctypes.c_size_t()
    buf = ctypes.create_string_buffer(4096)
    _lib.check(_lib.lib().dgpu_autotune_table(buf, ctypes.c_size_t(4096), ctypes.byref(need)))
    table = buf.value.decode()
    assert "model_convolve/fast/nx6" in table and "ms" in table, table


@pytest.mark.parametrize("n_max,radius,beta", [(2, 0, 2.0), (3, 0, 1.5), (4, 10, 1.0), (5, 7, 1.7), (6, 11, 1.36),
                                               (6, 16, 2.0), (6, 14, 1.8), (4, 4, 0.8)])
def test_model_convolve_fast_kernel_equals_generic(n_max, radius, beta):
    """The compile-time-shaped model convolve (common n_max and tap counts,
    taps zero padded to a multiple of 8, packed field blend) gives the generic
    tile kernel's bits on a frame with masked, non-finite and off-frame
    reference pixels, on the coarse-lattice and the exact-field paths."""
    import os

    for (h, w, nk) in ((530, 700, 3), (90, 75, 3)):
        rng = np.random.default_rng(n_max * 100 + radius)
        p = validation.synthetic_pair(w, h, 120, n_max, mask_fraction=0.01)
        ref = p.reference.copy()
        ref[rng.integers(0, h, 6), rng.integers(0, w, 6)] = np.nan
        ref[rng.integers(0, h, 3), rng.integers(0, w, 3)] = -np.inf
        knots = nr.grid_knots(0, 0, w - 1, h - 1, nk, nk)
        nc = (n_max + 1) * (n_max + 2) // 2
        theta = _theta(rng, nc, knots.shape[0])
        args = (p.science, ref, knots, theta, beta, n_max, radius, p.saturation, p.science_var, p.reference_var,
                p.science_mask, p.reference_mask)
        fast = _core.subtract(*args)
        try:
            os.environ["DELTA_MODEL_CONVOLVE_GENERIC"] = "1"
            generic = _core.subtract(*args)
        finally:
            os.environ.pop("DELTA_MODEL_CONVOLVE_GENERIC", None)
        for name in ("difference", "variance", "mask"):
            assert np.array_equal(fast[name].view(np.uint32) if name != "mask" else fast[name],
                                  generic[name].view(np.uint32) if name != "mask" else generic[name]), (name, h, w)


@pytest.mark.parametrize("n,seed", [(1, 0), (2, 1), (1001, 2), (1000, 3), (4_000_000, 4)])
def test_z2_median_equals_numpy(n, seed):
    """dgpu_z2_median: numpy's median of the FP64 z^2 = D^2 / Var over the good
    pixels (Var > 0, both finite, mask 0), odd and even counts."""
    import ctypes

    from delta_b200 import _lib

    rng = np.random.default_rng(seed)
    d = rng.normal(0, 3, n).astype(np.float32)
    v = rng.uniform(0.5, 20, n).astype(np.float32)
    m = (rng.random(n) < 0.05).astype(np.uint8)
    if n > 10:
        d[rng.random(n) < 0.01] = np.nan
        v[rng.random(n) < 0.01] = 0.0
        v[rng.random(n) < 0.01] = np.inf
    good = (v > 0) & np.isfinite(d) & np.isfinite(v) & (m == 0)
    med, cnt = ctypes.c_double(), ctypes.c_int64()
    ctx = _core.context()
    _lib.check(_lib.lib().dgpu_z2_median(ctx.handle, _lib.MEM_HOST, ctypes.c_int64(n),
                                         d.ctypes.data_as(ctypes.c_void_p), v.ctypes.data_as(ctypes.c_void_p),
                                         m.ctypes.data_as(ctypes.c_void_p), ctypes.byref(med), ctypes.byref(cnt)),
               ctx.handle)
    assert cnt.value == int(good.sum())
    if cnt.value:
        z2 = d[good].astype(np.float64) ** 2 / v[good].astype(np.float64)
        assert med.value == float(np.median(z2))
