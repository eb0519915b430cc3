"""Whole-pipeline parity on the two benchmark configurations, against the
oracle chain (oracle/chain.py) run on the same seeded inputs.

C2: the 4096 x 4096 spatially varying field the bench times (elliptical Moffat
science PSF, FWHM 3.0 -> 4.5 px along the diagonal, 20000 stars, 50
transients, n_max 6, 4 x 4 knots, GCV, decorrelate + score + catalog at 5
sigma), in the FP64 and the mixed-precision arithmetic.

C1: 1024 x 1024, 2000 stars, Gaussian FWHM 2.5 (reference) / 3.5 (science),
n_max 4, a 21 x 21 kernel (radius 10), 3 x 3 knots, score on, decorrelation
off, 1% masked.

Bars (the reference's stage order, python/delta/pipeline.py:654-806):
  stamps, direction, beta and the selected lambda equal;
  masks bit-exact;
  difference (whitened for C2) within 1e-3 of the local sigma at every pixel,
  RMS within 1e-4 sigma;
  score within 1e-3 at every pixel;
  CCL labels bit-exact (src/catalog.cpp:105-261): the device CCL on the
  oracle's score gives the reference CCL's labels and catalog, the reference
  CCL on the device's score gives the device's labels, and the two pipelines'
  label images are equal.
"""

from __future__ import annotations

import numpy as np
import pytest

import bench
import delta_b200 as delta
from delta_b200 import _core, validation
from delta_b200.catalog import CATALOG_DTYPE
from oracle import chain, refbuild
from oracle import numpy_ref as nr

pytestmark = pytest.mark.gpu

LAYERS = ("science_var", "reference_var", "science_mask", "reference_mask")
INT_COLS = ("peak_x", "peak_y", "n_pix", "fwhm_consistent", "mask_flags", "is_dipole", "quality", "psf_chi2_dof",
            "shape_consistent", "near_bright_star")


def _chain(p, **kw):
    if not chain.available():
        pytest.skip("oracle/_ref is not built")
    return chain.run(p.science, p.reference, p.science_var, p.reference_var, p.science_mask, p.reference_mask,
                     saturation=p.saturation, **kw)


@pytest.fixture(scope="module")
def c2():
    p = bench.make_frame(4096, 0)
    kw = {k: v for k, v in bench.subtract_kwargs(p).items() if k != "saturation"}
    return p, _chain(p, **kw)


@pytest.fixture(scope="module")
def c1():
    p = validation.config1_pair(seed=0)
    kw = dict(n_max=4, radius=10, n_knots=3, cv_folds=0, stamp_radius=15, decorrelate=False, score=True,
              source_catalog=True)
    return p, kw, _chain(p, **kw)


def _sigma_errors(got, want, var):
    v = np.asarray(var, np.float64)
    ok = (v > 0) & np.isfinite(got) & np.isfinite(want)
    z = (np.asarray(got, np.float64) - np.asarray(want, np.float64))[ok] / np.sqrt(v[ok])
    return float(np.max(np.abs(z))), float(np.sqrt(np.mean(z * z)))


def _psf_fwhm(psf):
    pos = np.clip(np.asarray(psf, np.float64), 0.0, None)
    ys, xs = np.mgrid[0 : psf.shape[0], 0 : psf.shape[1]]
    tot = pos.sum()
    mx, my = (pos * xs).sum() / tot, (pos * ys).sum() / tot
    vx, vy = (pos * (xs - mx) ** 2).sum() / tot, (pos * (ys - my) ** 2).sum() / tot
    return float(np.sqrt(0.5 * (vx + vy)) / (1.0 / nr.FWHM_PER_SIGMA))  # the chain's expression, same rounding


def _device_labels(score, difference, mask, fwhm):
    cat = _core.build_catalog(score, difference, mask=mask, expected_fwhm=fwhm)
    return cat, _core.catalog_labels(score.shape)


def _reference_labels(score, mask):
    return refbuild.label_components(nr.seed_mask(score, 5.0, +1, mask, True))[0]


def _assert_catalogs_equal(got, want):
    for name in CATALOG_DTYPE.names:
        g, w = np.asarray(got[name]), np.asarray(want[name])
        assert g.shape == w.shape, name
        if name in INT_COLS:
            np.testing.assert_array_equal(g, w, err_msg=name)
        else:
            np.testing.assert_allclose(g, w, rtol=1e-12, atol=1e-12, err_msg=name)


def _check_pipeline(p, res, want, kw):
    sel = _core.select_stamps(p.science, p.reference, p.science_mask, p.reference_mask,
                              stamp_radius=kw.get("stamp_radius", 15), saturation=p.saturation)
    np.testing.assert_array_equal(sel["x"], want["selection"]["x"])
    np.testing.assert_array_equal(sel["y"], want["selection"]["y"])
    assert res.solution.direction == want["direction"]
    assert res.solution.beta == want["beta"]
    assert res.solution.lam == want["fit"]["lambda"]
    th, th0 = np.asarray(res.solution.theta), np.asarray(want["fit"]["theta"])
    theta_rel = float(np.linalg.norm(th - th0) / np.linalg.norm(th0))
    np.testing.assert_array_equal(res.mask, want["mask"])
    d_max, d_rms = _sigma_errors(res.difference, want["difference"], want["variance"])
    s_err = float(np.max(np.abs(res.score.astype(np.float64) - want["score"])))
    assert d_max < 1e-3 and d_rms < 1e-4, (d_max, d_rms, theta_rel)
    assert s_err < 1e-3, s_err
    np.testing.assert_allclose(res.psf, want["psf"], rtol=1e-5, atol=1e-7)

    fwhm = _psf_fwhm(want["psf"])
    # 1. Device CCL on the oracle's products == the reference's CCL and catalog.
    cat, labels = _device_labels(want["score"], want["difference"], want["mask"], fwhm)
    np.testing.assert_array_equal(labels, _reference_labels(want["score"], want["mask"]))
    _assert_catalogs_equal(cat, want["catalog"])
    # 2. Reference CCL on the device's score == the device's labels.
    _, labels_dev = _device_labels(res.score, res.difference, res.mask, _psf_fwhm(res.psf))
    np.testing.assert_array_equal(labels_dev, _reference_labels(res.score, res.mask))
    # 3. End to end: the two pipelines' label images are the same.
    np.testing.assert_array_equal(labels_dev, labels)
    assert len(res.source_catalog) == len(want["catalog"]["x"])
    return {"theta_rel": theta_rel, "diff_max_sigma": d_max, "diff_rms_sigma": d_rms, "score_max_abs": s_err,
            "components": int(labels.max())}


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_c2_pipeline_matches_oracle_chain(c2, precision):
    p, want = c2
    res = delta.subtract(p.science, p.reference, **{k: getattr(p, k) for k in LAYERS},
                         **bench.subtract_kwargs(p, precision))
    stats = _check_pipeline(p, res, want, bench.subtract_kwargs(p))
    assert stats["theta_rel"] < (1e-6 if precision == "fp64" else 1e-5), stats
    print(f"C2 {precision}: {stats}")


def test_c1_pipeline_matches_oracle_chain(c1):
    p, kw, want = c1
    for precision in ("fp64", "mixed", "fp32"):
        res = delta.subtract(p.science, p.reference, **{k: getattr(p, k) for k in LAYERS}, saturation=p.saturation,
                             precision=precision, **kw)
        if precision == "fp32":
            # plain FP32 normal equations: same products up to the FP32 build's error
            assert res.solution.lam == want["fit"]["lambda"]
            np.testing.assert_array_equal(res.mask, want["mask"])
            continue
        stats = _check_pipeline(p, res, want, kw)
        assert stats["theta_rel"] < (1e-6 if precision == "fp64" else 1e-5), stats
        print(f"C1 {precision}: {stats}")
