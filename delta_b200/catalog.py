"""Source catalog from the score image (mirror of python/delta/catalog.py).

Thin wrapper over the device connected-component labeller
(``_core.build_catalog``): resolves the expected PSF FWHM, handles the
polarity selection and packs the columns into a structured array.
"""

from __future__ import annotations

import numpy as np
from numpy.typing import NDArray

from . import _core
from .validation import FWHM_TO_SIGMA

CATALOG_DTYPE = np.dtype(
    [
        ("x", np.float64), ("y", np.float64), ("peak_x", np.int32), ("peak_y", np.int32),
        ("peak_snr", np.float64), ("n_pix", np.int32), ("flux", np.float64), ("expected_n_pix", np.float64),
        ("fwhm_ratio", np.float64), ("fwhm_consistent", np.bool_), ("mask_flags", np.uint8),
        ("is_dipole", np.bool_), ("psf_chi2", np.float64), ("psf_chi2_dof", np.int32),
        ("psf_amplitude", np.float64), ("psf_amplitude_err", np.float64), ("shape_consistent", np.bool_),
        ("bright_star_dist", np.float64), ("near_bright_star", np.bool_), ("quality", np.uint8),
    ]
)

QUALITY_FWHM_INCONSISTENT = 1 << 0
QUALITY_DIPOLE = 1 << 1
QUALITY_MASKED = 1 << 2
QUALITY_SHAPE_INCONSISTENT = 1 << 3
QUALITY_NEAR_BRIGHT_STAR = 1 << 4


def _measure_psf_fwhm(psf) -> float:
    """Second-moment FWHM (px) of a small PSF stamp (positive part)."""
    psf = np.asarray(psf, dtype=np.float64)
    h, w = psf.shape
    ys, xs = np.mgrid[0:h, 0:w]
    weight = np.clip(psf, 0.0, None)
    total = weight.sum()
    if total <= 0:
        raise ValueError("PSF stamp has no positive flux")
    mx = (weight * xs).sum() / total
    my = (weight * ys).sum() / total
    varx = (weight * (xs - mx) ** 2).sum() / total
    vary = (weight * (ys - my) ** 2).sum() / total
    return float(np.sqrt(0.5 * (varx + vary)) / FWHM_TO_SIGMA)


def _pack(raw: dict) -> NDArray[np.void]:
    n = raw["x"].shape[0]
    cat = np.empty(n, dtype=CATALOG_DTYPE)
    for name in CATALOG_DTYPE.names:
        cat[name] = raw[name]
    return cat


def build_catalog(score, difference, *, mask=None, psf=None, expected_fwhm=None, threshold_sigma: float = 5.0,
                  threshold_sigma_dipole: float = 3.0, fwhm_tolerance_lo: float = 0.3,
                  fwhm_tolerance_hi: float = 3.0, aperture_radius: int = 0, exclude_bad_pixels: bool = True,
                  fit_psf_shape: bool = False, shape_chi2_tolerance: float = 3.0, variance=None, bright_x=None,
                  bright_y=None, bright_star_radius: float = 0.0, max_shape_fit: int = 5000,
                  polarity: str = "positive", as_table: bool = False):
    """Connected-component catalog of a match-filtered score image (8-connected,
    positive at threshold_sigma, negative at threshold_sigma_dipole for dipole
    flags); exactly one of ``psf`` / ``expected_fwhm``; polarity "positive",
    "negative" or "both" (adds a ``sign`` column)."""
    if (psf is None) == (expected_fwhm is None):
        raise ValueError("supply exactly one of `psf` or `expected_fwhm`")
    if fit_psf_shape and psf is None:
        raise ValueError("fit_psf_shape=True needs `psf` (not `expected_fwhm`)")
    if fit_psf_shape and variance is None:
        raise ValueError("fit_psf_shape=True needs `variance`")
    if polarity not in ("positive", "negative", "both"):
        raise ValueError('polarity must be one of "positive", "negative", "both"')
    fwhm = _measure_psf_fwhm(psf) if psf is not None else float(expected_fwhm or 0.0)
    score = np.ascontiguousarray(score, dtype=np.float32)
    difference = np.ascontiguousarray(difference, dtype=np.float32)
    mask = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint8)
    variance = None if variance is None else np.ascontiguousarray(variance, dtype=np.float32)
    psf_arr = None if psf is None else np.ascontiguousarray(psf, dtype=np.float32)
    bx = None if bright_x is None else np.ascontiguousarray(bright_x, dtype=np.float64)
    by = None if bright_y is None else np.ascontiguousarray(bright_y, dtype=np.float64)

    def _run(neg: bool):
        return _core.build_catalog(
            score, difference, mask=mask, threshold_sigma=threshold_sigma,
            threshold_sigma_dipole=threshold_sigma_dipole, expected_fwhm=fwhm, fwhm_tolerance_lo=fwhm_tolerance_lo,
            fwhm_tolerance_hi=fwhm_tolerance_hi, aperture_radius=aperture_radius,
            exclude_bad_pixels=exclude_bad_pixels, return_negative=neg, fit_psf_shape=fit_psf_shape,
            shape_chi2_tolerance=shape_chi2_tolerance, variance=variance,
            psf=psf_arr if fit_psf_shape else None, bright_star_radius=bright_star_radius,
            max_shape_fit=max_shape_fit, bright_x=bx, bright_y=by)

    if polarity == "positive":
        cat = _pack(_run(False))
    elif polarity == "negative":
        cat = _pack(_run(True))
    else:
        pos = _pack(_run(False))
        neg = _pack(_run(True))
        both = np.dtype([*CATALOG_DTYPE.descr, ("sign", np.int8)])
        cat = np.empty(len(pos) + len(neg), dtype=both)
        for name in CATALOG_DTYPE.names:
            cat[name] = np.concatenate([pos[name], neg[name]])
        cat["sign"] = np.concatenate([np.ones(len(pos), np.int8), -np.ones(len(neg), np.int8)])
    if as_table:
        from astropy.table import Table  # optional dependency

        return Table(cat)
    return cat
