"""CPU chain of delta.subtract for one frame -- TEST INFRASTRUCTURE ONLY.

The reference's Subtractor stage order (python/delta/pipeline.py:450-800:
select stamps -> direction -> fit -> subtract -> sign -> [decorrelate] ->
[PSF estimate, whitened PSF, matched filter] -> catalog), each stage run by the
oracle:

  stamp selection  the reference's detect.cpp compiled from source (oracle/_ref)
  kernel fit       numpy_ref.fit_kernel (FP64 restatement of src/fit.cpp's IRLS), each pass's
                   GLS assembly and lambda-grid solves in C with OpenMP (oracle/csrc/oracle_fit.c,
                   src/solve.cpp:70-262), B_n through the reference's convolve.cpp
  subtract         cref.subtract (C restatement of src/subtract.cpp, float semantics)
  decorrelate      numpy_ref.decorrelate (src/noise.cpp)
  PSF estimate     numpy_ref.estimate_psf (python/delta/pipeline.py:285-302)
  whitened PSF     numpy_ref.whiten_score_psf (src/bindings.cpp:796-874)
  score            cref.matched_filter (src/noise.cpp:535-632)
  catalog          the reference's catalog.cpp compiled from source (oracle/_ref)

Used by the tests as the stage-by-stage checker and by bench.py as the timed
CPU baseline. Needs oracle/_ref (built by oracle/Makefile from the reference
sources) for selection and the catalog.
"""

from __future__ import annotations

import time

import numpy as np

from . import cref, refbuild
from . import numpy_ref as nr

DESCRIPTION = ("the reference's detect/catalog/basis-convolve code compiled from source + C (OpenMP) restatements "
               "of subtract, the matched filter and the FP64 GLS assembly / lambda-grid solves of the fit + NumPy "
               "FP64 restatements of the IRLS control and the decorrelation")


def available() -> bool:
    return refbuild.available() and cref.available()


def run(science, reference, science_var, reference_var, science_mask, reference_mask, *, n_max=6, n_knots=5,
        radius=0, stamp_radius=15, threshold_sigma=5.0, max_stamps=200, saturation=0.0, match_radius=2,
        fwhm_radius=0, lambda_grid=None, clip_sigma=4.0, clip_iterations=5, min_stamps=5, cv_folds=0,
        decorrelate=True, score=True, source_catalog=True, block=256, timings=None) -> dict:
    """One frame through the CPU chain; ``timings`` (a dict) collects per-stage seconds."""
    t = timings if timings is not None else {}

    def mark(label, t0):
        t[label] = t.get(label, 0.0) + time.perf_counter() - t0
        return time.perf_counter()

    grid = np.logspace(-6.0, 6.0, 25) if lambda_grid is None else np.asarray(lambda_grid, np.float64)
    t0 = time.perf_counter()
    sel = refbuild.select_stamps(science, reference, science_mask, reference_mask, stamp_radius=stamp_radius,
                                 threshold_sigma=threshold_sigma, max_stamps=max_stamps, saturation=saturation,
                                 fwhm_radius=fwhm_radius, match_radius=match_radius)
    t0 = mark("stamp selection", t0)
    if sel["x"].size == 0:
        raise ValueError("no stamps selected")
    if sel["direction"] == "science":
        target, tvar, tmask, conv, cvar, cmask, sign = (reference, reference_var, reference_mask, science,
                                                        science_var, science_mask, -1.0)
    else:
        target, tvar, tmask, conv, cvar, cmask, sign = (science, science_var, science_mask, reference,
                                                        reference_var, reference_mask, 1.0)
    beta = nr.default_beta(sel["median_fwhm_science"], sel["median_fwhm_reference"])
    r = nr.resolve_radius(beta, n_max, radius)
    h, w = science.shape
    knots = nr.grid_knots(0.0, 0.0, w - 1.0, h - 1.0, n_knots, n_knots)
    bconv = (lambda patch: refbuild.basis_convolve(patch, beta, n_max, r)) if refbuild.available() else None
    fit = nr.fit_kernel(target, conv, knots, sel["x"], sel["y"], stamp_radius, beta, n_max, grid, radius=r,
                        clip_sigma=clip_sigma, clip_iterations=clip_iterations, min_stamps=min_stamps,
                        cv_folds=cv_folds, science_var=tvar, reference_var=cvar, science_mask=tmask,
                        reference_mask=cmask, basis_convolve_fn=bconv, gcv_solver=cref.gls_gcv)
    t0 = mark("kernel solve", t0)
    sub = cref.subtract(target, conv, knots, fit["theta"], beta, n_max, r, saturation, tvar, cvar, tmask, cmask)
    diff = sub["difference"]
    if sign < 0:
        np.negative(diff, out=diff)
    t0 = mark("full-frame subtraction", t0)
    whitened, white_var = diff, None
    if decorrelate and tvar is not None and cvar is not None:
        dec = nr.decorrelate(diff, knots, fit["theta"], beta, n_max, tvar, cvar, block=block, radius=r)
        whitened, white_var = dec["difference"], dec["variance"]
        t0 = mark("noise decorrelation", t0)
    out = {"selection": sel, "beta": beta, "radius": r, "knots": knots, "fit": fit, "direction": sel["direction"],
           "difference": whitened, "variance": white_var if white_var is not None else sub["variance"],
           "mask": sub["mask"], "psf": None, "score": None, "catalog": None}
    if score:
        psf = nr.estimate_psf(target, sel["x"], sel["y"], min(stamp_radius, 8))
        if white_var is not None:
            psf = nr.whiten_score_psf(psf, knots, fit["theta"], beta, n_max, tvar, cvar, block, radius=r)
            score_var = white_var
        elif sub["variance"] is not None:
            score_var = sub["variance"]
        else:
            score_var = np.full(whitened.shape, float(np.var(whitened)), np.float32)
        out["psf"] = psf
        out["score"] = cref.matched_filter(whitened, psf, score_var)
        t0 = mark("matched-filter score", t0)
        if source_catalog:
            pos = np.clip(psf.astype(np.float64), 0.0, None)
            ys, xs = np.mgrid[0 : psf.shape[0], 0 : psf.shape[1]]
            tot = pos.sum()
            mx, my = (pos * xs).sum() / tot, (pos * ys).sum() / tot
            vx, vy = (pos * (xs - mx) ** 2).sum() / tot, (pos * (ys - my) ** 2).sum() / tot
            # python/delta/catalog.py:60-74
            fwhm = float(np.sqrt(0.5 * (vx + vy)) / (1.0 / nr.FWHM_PER_SIGMA))
            out["catalog"] = refbuild.build_catalog(out["score"], whitened, out["mask"], expected_fwhm=fwhm)
            mark("catalog", t0)
    return out
