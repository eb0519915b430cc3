"""High-level difference-imaging pipeline (mirror of python/delta/pipeline.py).

Same classes, keywords and stage order as the reference: coerce inputs, select
stamps and the convolution direction, fit the spatially varying kernel +
background, subtract, optionally decorrelate and score, build the catalog.
Every stage is a ``_core`` call into the sm_100a library.
"""

from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np
from numpy.typing import NDArray

from . import _core
from ._inputs import as_layers, synth_variance
from ._log import log_timing, logger
from ._provenance import environment_cards
from .solution import KernelSolution

_FWHM_TO_SIGMA = 1.0 / 2.354820045030949

_CONFIG_KEYS = frozenset({
    "n_max", "beta", "n_knots", "radius", "stamp_radius", "threshold_sigma", "max_stamps", "saturation",
    "match_radius", "fwhm_radius", "bright_mask", "lambda_grid", "clip_sigma", "clip_iterations", "min_stamps",
    "cv_folds", "spatial_scale", "decorrelate", "score", "source_catalog", "block", "rescale_variance",
    # extensions: normal-equation arithmetic of the device fit ("fp64", "fp32", "mixed") and
    # whether the layers stay resident in HBM across stages (None = when a CUDA device is visible)
    "precision", "device_resident",
})

_CV_EXACT_DESIGN_WARN_BYTES = 256 * 1024 * 1024
_MEDIAN_CHI2_1 = 0.4549364231195724


def _variance_rescale_factor(difference, variance, mask) -> float:
    """median(difference^2 / variance) / median(chi2_1) over good pixels."""
    good = (variance > 0) & np.isfinite(difference) & np.isfinite(variance)
    if mask is not None:
        good &= mask == 0
    if not np.any(good):
        return 1.0
    z2 = difference[good].astype(np.float64) ** 2 / variance[good].astype(np.float64)
    return float(np.median(z2) / _MEDIAN_CHI2_1)


def _log_core_timings(timing) -> None:
    if not timing:
        return
    for label, seconds in timing.items():
        logger.debug("{} done in {:.3f}s", label, seconds)


@dataclass
class DiffResult:
    """Products of a subtraction run."""

    difference: NDArray[np.float32]
    variance: NDArray[np.float32] | None
    mask: NDArray[np.uint8] | None
    score: NDArray[np.float32] | None
    solution: KernelSolution
    psf: NDArray[np.float32] | None = None
    source_catalog: NDArray | None = None
    config: dict[str, object] = field(default_factory=dict)
    elapsed: float = float("nan")
    variance_scale: float | None = None

    def header_cards(self) -> dict[str, object]:
        return {**self.solution.header_cards(), **self.config, **environment_cards(), "DLTELAP": self.elapsed}

    def write(self, path: str, overwrite: bool = False, *, compress: bool = True, extra_cards=None) -> None:
        """Multi-extension FITS with provenance (python/delta/pipeline.py:150-194;
        astropy, as in the reference). Without astropy the uncompressed layout
        (compress=False) is written natively with the same HDUs; the tile-
        compressed layout still needs astropy."""
        cards = self.header_cards()
        if self.variance_scale is not None:
            cards["DLTVSCL"] = self.variance_scale
        if extra_cards:
            cards.update(extra_cards)
        layers = [("VARIANCE", self.variance), ("MASK", self.mask), ("SCORE", self.score)]
        try:
            from astropy.io import fits  # optional dependency
        except ImportError:
            if compress:
                raise ImportError("DiffResult.write(compress=True) needs astropy; compress=False is written "
                                  "without it") from None
            from ._fits_products import write_products

            write_products(str(path), self.difference, layers, self.source_catalog, cards, overwrite=overwrite)
            return
        if compress:
            primary = fits.PrimaryHDU()
            for k, v in cards.items():
                primary.header[k] = v
            hdus = [primary, fits.CompImageHDU(self.difference, name="DIFFERENCE")]
            hdus += [fits.CompImageHDU(a, name=n) for n, a in layers if a is not None]
        else:
            primary = fits.PrimaryHDU(self.difference)
            for k, v in cards.items():
                primary.header[k] = v
            hdus = [primary] + [fits.ImageHDU(a, name=n) for n, a in layers if a is not None]
        if self.source_catalog is not None:
            hdus.append(fits.BinTableHDU(self.source_catalog, name="CATALOG"))
        fits.HDUList(hdus).writeto(path, overwrite=overwrite)

    def build_catalog(self, *, threshold_sigma=5.0, threshold_sigma_dipole=3.0, fwhm_tolerance_lo=0.3,
                      fwhm_tolerance_hi=3.0, aperture_radius=0, exclude_bad_pixels=True, fit_psf_shape=False,
                      shape_chi2_tolerance=3.0, bright_x=None, bright_y=None, bright_star_radius=0.0,
                      max_shape_fit=5000, polarity="positive", as_table=False):
        """Rebuild the source catalog from self.score with custom thresholds."""
        if self.score is None or self.psf is None:
            raise ValueError("build_catalog() requires a score image and PSF stamp; pass score=True to subtract()")
        if fit_psf_shape and self.variance is None:
            raise ValueError("fit_psf_shape=True requires a variance map (self.variance)")
        from .catalog import build_catalog as _build_catalog

        if bright_x is None and bright_y is None and self.solution is not None:
            bright_x = self.solution.stamp_x
            bright_y = self.solution.stamp_y
        return _build_catalog(
            self.score, self.difference, mask=self.mask, psf=self.psf, threshold_sigma=threshold_sigma,
            threshold_sigma_dipole=threshold_sigma_dipole, fwhm_tolerance_lo=fwhm_tolerance_lo,
            fwhm_tolerance_hi=fwhm_tolerance_hi, aperture_radius=aperture_radius,
            exclude_bad_pixels=exclude_bad_pixels, fit_psf_shape=fit_psf_shape,
            shape_chi2_tolerance=shape_chi2_tolerance, variance=self.variance if fit_psf_shape else None,
            bright_x=bright_x, bright_y=bright_y, bright_star_radius=bright_star_radius,
            max_shape_fit=max_shape_fit, polarity=polarity, as_table=as_table)


def _default_beta(fwhm_a: float, fwhm_b: float) -> float:
    """Kernel scale from the two median FWHMs: max(0.8 sqrt(s_broad^2 - s_narrow^2), 0.5)."""
    fwhms = [f for f in (fwhm_a, fwhm_b) if np.isfinite(f) and f > 0]
    if not fwhms:
        return 2.0
    broad, narrow = max(fwhms), min(fwhms)
    diff = (broad * _FWHM_TO_SIGMA) ** 2 - (narrow * _FWHM_TO_SIGMA) ** 2
    k_sigma = np.sqrt(diff) if diff > 0 else 0.0
    return float(max(0.8 * k_sigma, 0.5))


def _estimate_psf(image, xs, ys, radius: int) -> NDArray[np.float32]:
    """Median, unit-sum postage stamp of the listed sources (on the device)."""
    return _core.estimate_psf(image, np.asarray(xs), np.asarray(ys), radius)


class Subtractor:
    """Reusable difference-imaging configuration."""

    def __init__(self, *, n_max: int = 6, beta: float | None = None, n_knots: int = 5, radius: int = 0,
                 stamp_radius: int = 15, threshold_sigma: float = 5.0, max_stamps: int = 200,
                 saturation: float = 0.0, match_radius: int = 2, fwhm_radius: int = 0, bright_mask: float = 0.0,
                 lambda_grid=None, clip_sigma: float = 4.0, clip_iterations: int = 5, min_stamps: int = 5,
                 cv_folds: int = 5, spatial_scale: float | None = None, decorrelate: bool = False,
                 score: bool = False, source_catalog: bool = True, block: int = 256,
                 rescale_variance: bool = False, precision: str = "fp64",
                 device_resident: bool | None = None) -> None:
        self.n_max = n_max
        self.beta = beta
        self.n_knots = n_knots
        self.radius = radius
        self.stamp_radius = stamp_radius
        self.threshold_sigma = threshold_sigma
        self.max_stamps = max_stamps
        self.match_radius = match_radius
        self.fwhm_radius = fwhm_radius
        self.saturation = saturation
        self.bright_mask = bright_mask
        self.lambda_grid = (np.logspace(-6.0, 6.0, 25, dtype=np.float64) if lambda_grid is None
                            else np.asarray(lambda_grid, dtype=np.float64))
        self.clip_sigma = clip_sigma
        self.clip_iterations = clip_iterations
        self.min_stamps = min_stamps
        self.cv_folds = cv_folds
        self.spatial_scale = spatial_scale
        self.decorrelate = decorrelate
        self.score = score
        self.source_catalog = source_catalog
        self.block = block
        self.rescale_variance = rescale_variance
        if precision not in _core.PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(_core.PRECISIONS)}")
        self.precision = precision
        self.device_resident = device_resident

    def config_cards(self) -> dict[str, object]:
        return {
            "DLTSRAD": self.stamp_radius, "DLTTHSIG": self.threshold_sigma, "DLTMAXST": self.max_stamps,
            "DLTSAT": self.saturation, "DLTMRAD": self.match_radius, "DLTFRAD": self.fwhm_radius,
            "DLTBMASK": self.bright_mask, "DLTCLPSG": self.clip_sigma, "DLTCLPIT": self.clip_iterations,
            "DLTMINST": self.min_stamps, "DLTCVF": self.cv_folds,
            "DLTSSCL": self.spatial_scale if self.spatial_scale is not None else 0.0,
            "DLTDECOR": self.decorrelate, "DLTSCORE": self.score, "DLTSCAT": self.source_catalog,
            "DLTBLK": self.block, "DLTPREC": self.precision,
        }

    # -- internals -------------------------------------------------------------

    def _select(self, sci, ref, sci_mask, ref_mask, catalog):
        cat_x = cat_y = None
        if catalog is not None:
            cat = np.asarray(catalog, dtype=np.int32)
            cat_x = np.ascontiguousarray(cat[:, 0])
            cat_y = np.ascontiguousarray(cat[:, 1])
        return _core.select_stamps(sci, ref, science_mask=sci_mask, reference_mask=ref_mask, catalog_x=cat_x,
                                   catalog_y=cat_y, stamp_radius=self.stamp_radius,
                                   threshold_sigma=self.threshold_sigma, max_stamps=self.max_stamps,
                                   saturation=self.saturation, match_radius=self.match_radius,
                                   fwhm_radius=self.fwhm_radius)

    def _fit(self, science, reference, *, science_var, reference_var, science_mask, reference_mask, gain,
             read_noise, catalog, direction):
        sci, svar, smask = as_layers(science, science_var, science_mask)
        ref, rvar, rmask = as_layers(reference, reference_var, reference_mask)
        if sci.shape != ref.shape:
            raise ValueError("science and reference must share a shape")
        if svar is None and gain is not None:
            svar = synth_variance(sci, gain, read_noise)
        if rvar is None and gain is not None:
            rvar = synth_variance(ref, gain, read_noise)
        logger.info("fitting {} x {} frame", sci.shape[1], sci.shape[0])
        with log_timing("stamp selection"):
            sel = self._select(sci, ref, smask, rmask, catalog)
        n_stamps = int(np.asarray(sel["x"]).size)
        logger.info("selected {} stamps (median FWHM: science={:.2f}, reference={:.2f} px)", n_stamps,
                    sel["median_fwhm_science"], sel["median_fwhm_reference"])
        if n_stamps == 0:
            raise ValueError("no stamps selected; lower threshold_sigma, supply a catalog, or widen match_radius "
                             "if science/reference are astrometrically misregistered")
        if direction is None:
            direction = sel["direction"]
        elif direction not in ("science", "reference"):
            raise ValueError(f"direction must be 'science', 'reference', or None, got {direction!r}")
        logger.info("convolution direction: {}", direction)
        if direction == "science":
            target, tvar, tmask = ref, rvar, rmask
            conv, cvar, cmask = sci, svar, smask
            sign = -1.0
        else:
            target, tvar, tmask = sci, svar, smask
            conv, cvar, cmask = ref, rvar, rmask
            sign = 1.0
        beta = self.beta
        if beta is None:
            beta = _default_beta(sel["median_fwhm_science"], sel["median_fwhm_reference"])
            logger.debug("auto-selected basis scale beta={:.3f}", beta)
        h, w = sci.shape
        nkx = nky = self.n_knots
        if self.spatial_scale is not None and self.spatial_scale > 0:
            nkx = int(np.clip(round((w - 1) / self.spatial_scale) + 1, 3, self.n_knots))
            nky = int(np.clip(round((h - 1) / self.spatial_scale) + 1, 3, self.n_knots))
        knots = _core.grid_knots(0.0, 0.0, w - 1.0, h - 1.0, nkx, nky)
        stamp_x = np.ascontiguousarray(sel["x"], dtype=np.int32)
        stamp_y = np.ascontiguousarray(sel["y"], dtype=np.int32)
        with log_timing("kernel solve"):
            fit = _core.fit_kernel(target, conv, knots, stamp_x, stamp_y, self.stamp_radius, beta, self.n_max,
                                   self.lambda_grid, radius=self.radius, clip_sigma=self.clip_sigma,
                                   clip_iterations=self.clip_iterations, min_stamps=self.min_stamps,
                                   cv_folds=self.cv_folds, science_var=tvar, reference_var=cvar,
                                   science_mask=tmask, reference_mask=cmask, precision=self.precision)
        _log_core_timings(fit.get("timing"))
        selector = f"{self.cv_folds}-fold CV" if self.cv_folds > 1 else "GCV"
        logger.info("kernel fit: lambda={:.3g} ({}), eff.dof={:.1f}, reduced chi2={:.3f} ({} stamps used, {} "
                    "rejected of {}, {} px)", fit["lambda"], selector, fit["effective_dof"], fit["reduced_chi2"],
                    fit["n_stamps_used"], fit["n_stamps_rejected"], fit["n_stamps_total"], fit["n_pixels"])
        lam_grid = np.asarray(fit["lambda_grid"])
        if lam_grid.size > 1 and fit["lambda"] in (lam_grid[0], lam_grid[-1]):
            edge = "lower" if fit["lambda"] == lam_grid[0] else "upper"
            logger.warning("selected lambda={:.3g} ({}) sits at the {} edge of lambda_grid [{:.3g}, {:.3g}] -- "
                           "consider widening lambda_grid", fit["lambda"], selector, edge, lam_grid[0], lam_grid[-1])
        if fit.get("cv_exact_design_bytes", 0) > _CV_EXACT_DESIGN_WARN_BYTES:
            logger.warning("exact (non-stamped) k-fold CV path used a whitened design equivalent to {:.2f} GB, "
                           "rebuilt every IRLS pass", fit["cv_exact_design_bytes"] / 1e9)
        if fit["reduced_chi2"] > 3.0:
            logger.warning("kernel fit reduced chi2={:.2f} >> 1: stellar residuals likely", fit["reduced_chi2"])
        solution = KernelSolution(
            beta=beta, n_max=self.n_max, radius=self.radius, knots=knots, theta=fit["theta"],
            n_components=fit["n_components"], n_spatial=fit["n_spatial"], lam=fit["lambda"], gcv=fit["gcv"],
            effective_dof=fit["effective_dof"], rss=fit["rss"], component_sums=fit["component_sums"],
            direction=direction, shape=(h, w), reduced_chi2=fit["reduced_chi2"],
            n_stamps_used=fit["n_stamps_used"], n_stamps_rejected=fit["n_stamps_rejected"],
            stamp_x=fit["stamp_x"], stamp_y=fit["stamp_y"], stamp_chi2=fit["stamp_chi2"],
            stamp_accepted=fit["stamp_accepted"])
        return solution, (target, conv, tvar, cvar, tmask, cmask, sign, stamp_x, stamp_y)

    def _coerce_apply_layers(self, solution, science, reference, *, science_var, reference_var, science_mask,
                             reference_mask, gain, read_noise):
        sci, svar, smask = as_layers(science, science_var, science_mask)
        ref, rvar, rmask = as_layers(reference, reference_var, reference_mask)
        if sci.shape != ref.shape:
            raise ValueError("science and reference must share a shape")
        if sci.shape != tuple(solution.shape):
            raise ValueError(f"solution shape {solution.shape} does not match input frame shape {sci.shape}")
        if svar is None and gain is not None:
            svar = synth_variance(sci, gain, read_noise)
        if rvar is None and gain is not None:
            rvar = synth_variance(ref, gain, read_noise)
        if solution.direction == "science":
            return (ref, sci, rvar, svar, rmask, smask, -1.0, solution.stamp_x, solution.stamp_y)
        return (sci, ref, svar, rvar, smask, rmask, 1.0, solution.stamp_x, solution.stamp_y)

    def _subtract(self, solution, layers) -> DiffResult:
        target, conv, tvar, cvar, tmask, cmask, sign, stamp_x, stamp_y = layers
        out_levels = [v for v in (self.saturation, self.bright_mask) if v and v > 0]
        out_saturation = min(out_levels) if out_levels else 0.0
        with log_timing("full-frame subtraction"):
            diff = _core.subtract(target, conv, solution.knots, solution.theta, solution.beta, solution.n_max,
                                  radius=solution.radius, saturation=out_saturation, science_var=tvar,
                                  reference_var=cvar, science_mask=tmask, reference_mask=cmask)
        _log_core_timings(diff.get("timing"))
        difference = diff["difference"]
        if sign < 0:
            np.negative(difference, out=difference)
        variance = diff["variance"]
        mask = diff["mask"]
        variance_scale = None
        if self.rescale_variance and variance is not None:
            variance_scale = _variance_rescale_factor(difference, variance, mask)
            variance = variance * variance_scale
            logger.info("variance rescaled by {:.4f} to force diff-image reduced chi2=1", variance_scale)
        elif self.rescale_variance:
            logger.warning("variance rescale requested but no variance available; skipping")
        whitened = difference
        white_var = None
        if self.decorrelate:
            if tvar is not None and cvar is not None:
                with log_timing("noise decorrelation"):
                    dec = _core.decorrelate(difference, solution.knots, solution.theta, solution.beta,
                                            solution.n_max, tvar, cvar, block=self.block)
                whitened = dec["difference"]
                white_var = dec["variance"]
                _log_core_timings(dec.get("timing"))
                if variance_scale is not None:
                    white_var *= variance_scale
            else:
                logger.warning("decorrelation requested but no variance available; skipping")
        score = None
        psf = None
        if self.score:
            with log_timing("matched-filter score"):
                if stamp_x is None or np.asarray(stamp_x).size == 0:
                    raise ValueError("score requested but the solution carries no stamp positions for PSF "
                                     "estimation")
                psf_radius = min(self.stamp_radius, 8)
                psf = _estimate_psf(target, stamp_x, stamp_y, psf_radius)
                if white_var is not None:
                    score_var = np.asarray(white_var, dtype=np.float32)
                    if tvar is not None and cvar is not None:
                        psf = _core.whiten_score_psf(psf, solution.knots, solution.theta, solution.beta,
                                                     solution.n_max, tvar, cvar, self.block, radius=solution.radius)
                elif variance is not None:
                    score_var = np.asarray(variance, dtype=np.float32)
                else:
                    score_var = np.full(whitened.shape, float(np.var(whitened)), dtype=np.float32)
                score = _core.matched_filter(whitened, psf, score_var)
            _log_core_timings(_core.drain_timing())
        out_var = white_var if white_var is not None else variance
        source_catalog = None
        if score is not None and self.source_catalog:
            with log_timing("catalog"):
                from .catalog import build_catalog as _build_catalog

                source_catalog = _build_catalog(score, whitened, mask=mask, psf=psf)
        return DiffResult(difference=whitened, variance=out_var, mask=mask, score=score, solution=solution, psf=psf,
                          source_catalog=source_catalog, variance_scale=variance_scale)

    def _use_device(self) -> bool:
        from . import _device

        if self.device_resident is None:
            return _device.available()
        if self.device_resident and not _device.available():
            raise RuntimeError("device_resident=True needs a visible CUDA device")
        return bool(self.device_resident)

    def _run_resident(self, science, reference, *, science_var, reference_var, science_mask, reference_mask, gain,
                      read_noise, catalog=None, direction=None, solution=None) -> DiffResult:
        """Same stages as _fit/_subtract with every layer uploaded once and kept in HBM
        between stages; only the products come back (into pinned host memory)."""
        from . import _device

        sci, svar, smask = as_layers(science, science_var, science_mask)
        ref, rvar, rmask = as_layers(reference, reference_var, reference_mask)
        if sci.shape != ref.shape:
            raise ValueError("science and reference must share a shape")
        if solution is not None and sci.shape != tuple(solution.shape):
            raise ValueError(f"solution shape {solution.shape} does not match input frame shape {sci.shape}")
        if direction is not None and direction not in ("science", "reference"):
            raise ValueError(f"direction must be 'science', 'reference', or None, got {direction!r}")
        if svar is None and gain is not None:
            svar = synth_variance(sci, gain, read_noise)
        if rvar is None and gain is not None:
            rvar = synth_variance(ref, gain, read_noise)
        logger.info("fitting {} x {} frame (device resident)", sci.shape[1], sci.shape[0])
        frame = _device.DeviceFrame.from_numpy(sci, ref, svar, rvar, smask, rmask, non_blocking=True, serialize=True)
        started = {}

        def early(products):  # final before the score and catalog: start their download
            started["dl"] = _device.EarlyDownload(products)

        try:
            if solution is None:
                out = _device.run(self, frame, catalog, direction, early=early)
            else:
                out = _device.apply_solution(self, solution, frame, early=early)
        except BaseException:
            frame.finish_upload()  # the host layers must outlive their copies
            raise
        host = _device.download(out, started.get("dl"))
        return DiffResult(difference=host["difference"], variance=host["variance"], mask=host["mask"],
                          score=host["score"], solution=out["solution"], psf=out["psf"],
                          source_catalog=out["catalog"], variance_scale=out["variance_scale"])

    # -- public API --------------------------------------------------------------

    def fit(self, science, reference, *, science_var=None, reference_var=None, science_mask=None,
            reference_mask=None, gain=None, read_noise=0.0, catalog=None, direction=None) -> KernelSolution:
        solution, _ = self._fit(science, reference, science_var=science_var, reference_var=reference_var,
                                science_mask=science_mask, reference_mask=reference_mask, gain=gain,
                                read_noise=read_noise, catalog=catalog, direction=direction)
        return solution

    def subtract(self, science, reference, *, science_var=None, reference_var=None, science_mask=None,
                 reference_mask=None, gain=None, read_noise=0.0, catalog=None, direction=None) -> DiffResult:
        start = time.perf_counter()
        if self._use_device():
            result = self._run_resident(science, reference, science_var=science_var, reference_var=reference_var,
                                        science_mask=science_mask, reference_mask=reference_mask, gain=gain,
                                        read_noise=read_noise, catalog=catalog, direction=direction)
            result.config = self.config_cards()
            result.elapsed = time.perf_counter() - start
            return result
        solution, layers = self._fit(science, reference, science_var=science_var, reference_var=reference_var,
                                     science_mask=science_mask, reference_mask=reference_mask, gain=gain,
                                     read_noise=read_noise, catalog=catalog, direction=direction)
        result = self._subtract(solution, layers)
        result.config = self.config_cards()
        result.elapsed = time.perf_counter() - start
        return result

    def subtract_batch(self, frames, *, max_in_flight: int | None = None) -> list[DiffResult]:
        """Subtract several frames concurrently (an extension: the reference has no
        batch call). Each item of `frames` is a dict of subtract() keyword
        arguments (science, reference and optionally the variance / mask layers,
        gain, read_noise, catalog, direction). With a CUDA device visible, up to
        `max_in_flight` frames (default: up to 4) run at once, each on its own
        host thread, library context and CUDA stream; results are returned in
        input order. Without a device the frames run one after another."""
        items = [dict(f) for f in frames]
        if not items:
            return []
        if not self._use_device():
            return [self.subtract(**it) for it in items]
        from . import _device

        ex = _device.runner(max_in_flight or min(len(items), 4))
        futs = [ex.submit(_device.on_own_stream, self.subtract, **it) for it in items]
        return [f.result() for f in futs]

    def apply(self, solution: KernelSolution, science, reference, *, science_var=None, reference_var=None,
              science_mask=None, reference_mask=None, gain=None, read_noise=0.0) -> DiffResult:
        start = time.perf_counter()
        if self._use_device():
            result = self._run_resident(science, reference, science_var=science_var, reference_var=reference_var,
                                        science_mask=science_mask, reference_mask=reference_mask, gain=gain,
                                        read_noise=read_noise, solution=solution)
            result.config = self.config_cards()
            result.elapsed = time.perf_counter() - start
            return result
        layers = self._coerce_apply_layers(solution, science, reference, science_var=science_var,
                                           reference_var=reference_var, science_mask=science_mask,
                                           reference_mask=reference_mask, gain=gain, read_noise=read_noise)
        result = self._subtract(solution, layers)
        result.config = self.config_cards()
        result.elapsed = time.perf_counter() - start
        return result

    def subtract_files(self, pairs, outputs=None, *, max_in_flight: int | None = None, overwrite: bool = False,
                       **call) -> list[DiffResult]:
        """Subtract frame pairs stored as FITS files (an extension: the batched form
        of the reference CLI's read -> subtract -> write, python/delta/cli.py). Each
        item of `pairs` is (science_path, reference_path); the data, VARIANCE and
        MASK layers of each file are its inputs. With `outputs` (one path per pair)
        the difference, variance and mask are written as the reference's
        write_fits lays them out. Every frame is read, subtracted and written by
        its own worker (up to `max_in_flight`, default up to 4), so one frame's
        file I/O overlaps the others' compute; with a device the layers are read
        straight into pinned host memory. Results come back in input order."""
        items = [tuple(p) for p in pairs]
        outs = list(outputs) if outputs is not None else [None] * len(items)
        if len(outs) != len(items):
            raise ValueError("outputs must give one path per pair")
        use_device = self._use_device()
        alloc = None
        if use_device:
            import torch

            def alloc(shape, dtype):
                return torch.empty(shape, dtype=torch.from_numpy(np.zeros(1, dtype)).dtype, pin_memory=True).numpy()

        def one(sci_path, ref_path, out_path):
            sci = _core.read_fits(str(sci_path), alloc=alloc)
            ref = _core.read_fits(str(ref_path), alloc=alloc)
            result = self.subtract(sci["data"], ref["data"], science_var=sci["variance"],
                                   reference_var=ref["variance"], science_mask=sci["mask"],
                                   reference_mask=ref["mask"], **call)
            if out_path is not None:
                _core.write_fits(str(out_path), result.difference, result.variance, result.mask, overwrite=overwrite)
            return result

        if not items:
            return []
        if not use_device:
            return [one(s, r, o) for (s, r), o in zip(items, outs, strict=True)]
        from . import _device

        ex = _device.runner(max_in_flight or min(len(items), 4))
        futs = [ex.submit(_device.on_own_stream, one, s, r, o) for (s, r), o in zip(items, outs, strict=True)]
        return [f.result() for f in futs]

    def apply_batch(self, solution: KernelSolution, frames, *, max_in_flight: int | None = None) -> list[DiffResult]:
        """Apply one frozen solution to several frame pairs concurrently (an
        extension: the reference applies a solution one frame at a time, through
        apply()). Each item of `frames` is a dict of apply() keyword arguments
        (science, reference and optionally the variance / mask layers, gain,
        read_noise). Runs like subtract_batch(): up to `max_in_flight` frames
        (default: up to 4) at once, each on its own host thread, library context
        and CUDA stream, results in input order; every result equals what apply()
        returns for that frame alone."""
        items = [dict(f) for f in frames]
        if not items:
            return []
        if not self._use_device():
            return [self.apply(solution, **it) for it in items]
        from . import _device

        ex = _device.runner(max_in_flight or min(len(items), 4))
        futs = [ex.submit(_device.on_own_stream, self.apply, solution, **it) for it in items]
        return [f.result() for f in futs]


def subtract(science, reference, **kwargs) -> DiffResult:
    """Configure a Subtractor from the config keywords and run it once."""
    config = {k: v for k, v in kwargs.items() if k in _CONFIG_KEYS}
    call = {k: v for k, v in kwargs.items() if k not in _CONFIG_KEYS}
    return Subtractor(**config).subtract(science, reference, **call)


def subtract_batch(frames, *, max_in_flight: int | None = None, **kwargs) -> list[DiffResult]:
    """Configure a Subtractor from the config keywords and subtract several frames
    concurrently (extension). Non-config keywords (gain, read_noise, ...) apply
    to every frame unless the frame's own dict sets them."""
    config = {k: v for k, v in kwargs.items() if k in _CONFIG_KEYS}
    call = {k: v for k, v in kwargs.items() if k not in _CONFIG_KEYS}
    items = [{**call, **dict(f)} for f in frames]
    return Subtractor(**config).subtract_batch(items, max_in_flight=max_in_flight)


def apply(solution: KernelSolution, science, reference, **kwargs) -> DiffResult:
    """Apply a frozen solution without re-fitting."""
    config = {k: v for k, v in kwargs.items() if k in _CONFIG_KEYS}
    call = {k: v for k, v in kwargs.items() if k not in _CONFIG_KEYS}
    return Subtractor(**config).apply(solution, science, reference, **call)


def subtract_files(pairs, outputs=None, *, max_in_flight: int | None = None, overwrite: bool = False,
                   **kwargs) -> list[DiffResult]:
    """Configure a Subtractor from the config keywords and subtract FITS frame
    pairs (extension; see Subtractor.subtract_files)."""
    config = {k: v for k, v in kwargs.items() if k in _CONFIG_KEYS}
    call = {k: v for k, v in kwargs.items() if k not in _CONFIG_KEYS}
    return Subtractor(**config).subtract_files(pairs, outputs, max_in_flight=max_in_flight, overwrite=overwrite,
                                               **call)


def apply_batch(solution: KernelSolution, frames, *, max_in_flight: int | None = None, **kwargs) -> list[DiffResult]:
    """Configure a Subtractor from the config keywords and apply one frozen
    solution to several frame pairs concurrently (extension). Non-config
    keywords apply to every frame unless the frame's own dict sets them."""
    config = {k: v for k, v in kwargs.items() if k in _CONFIG_KEYS}
    call = {k: v for k, v in kwargs.items() if k not in _CONFIG_KEYS}
    items = [{**call, **dict(f)} for f in frames]
    return Subtractor(**config).apply_batch(solution, items, max_in_flight=max_in_flight)
