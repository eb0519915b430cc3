"""Synthetic source injection and recovery helpers (mirror of the reference's
python/delta/validation.py), plus seeded synthesizers for the benchmark
configurations (Gaussian / elliptical-Moffat PSFs, power-law fluxes, Poisson +
read noise, bad columns, saturated cores, injected transients).

Everything here is host-side NumPy input generation; it is not part of the
subtraction path.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
from numpy.typing import NDArray

# 1 / (2*sqrt(2 ln 2)).
FWHM_TO_SIGMA = 1.0 / 2.354820045030949


def gaussian_psf(shape, x, y, flux, sigma) -> NDArray[np.float64]:
    """A Gaussian point source of given total `flux` and `sigma` on a blank frame."""
    h, w = shape
    ys, xs = np.mgrid[0:h, 0:w]
    amp = flux / (2.0 * np.pi * sigma**2)
    return amp * np.exp(-((xs - x) ** 2 + (ys - y) ** 2) / (2.0 * sigma**2))


def inject(image, positions, fluxes, sigma) -> NDArray:
    """Copy of `image` with Gaussian sources added at `positions`."""
    out = np.array(image, dtype=np.float64, copy=True)
    out += render_stars(out.shape, positions, fluxes, sigma)
    return out.astype(image.dtype, copy=False)


def render_stars(shape, positions, fluxes, sigma, radius: int | None = None) -> NDArray[np.float64]:
    """Render Gaussian point sources within a local box (~5 sigma) each."""
    h, w = shape
    out = np.zeros((h, w), dtype=np.float64)
    if radius is None:
        radius = int(np.ceil(5.0 * sigma))
    norm = 1.0 / (2.0 * np.pi * sigma**2)
    two_s2 = 2.0 * sigma**2
    for (x, y), f in zip(positions, fluxes, strict=True):
        ix, iy = int(round(x)), int(round(y))
        x0, x1 = max(0, ix - radius), min(w, ix + radius + 1)
        y0, y1 = max(0, iy - radius), min(h, iy + radius + 1)
        if x0 >= x1 or y0 >= y1:
            continue
        ys, xs = np.mgrid[y0:y1, x0:x1]
        out[y0:y1, x0:x1] += (f * norm) * np.exp(-((xs - x) ** 2 + (ys - y) ** 2) / two_s2)
    return out


def sample_starfield(shape, n_stars: int, rng, flux_range=(200.0, 60000.0), slope: float = 1.8,
                     border: int = 16, min_separation: float = 0.0):
    """Uniform positions and bounded power-law fluxes p(F) ~ F^-slope."""
    rng = np.random.default_rng(rng)
    h, w = shape
    fmin, fmax = flux_range
    u = rng.random(n_stars)
    if abs(slope - 1.0) < 1e-9:
        fluxes = fmin * (fmax / fmin) ** u
    else:
        a = 1.0 - slope
        fluxes = (fmin**a + u * (fmax**a - fmin**a)) ** (1.0 / a)
    xs = np.empty(n_stars)
    ys = np.empty(n_stars)
    min_sep2 = min_separation**2
    count = attempts = 0
    while count < n_stars and attempts < 100 * n_stars:
        attempts += 1
        x = rng.uniform(border, w - 1 - border)
        y = rng.uniform(border, h - 1 - border)
        if min_sep2 > 0.0 and count > 0:
            d2 = (xs[:count] - x) ** 2 + (ys[:count] - y) ** 2
            if d2.min() < min_sep2:
                continue
        xs[count], ys[count] = x, y
        count += 1
    return np.column_stack([xs[:count], ys[:count]]), fluxes[:count]


def peak_near(image, xy, radius: int):
    x, y = xy
    win = image[y - radius : y + radius + 1, x - radius : x + radius + 1]
    iy, ix = np.unravel_index(int(np.argmax(win)), win.shape)
    return float(win[iy, ix]), (x - radius + int(ix), y - radius + int(iy))


def aperture_flux(image, xy, radius: int) -> float:
    x, y = xy
    ys, xs = np.mgrid[-radius : radius + 1, -radius : radius + 1]
    disk = xs**2 + ys**2 <= radius**2
    win = image[y - radius : y + radius + 1, x - radius : x + radius + 1]
    return float(np.asarray(win, dtype=np.float64)[disk].sum())


def completeness(score, positions, threshold: float, radius: int = 3) -> NDArray[np.bool_]:
    return np.array([peak_near(score, xy, radius)[0] >= threshold for xy in positions], dtype=bool)


# ---------------------------------------------------------------------------
# Benchmark-configuration synthesizers
# ---------------------------------------------------------------------------


def moffat_alpha(fwhm: float, beta: float) -> float:
    """Moffat core width alpha for a given FWHM: FWHM = 2 alpha sqrt(2^(1/beta) - 1)."""
    return fwhm / (2.0 * np.sqrt(2.0 ** (1.0 / beta) - 1.0))


def render_psf_field(shape, positions, fluxes, fwhm_fn, kind: str = "gaussian", beta: float = 3.0,
                     q: float = 1.0, pa_deg: float = 0.0, box: float = 5.0) -> NDArray[np.float64]:
    """Render point sources whose PSF FWHM may vary with position.

    kind "gaussian": circular Gaussian; kind "moffat": elliptical Moffat with
    axis ratio q and position angle pa_deg (major-axis FWHM = fwhm_fn(x, y)).
    Each source is drawn within a box of ``box * FWHM`` (unit-flux normalised
    analytically, so truncation loses only the far wings).
    """
    h, w = shape
    out = np.zeros((h, w), dtype=np.float64)
    c, s = np.cos(np.deg2rad(pa_deg)), np.sin(np.deg2rad(pa_deg))
    for (x, y), f in zip(positions, fluxes, strict=True):
        fw = float(fwhm_fn(x, y))
        rad = int(np.ceil(box * fw))
        ix, iy = int(round(x)), int(round(y))
        x0, x1 = max(0, ix - rad), min(w, ix + rad + 1)
        y0, y1 = max(0, iy - rad), min(h, iy + rad + 1)
        if x0 >= x1 or y0 >= y1:
            continue
        ys, xs = np.mgrid[y0:y1, x0:x1]
        dx, dy = xs - x, ys - y
        if kind == "gaussian":
            sig = fw * FWHM_TO_SIGMA
            out[y0:y1, x0:x1] += f / (2 * np.pi * sig**2) * np.exp(-(dx**2 + dy**2) / (2 * sig**2))
        else:
            a = moffat_alpha(fw, beta)
            u = (c * dx + s * dy) / a
            v = (-s * dx + c * dy) / (a * q)
            norm = (beta - 1.0) / (np.pi * a * a * q)
            out[y0:y1, x0:x1] += f * norm * (1.0 + u * u + v * v) ** (-beta)
    return out


@dataclass
class SyntheticPair:
    """A seeded science/reference pair in ADU with variance and mask layers."""

    science: NDArray[np.float32]
    reference: NDArray[np.float32]
    science_var: NDArray[np.float32]
    reference_var: NDArray[np.float32]
    science_mask: NDArray[np.uint8]
    reference_mask: NDArray[np.uint8]
    star_xy: NDArray[np.float64]
    star_flux: NDArray[np.float64]
    transient_xy: NDArray[np.float64] = field(default_factory=lambda: np.zeros((0, 2)))
    transient_flux: NDArray[np.float64] = field(default_factory=lambda: np.zeros(0))
    saturation: float = 0.0
    meta: dict = field(default_factory=dict)


def synthetic_pair(width: int, height: int, n_stars: int, seed: int = 0, *,
                   flux_range=(1e3, 1e6), slope: float = 2.5, sky_e: float = 500.0, gain: float = 1.5,
                   read_noise_e: float = 4.0, ref_fwhm: float = 2.5, sci_fwhm=3.5,
                   sci_kind: str = "gaussian", moffat_beta: float = 3.0, moffat_q: float = 0.85,
                   moffat_pa: float = 30.0, mask_fraction: float = 0.01, n_transients: int = 0,
                   transient_snr=(5.0, 50.0), saturation_e: float | None = None, science_shift=(0.0, 0.0),
                   science_scale: float = 1.0) -> SyntheticPair:
    """Seeded pair for the benchmark configurations.

    Fluxes in e- follow dN/dF ~ F^-slope on flux_range; images are rendered in
    e- (sky + sources), Poisson + Gaussian read noise drawn, then converted to
    ADU = e-/gain. Variance (ADU^2) = max(signal_e, 0)/gain^2 + (rn/gain)^2 --
    the reference's synth_variance(data, gain, rn/gain). ``sci_fwhm`` may be a
    number or a callable fwhm(x, y). Masks: random bad columns (kMaskBad = 1)
    covering about ``mask_fraction`` of the pixels with saturated cores
    (kMaskSaturated = 2) flagged where a source exceeds the saturation level
    (values clipped there). ``science_shift`` = (dx, dy) renders the science
    sources displaced by that many pixels and ``science_scale`` multiplies the
    whole science frame (sky and sources, before noise): a misregistered,
    photometrically scaled exposure of the same field.
    """
    rng = np.random.default_rng(seed)
    shape = (height, width)
    pos, flux = sample_starfield(shape, n_stars, rng, flux_range=flux_range, slope=slope, border=8)
    fw_fn = sci_fwhm if callable(sci_fwhm) else (lambda x, y, f=float(sci_fwhm): f)
    ref_e = sky_e + render_psf_field(shape, pos, flux, lambda x, y: ref_fwhm, "gaussian")
    shift = np.asarray(science_shift, np.float64).reshape(1, 2)
    sci_e = sky_e + render_psf_field(shape, pos + shift, flux, fw_fn, sci_kind, beta=moffat_beta, q=moffat_q,
                                     pa_deg=moffat_pa)
    t_xy = np.zeros((0, 2))
    t_flux = np.zeros(0)
    if n_transients > 0:
        border = 24
        t_xy = np.column_stack([rng.uniform(border, width - 1 - border, n_transients),
                                rng.uniform(border, height - 1 - border, n_transients)])
        snr = np.exp(rng.uniform(np.log(transient_snr[0]), np.log(transient_snr[1]), n_transients))
        sig_bg = np.sqrt(sky_e + read_noise_e**2)
        t_flux = np.empty(n_transients)
        for i, (x, y) in enumerate(t_xy):
            fwt = float(fw_fn(x, y))
            sig = fwt * FWHM_TO_SIGMA
            # S/N of optimal PSF photometry ~ F sqrt(sum p^2) / sigma, sum p^2 = 1/(4 pi s^2).
            t_flux[i] = snr[i] * sig_bg * np.sqrt(4.0 * np.pi) * sig
        sci_e += render_psf_field(shape, t_xy, t_flux, fw_fn, sci_kind, beta=moffat_beta, q=moffat_q,
                                  pa_deg=moffat_pa)
    sci_e = sci_e * float(science_scale)
    ref_n = rng.poisson(np.clip(ref_e, 0, None)).astype(np.float64) + rng.normal(0, read_noise_e, shape)
    sci_n = rng.poisson(np.clip(sci_e, 0, None)).astype(np.float64) + rng.normal(0, read_noise_e, shape)
    ref_adu = ref_n / gain
    sci_adu = sci_n / gain
    ref_var = (np.clip(ref_e, 0, None) + read_noise_e**2) / gain**2
    sci_var = (np.clip(sci_e, 0, None) + read_noise_e**2) / gain**2
    if saturation_e is None:
        saturation_e = 2.0e5
    sat_adu = saturation_e / gain
    smask = np.zeros(shape, np.uint8)
    rmask = np.zeros(shape, np.uint8)
    ssat = sci_adu >= sat_adu
    rsat = ref_adu >= sat_adu
    smask[ssat] |= 2
    rmask[rsat] |= 2
    sci_adu[ssat] = sat_adu
    ref_adu[rsat] = sat_adu
    n_bad = int(mask_fraction * width * height) - int(ssat.sum() + rsat.sum()) // 2
    while n_bad > 0:
        col = int(rng.integers(0, width))
        y0 = int(rng.integers(0, height))
        run = int(min(height - y0, max(16, rng.integers(height // 8, height + 1))))
        target = smask if rng.random() < 0.5 else rmask
        target[y0 : y0 + run, col] |= 1
        n_bad -= run
    return SyntheticPair(
        science=sci_adu.astype(np.float32), reference=ref_adu.astype(np.float32),
        science_var=sci_var.astype(np.float32), reference_var=ref_var.astype(np.float32),
        science_mask=smask, reference_mask=rmask, star_xy=pos, star_flux=flux, transient_xy=t_xy,
        transient_flux=t_flux, saturation=float(sat_adu),
        meta={"seed": seed, "gain": gain, "read_noise_e": read_noise_e, "sky_e": sky_e})


def config1_pair(seed: int = 0, size: int = 1024, n_stars: int = 2000) -> SyntheticPair:
    """1024^2, Gaussian PSFs FWHM 2.5 (reference) / 3.5 (science), sky 500 e-."""
    return synthetic_pair(size, size, n_stars, seed, ref_fwhm=2.5, sci_fwhm=3.5)


def config2_pair(seed: int = 0, size: int = 4096, n_stars: int = 20000, n_transients: int = 50) -> SyntheticPair:
    """4096^2 spatially varying elliptical Moffat (beta 3, q 0.85, PA 30 deg),
    science FWHM 3.0 -> 4.5 px along the (0,0) -> (W,H) diagonal, Gaussian
    FWHM 2.5 reference, 50 transients at S/N 5-50."""
    denom = 2.0 * (size - 1)

    def fwhm(x, y):
        return 3.0 + 1.5 * (x + y) / denom

    return synthetic_pair(size, size, n_stars, seed, ref_fwhm=2.5, sci_fwhm=fwhm, sci_kind="moffat",
                          n_transients=n_transients)
