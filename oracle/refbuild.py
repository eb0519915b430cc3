"""Loader for oracle/_ref/libdelta_ref.so -- TEST INFRASTRUCTURE ONLY.

The library is the reference's own src/basis.cpp, src/convolve.cpp,
src/catalog.cpp, src/detect.cpp and src/timing.cpp compiled in place by
oracle/Makefile (see oracle/ref_wrap.cpp). ``available()`` is False when it was
never built (e.g. no reference tree was present at build time).
"""

from __future__ import annotations

import ctypes

import numpy as np

from ._loader import HERE, f32, f64, i32, ptr, u8

_LIB_PATH = HERE / "_ref" / "libdelta_ref.so"
_lib = None

CATALOG_COLUMNS = [
    ("x", np.float64), ("y", np.float64), ("peak_x", np.int32), ("peak_y", np.int32),
    ("peak_snr", np.float64), ("n_pix", np.int32), ("flux", np.float64),
    ("expected_n_pix", np.float64), ("fwhm_ratio", np.float64), ("fwhm_consistent", np.uint8),
    ("mask_flags", np.uint8), ("is_dipole", np.uint8), ("quality", np.uint8),
    ("psf_chi2", np.float64), ("psf_chi2_dof", np.int32), ("psf_amplitude", np.float64),
    ("psf_amplitude_err", np.float64), ("shape_consistent", np.uint8),
    ("bright_star_dist", np.float64), ("near_bright_star", np.uint8),
]


def available() -> bool:
    return _LIB_PATH.exists()


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"{_LIB_PATH} not built (make -C oracle ref)")
        _lib = ctypes.CDLL(str(_LIB_PATH))
        _lib.ref_build_catalog.restype = ctypes.c_int
        _lib.ref_select_stamps.restype = ctypes.c_int
    return _lib


def basis1d(beta: float, n_max: int, radius: int) -> np.ndarray:
    out = np.zeros((n_max + 1, 2 * radius + 1))
    rc = lib().ref_basis1d(ctypes.c_double(beta), n_max, radius, ptr(out))
    if rc:
        raise ValueError("invalid basis parameters")
    return out


def basis_convolve(img, beta: float, n_max: int, radius: int) -> np.ndarray:
    img = f32(img)
    h, w = img.shape
    nc = (n_max + 1) * (n_max + 2) // 2
    out = np.zeros((nc, h, w), np.float32)
    rc = lib().ref_basis_convolve(ptr(img), w, h, ctypes.c_double(beta), n_max, radius, ptr(out))
    if rc:
        raise ValueError("basis_convolve failed")
    return out


def label_components(seed) -> tuple[np.ndarray, int]:
    seed = u8(seed)
    h, w = seed.shape
    labels = np.zeros((h, w), np.int32)
    n = lib().ref_label_components(ptr(seed), w, h, ptr(labels))
    return labels, int(n)


def build_catalog(score, difference, mask=None, threshold_sigma=5.0, threshold_sigma_dipole=3.0,
                  expected_fwhm=3.5, fwhm_tolerance_lo=0.3, fwhm_tolerance_hi=3.0, aperture_radius=0,
                  exclude_bad_pixels=True, return_negative=False, fit_psf_shape=False,
                  shape_chi2_tolerance=3.0, variance=None, psf=None, bright_star_radius=0.0,
                  max_shape_fit=5000, bright_x=None, bright_y=None) -> dict:
    score, difference = f32(score), f32(difference)
    mask, variance, psf = u8(mask), f32(variance), f32(psf)
    bx, by = f64(bright_x), f64(bright_y)
    h, w = score.shape
    cap = 16
    while True:
        cols = {name: np.zeros(cap, dt) for name, dt in CATALOG_COLUMNS}
        n = lib().ref_build_catalog(
            ptr(score), ptr(difference), ptr(mask), w, h, ctypes.c_double(threshold_sigma),
            ctypes.c_double(threshold_sigma_dipole), ctypes.c_double(expected_fwhm),
            ctypes.c_double(fwhm_tolerance_lo), ctypes.c_double(fwhm_tolerance_hi), int(aperture_radius),
            int(bool(exclude_bad_pixels)), int(bool(return_negative)), int(bool(fit_psf_shape)),
            ctypes.c_double(shape_chi2_tolerance), ptr(variance), ptr(psf),
            0 if psf is None else psf.shape[0], ctypes.c_double(bright_star_radius), int(max_shape_fit),
            ptr(bx), ptr(by), 0 if bx is None else bx.size, cap,
            *[ptr(cols[name]) for name, _ in CATALOG_COLUMNS])
        if n < 0:
            raise RuntimeError("reference build_catalog failed")
        if n <= cap:
            return {name: cols[name][:n].copy() for name, _ in CATALOG_COLUMNS}
        cap = n


def estimate_background(data, mask=None) -> tuple[float, float]:
    data, mask = f32(data), u8(mask)
    h, w = data.shape
    med, sig = ctypes.c_double(), ctypes.c_double()
    lib().ref_estimate_background(ptr(data), ptr(mask), w, h, ctypes.byref(med), ctypes.byref(sig))
    return med.value, sig.value


def select_stamps(science, reference, science_mask=None, reference_mask=None, catalog_x=None,
                  catalog_y=None, stamp_radius=15, threshold_sigma=5.0, max_stamps=200, saturation=0.0,
                  isolation_radius=0, border=0, fwhm_radius=0, match_radius=2) -> dict:
    s, r = f32(science), f32(reference)
    sm, rm = u8(science_mask), u8(reference_mask)
    cx, cy = i32(catalog_x), i32(catalog_y)
    h, w = s.shape
    cap = max(max_stamps, 0 if cx is None else cx.size) + 1
    ox, oy = np.zeros(cap, np.int32), np.zeros(cap, np.int32)
    fs, fr = np.zeros(cap), np.zeros(cap)
    ms, mr = ctypes.c_double(), ctypes.c_double()
    dref = ctypes.c_int()
    n = lib().ref_select_stamps(
        ptr(s), ptr(r), ptr(sm), ptr(rm), w, h, ptr(cx), ptr(cy), 0 if cx is None else cx.size,
        stamp_radius, ctypes.c_double(threshold_sigma), max_stamps, ctypes.c_double(saturation),
        isolation_radius, border, fwhm_radius, match_radius, cap, ptr(ox), ptr(oy), ptr(fs), ptr(fr),
        ctypes.byref(ms), ctypes.byref(mr), ctypes.byref(dref))
    if n < 0:
        raise RuntimeError("reference select_stamps failed")
    return {"x": ox[:n].copy(), "y": oy[:n].copy(), "fwhm_science": fs[:n].copy(),
            "fwhm_reference": fr[:n].copy(), "median_fwhm_science": ms.value,
            "median_fwhm_reference": mr.value, "direction": "reference" if dref.value else "science"}
