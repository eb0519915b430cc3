"""Generate the golden fixtures in tests/golden/ from the reference itself.

Run in a container that has the reference tree (the default REFERENCE_DIR is
used by oracle/Makefile):

    make -C oracle ref && python tests/golden/make_golden.py

Every expected value here comes from oracle/_ref/libdelta_ref.so, i.e. the
reference's own src/basis.cpp, src/convolve.cpp, src/catalog.cpp and
src/detect.cpp compiled in place -- not from this repository's code. Inputs are
small and seeded so the .npz files stay a few hundred KB in total.
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import refbuild  # noqa: E402

OUT = Path(__file__).resolve().parent


def basis_cases():
    out = {}
    for i, (beta, n_max, r) in enumerate([(1.7, 3, 6), (0.95, 6, 8), (2.0, 4, 10), (0.6, 0, 3)]):
        out[f"params_{i}"] = np.array([beta, n_max, r], np.float64)
        out[f"basis1d_{i}"] = refbuild.basis1d(beta, n_max, r)
    rng = np.random.default_rng(3)
    img = rng.standard_normal((24, 31)).astype(np.float32)
    out["conv_image"] = img
    out["conv_params"] = np.array([1.5, 2, 5], np.float64)
    out["conv_out"] = refbuild.basis_convolve(img, 1.5, 2, 5)
    return out


def _blob(shape, x, y, peak, sigma):
    ys, xs = np.mgrid[0 : shape[0], 0 : shape[1]]
    return (peak * np.exp(-((xs - x) ** 2 + (ys - y) ** 2) / (2 * sigma**2))).astype(np.float32)


def catalog_cases():
    out = {}
    rng = np.random.default_rng(11)
    cases = []
    # 0: noise + blobs + a dipole + masked column, raster-order numbering test.
    h, w = 96, 120
    s = rng.normal(0, 1.0, (h, w)).astype(np.float32)
    for x, y, pk, sg in [(20, 15, 9.0, 1.5), (90, 12, 12.0, 2.0), (60, 50, 7.0, 1.2), (100, 80, 20.0, 2.5)]:
        s += _blob((h, w), x, y, pk, sg)
    s[40:44, 10:14] = 8.0
    s[41, 14] = -4.0
    m = np.zeros((h, w), np.uint8)
    m[70:90, 100] = 1
    m[5, 20] = 4
    cases.append((s, s * 0.5 + 1.0, m))
    # 1: U-shaped component spanning row blocks (seam stitching + numbering).
    s = np.zeros((64, 64), np.float32)
    s[10:50, 10] = 6.0
    s[10:50, 30] = 6.0
    s[49, 10:31] = 6.0
    s[5, 40:60] = 6.0
    s[20:22, 20:22] = 6.0
    cases.append((s, s.copy(), None))
    # 2: dense 8-connected noise field at a low threshold.
    s = rng.normal(0, 1.0, (80, 72)).astype(np.float32)
    cases.append((s * 2.2, s, None))
    for i, (score, diff, mask) in enumerate(cases):
        out[f"score_{i}"] = score
        out[f"diff_{i}"] = diff
        if mask is not None:
            out[f"mask_{i}"] = mask
        for pol in (0, 1):
            cat = refbuild.build_catalog(score, diff, mask=mask, threshold_sigma=5.0, threshold_sigma_dipole=3.0,
                                         expected_fwhm=3.0, return_negative=bool(pol))
            for k, v in cat.items():
                out[f"cat{pol}_{i}_{k}"] = v
        seed = np.isfinite(score) & (score >= np.float32(5.0))
        if mask is not None:
            seed &= mask == 0
        labels, n = refbuild.label_components(seed.astype(np.uint8))
        out[f"labels_{i}"] = labels
    return out


def detect_cases():
    out = {}
    rng = np.random.default_rng(5)
    h = w = 160
    pos = np.array([[30.0, 30.0], [80.0, 40.0], [120.0, 110.0], [50.0, 120.0], [130.0, 30.0], [60.0, 75.0]])
    flux = np.array([5e4, 3e4, 8e4, 2e4, 4e4, 1e4])
    ys, xs = np.mgrid[0:h, 0:w]
    ref = np.full((h, w), 100.0)
    sci = np.full((h, w), 100.0)
    for (x, y), f in zip(pos, flux):
        ref += f / (2 * np.pi * 1.5**2) * np.exp(-((xs - x) ** 2 + (ys - y) ** 2) / (2 * 1.5**2))
        sci += f / (2 * np.pi * 2.2**2) * np.exp(-((xs - x) ** 2 + (ys - y) ** 2) / (2 * 2.2**2))
    ref = (ref + rng.normal(0, 3, (h, w))).astype(np.float32)
    sci = (sci + rng.normal(0, 3, (h, w))).astype(np.float32)
    out["sci"], out["ref"] = sci, ref
    sel = refbuild.select_stamps(sci, ref, stamp_radius=8, threshold_sigma=5.0, max_stamps=20)
    for k, v in sel.items():
        out[f"sel_{k}"] = np.asarray(v)
    out["bg_sci"] = np.array(refbuild.estimate_background(sci))
    return out


def main():
    if not refbuild.available():
        raise SystemExit("oracle/_ref/libdelta_ref.so missing: run `make -C oracle ref` with the reference tree")
    np.savez_compressed(OUT / "basis.npz", **basis_cases())
    np.savez_compressed(OUT / "catalog.npz", **catalog_cases())
    sel = detect_cases()
    sel["sel_direction"] = np.array(sel["sel_direction"] == "reference")
    np.savez_compressed(OUT / "detect.npz", **sel)
    for p in sorted(OUT.glob("*.npz")):
        print(p.name, p.stat().st_size)


if __name__ == "__main__":
    main()
