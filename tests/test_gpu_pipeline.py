"""GPU stamp selection, PSF estimate and the end-to-end pipeline.

Stamp selection is checked against the reference-built detect.cpp
(oracle/_ref) and its golden fixture; the pipeline against the reference's own
statistical assertions (tests/test_pipeline.py of tkillestein/delta) and, stage
by stage, against the oracle chain on the same inputs."""

from __future__ import annotations

import numpy as np
import pytest
from conftest import load_golden

import delta_b200 as delta
from delta_b200 import _core, validation
from oracle import cref, refbuild
from oracle import numpy_ref as nr

pytestmark = pytest.mark.gpu


def _stars(h, w, positions, total, sigma):
    img = np.zeros((h, w), np.float64)
    ys, xs = np.mgrid[0:h, 0:w]
    amp = total / (2 * np.pi * sigma**2)
    for x, y in positions:
        img += amp * np.exp(-((xs - x) ** 2 + (ys - y) ** 2) / (2 * sigma**2))
    return img, amp


def _pair(sig_ref, sig_sci, transient_xy=(60, 140), seed=0):
    h = w = 200
    rng = np.random.default_rng(seed)
    grid = [(x, y) for x in (40, 80, 120, 160) for y in (40, 80, 120, 160)]
    ref, _ = _stars(h, w, grid, total=12000.0, sigma=sig_ref)
    sci, _ = _stars(h, w, grid, total=12000.0, sigma=sig_sci)
    trans, amp_t = _stars(h, w, [transient_xy], total=6000.0, sigma=sig_sci)
    sci = sci + trans
    ref = ref + 100.0 + rng.normal(0, 3.0, (h, w))
    sci = sci + 100.0 + rng.normal(0, 3.0, (h, w))
    return ref.astype(np.float32), sci.astype(np.float32), amp_t


def _window_max(img, xy, r=8):
    x, y = xy
    return img[y - r : y + r + 1, x - r : x + r + 1].max()


# --------------------------------------------------------------- stamp selection


def test_background_and_selection_match_reference_golden():
    g = load_golden("detect")
    med, sig = _core.estimate_background(g["sci"])
    np.testing.assert_allclose([med, sig], g["bg_sci"], rtol=0, atol=0)
    sel = _core.select_stamps(g["sci"], g["ref"], stamp_radius=8, threshold_sigma=5.0, max_stamps=20)
    np.testing.assert_array_equal(sel["x"], g["sel_x"])
    np.testing.assert_array_equal(sel["y"], g["sel_y"])
    np.testing.assert_allclose(sel["fwhm_science"], g["sel_fwhm_science"], rtol=1e-12)
    np.testing.assert_allclose(sel["fwhm_reference"], g["sel_fwhm_reference"], rtol=1e-12)
    assert (sel["direction"] == "reference") == bool(g["sel_direction"])


@pytest.mark.parametrize("seed,size,n_star,max_stamps", [(0, 512, 300, 200), (1, 1024, 2000, 200),
                                                         (2, 700, 900, 50)])
def test_select_stamps_matches_reference(seed, size, n_star, max_stamps):
    if not refbuild.available():
        pytest.skip("reference library not built")
    p = validation.synthetic_pair(size, size, n_star, seed, mask_fraction=0.005)
    kw = dict(stamp_radius=12, threshold_sigma=5.0, max_stamps=max_stamps, saturation=p.saturation)
    got = _core.select_stamps(p.science, p.reference, p.science_mask, p.reference_mask, **kw)
    want = refbuild.select_stamps(p.science, p.reference, p.science_mask, p.reference_mask, **kw)
    np.testing.assert_array_equal(got["x"], want["x"])
    np.testing.assert_array_equal(got["y"], want["y"])
    np.testing.assert_allclose(got["fwhm_science"], want["fwhm_science"], rtol=1e-12)
    assert got["direction"] == want["direction"]
    for k in ("median_fwhm_science", "median_fwhm_reference"):
        np.testing.assert_allclose(got[k], want[k], rtol=1e-12)
    # catalog-supplied positions
    cx = np.asarray(want["x"][:40], np.int32)
    cy = np.asarray(want["y"][:40], np.int32)
    got_c = _core.select_stamps(p.science, p.reference, p.science_mask, p.reference_mask, cx, cy, **kw)
    want_c = refbuild.select_stamps(p.science, p.reference, p.science_mask, p.reference_mask, cx, cy, **kw)
    np.testing.assert_array_equal(got_c["x"], want_c["x"])
    np.testing.assert_allclose(got_c["fwhm_reference"], want_c["fwhm_reference"], rtol=1e-12)


def test_estimate_psf_and_weighted_mean():
    p = validation.synthetic_pair(400, 400, 120, 3)
    sel = _core.select_stamps(p.science, p.reference, stamp_radius=10)
    for r in (8, 5):
        got = _core.estimate_psf(p.science, sel["x"], sel["y"], r)
        np.testing.assert_allclose(got, nr.estimate_psf(p.science, sel["x"], sel["y"], r), rtol=1e-6, atol=1e-9)
    with pytest.raises(ValueError):
        _core.estimate_psf(p.science, np.array([0]), np.array([0]), 8)
    d = p.science.astype(np.float64)
    v = p.science_var.astype(np.float64)
    m = p.science_mask
    good = (m == 0) & (v > 0)
    want = np.sum(d[good] / v[good]) / np.sum(1.0 / v[good])
    np.testing.assert_allclose(_core.weighted_mean(p.science, p.science_var, m), want, rtol=1e-12)


# ---------------------------------------------------------------------- pipeline


def test_subtract_removes_statics_keeps_transient_reference_sharper():
    ref, sci, amp_t = _pair(sig_ref=1.6, sig_sci=2.4)
    res = delta.subtract(sci, ref, gain=1.5, read_noise=4.0, n_knots=4, stamp_radius=12)
    assert isinstance(res, delta.DiffResult)
    assert res.solution.direction == "reference"
    assert np.isfinite(res.solution.gcv)
    assert np.abs(_window_max(res.difference, (80, 80))) < 0.25 * amp_t
    assert _window_max(res.difference, (60, 140)) > 0.4 * amp_t


def test_direction_flips_when_science_sharper():
    ref, sci, amp_t = _pair(sig_ref=2.4, sig_sci=1.6)
    res = delta.subtract(sci, ref, gain=1.5, read_noise=4.0, n_knots=4, stamp_radius=12)
    assert res.solution.direction == "science"
    assert _window_max(res.difference, (60, 140)) > 0.3 * amp_t


def test_score_catalog_decorrelate_and_solution_roundtrip(tmp_path):
    ref, sci, amp_t = _pair(sig_ref=1.6, sig_sci=2.4, seed=4)
    sub = delta.Subtractor(n_knots=3, stamp_radius=12, score=True, decorrelate=True, block=64, cv_folds=0)
    res = sub.subtract(sci, ref, gain=1.5, read_noise=4.0)
    assert res.score is not None and res.psf is not None
    assert res.source_catalog is not None
    assert np.any(np.hypot(res.source_catalog["x"] - 60, res.source_catalog["y"] - 140) < 3)
    path = tmp_path / "sol.npz"
    res.solution.save(str(path))
    sol = delta.KernelSolution.load(str(path))
    again = sub.apply(sol, sci, ref, gain=1.5, read_noise=4.0)
    np.testing.assert_array_equal(again.difference, res.difference)
    cat2 = res.build_catalog(threshold_sigma=4.0, polarity="both")
    assert "sign" in cat2.dtype.names


@pytest.mark.parametrize("cv_folds", [0, 5])
def test_pipeline_stages_match_oracle_chain(cv_folds):
    """Stage-by-stage: the device pipeline on one 384x384 frame (n_max 4, radius 10, 3x3 knots) vs the oracle
    fed the same stamps (fit -> subtract -> score -> catalog)."""
    p = validation.synthetic_pair(384, 384, 220, 7, mask_fraction=0.005)
    kw = dict(n_max=4, radius=10, n_knots=3, stamp_radius=12, cv_folds=cv_folds, score=True, decorrelate=False,
              saturation=p.saturation)
    res = delta.subtract(p.science, p.reference, science_var=p.science_var, reference_var=p.reference_var,
                         science_mask=p.science_mask, reference_mask=p.reference_mask, **kw)
    sol = res.solution
    assert sol.direction == "reference"
    sel = _core.select_stamps(p.science, p.reference, p.science_mask, p.reference_mask, stamp_radius=12,
                              saturation=p.saturation)
    knots = nr.grid_knots(0, 0, 383, 383, 3, 3)
    bconv = (lambda patch: refbuild.basis_convolve(patch, sol.beta, 4, 10)) if refbuild.available() else None
    fit = nr.fit_kernel(p.science, p.reference, knots, sel["x"], sel["y"], 12, sol.beta, 4, np.logspace(-6, 6, 25),
                        radius=10, cv_folds=cv_folds, science_var=p.science_var, reference_var=p.reference_var,
                        science_mask=p.science_mask, reference_mask=p.reference_mask, basis_convolve_fn=bconv)
    assert fit["lambda"] == sol.lam
    np.testing.assert_allclose(sol.theta, fit["theta"], rtol=1e-6, atol=1e-9 * np.abs(fit["theta"]).max())
    sub = cref.subtract(p.science, p.reference, knots, sol.theta, sol.beta, 4, 10, p.saturation, p.science_var,
                        p.reference_var, p.science_mask, p.reference_mask)
    assert np.array_equal(res.mask, sub["mask"])
    pos = sub["variance"] > 0
    assert np.max(np.abs(res.difference - sub["difference"])[pos] / np.sqrt(sub["variance"][pos])) < 1e-3
    np.testing.assert_allclose(res.psf, nr.estimate_psf(p.science, sel["x"], sel["y"], 8), rtol=1e-6, atol=1e-9)
    score = cref.matched_filter(res.difference, res.psf, res.variance)
    np.testing.assert_array_equal(res.score, score)


@pytest.mark.parametrize("direction", [None, "science"])
def test_device_resident_path_matches_host_staged(direction):
    """The HBM-resident stage chain (one upload) gives the same bits as the
    per-call host-staged chain: same kernels, same inputs."""
    p = validation.synthetic_pair(384, 384, 220, 7, mask_fraction=0.005)
    kw = dict(n_max=4, radius=10, n_knots=3, stamp_radius=12, cv_folds=0, score=True, decorrelate=True, block=64,
              saturation=p.saturation, direction=direction)
    layers = dict(science_var=p.science_var, reference_var=p.reference_var, science_mask=p.science_mask,
                  reference_mask=p.reference_mask)
    a = delta.subtract(p.science, p.reference, device_resident=True, **layers, **kw)
    b = delta.subtract(p.science, p.reference, device_resident=False, **layers, **kw)
    assert a.solution.direction == b.solution.direction
    np.testing.assert_array_equal(a.solution.theta, b.solution.theta)
    for name in ("difference", "variance", "mask", "score", "psf"):
        np.testing.assert_array_equal(getattr(a, name), getattr(b, name), err_msg=name)
    assert a.source_catalog.dtype == b.source_catalog.dtype
    np.testing.assert_array_equal(a.source_catalog, b.source_catalog)
    again = delta.apply(a.solution, p.science, p.reference, device_resident=True, **layers,
                        **{k: v for k, v in kw.items() if k != "direction"})
    np.testing.assert_array_equal(again.difference, a.difference)


@pytest.mark.parametrize("size", [1024, 2048])
def test_strided_background_and_selection_match_reference(size):
    """Frames above 2^18 px take the strided background sample (step n / 2^18,
    src/detect.cpp:96-106); selection must still equal the reference's."""
    if not refbuild.available():
        pytest.skip("oracle/_ref not built")
    scale = (size / 4096.0) ** 2
    p = validation.config2_pair(seed=3, size=size, n_stars=int(20000 * scale), n_transients=2)
    for img, m in ((p.science, p.science_mask), (p.reference, p.reference_mask)):
        assert _core.estimate_background(img, m) == refbuild.estimate_background(img, m)
    kw = dict(stamp_radius=15, threshold_sigma=5.0, max_stamps=200, saturation=p.saturation)
    got = _core.select_stamps(p.science, p.reference, p.science_mask, p.reference_mask, **kw)
    want = refbuild.select_stamps(p.science, p.reference, p.science_mask, p.reference_mask, **kw)
    np.testing.assert_array_equal(got["x"], want["x"])
    np.testing.assert_array_equal(got["y"], want["y"])
    np.testing.assert_allclose(got["fwhm_science"], want["fwhm_science"], rtol=1e-12)
    assert got["direction"] == want["direction"]


def test_device_resident_large_frame_matches_host_staged():
    """2048^2 frame: large enough that an upload left unordered against the
    library's stream would be caught."""
    p = validation.config2_pair(seed=5, size=2048, n_stars=5000, n_transients=12)
    kw = dict(n_knots=4, cv_folds=0, decorrelate=True, score=True, saturation=p.saturation, precision="mixed")
    layers = dict(science_var=p.science_var, reference_var=p.reference_var, science_mask=p.science_mask,
                  reference_mask=p.reference_mask)
    a = delta.subtract(p.science, p.reference, device_resident=True, **layers, **kw)
    b = delta.subtract(p.science, p.reference, device_resident=False, **layers, **kw)
    np.testing.assert_array_equal(a.solution.theta, b.solution.theta)
    for name in ("difference", "variance", "mask", "score"):
        np.testing.assert_array_equal(getattr(a, name), getattr(b, name), err_msg=name)
    np.testing.assert_array_equal(a.source_catalog, b.source_catalog)


def test_subtract_batch_matches_one_at_a_time():
    """Frames in flight on their own threads, contexts and streams give the same
    bits as subtracting them one after another."""
    ps = [validation.synthetic_pair(512, 512, 300, s, mask_fraction=0.005) for s in (21, 22, 23)]
    kw = dict(n_max=4, n_knots=3, stamp_radius=12, cv_folds=0, score=True, decorrelate=True, block=64,
              precision="mixed", saturation=ps[0].saturation)
    items = [dict(science=p.science, reference=p.reference, science_var=p.science_var,
                  reference_var=p.reference_var, science_mask=p.science_mask, reference_mask=p.reference_mask)
             for p in ps]
    batch = delta.subtract_batch(items, max_in_flight=3, **kw)
    assert len(batch) == len(ps)
    for it, r in zip(items, batch, strict=True):
        one = delta.subtract(**it, **kw)
        np.testing.assert_array_equal(r.solution.theta, one.solution.theta)
        for name in ("difference", "variance", "mask", "score"):
            np.testing.assert_array_equal(getattr(r, name), getattr(one, name), err_msg=name)
        np.testing.assert_array_equal(r.source_catalog, one.source_catalog)


def test_batch_from_pageable_and_pinned_arrays_gives_the_same_bits():
    """Pageable layers of 1 MB or more are staged into pinned memory by several
    host threads before their ordered upload; pinned layers go as they are. Both
    give the same bits, and the layers' host arrays may be dropped as soon as
    the call returns."""
    import torch

    ps = [validation.synthetic_pair(1024, 1024, 1500, s, mask_fraction=0.005) for s in (31, 32)]
    kw = dict(n_max=4, n_knots=3, stamp_radius=12, cv_folds=0, score=True, decorrelate=True, block=256,
              precision="mixed", saturation=ps[0].saturation)
    names = ("science", "reference", "science_var", "reference_var", "science_mask", "reference_mask")

    def pinned(a):
        t = torch.empty(a.shape, dtype=torch.from_numpy(a[:1].copy()).dtype, pin_memory=True)
        out = t.numpy()
        out[...] = a
        return out

    page = [{k: np.array(getattr(p, k), copy=True) for k in names} for p in ps]
    pin = [{k: pinned(getattr(p, k)) for k in names} for p in ps]
    a = delta.subtract_batch(page, max_in_flight=2, **kw)
    del page
    b = delta.subtract_batch(pin, max_in_flight=2, **kw)
    for ra, rb in zip(a, b, strict=True):
        np.testing.assert_array_equal(ra.solution.theta, rb.solution.theta)
        for name in ("difference", "variance", "mask", "score"):
            np.testing.assert_array_equal(getattr(ra, name), getattr(rb, name), err_msg=name)
        np.testing.assert_array_equal(ra.source_catalog, rb.source_catalog)


def test_apply_batch_matches_one_at_a_time():
    """One frozen solution applied to several frame pairs in flight gives the
    same bits as apply() on each pair alone."""
    ps = [validation.synthetic_pair(512, 512, 300, s, mask_fraction=0.005) for s in (31, 32, 33)]
    kw = dict(n_max=4, n_knots=3, stamp_radius=12, cv_folds=0, score=True, decorrelate=True, block=64,
              precision="mixed", saturation=ps[0].saturation)
    items = [dict(science=p.science, reference=p.reference, science_var=p.science_var,
                  reference_var=p.reference_var, science_mask=p.science_mask, reference_mask=p.reference_mask)
             for p in ps]
    solution = delta.subtract(**items[0], **kw).solution
    batch = delta.apply_batch(solution, items, max_in_flight=3, **kw)
    assert len(batch) == len(ps)
    for it, r in zip(items, batch, strict=True):
        one = delta.apply(solution, **it, **kw)
        np.testing.assert_array_equal(r.solution.theta, solution.theta)
        for name in ("difference", "variance", "mask", "score"):
            np.testing.assert_array_equal(getattr(r, name), getattr(one, name), err_msg=name)
        np.testing.assert_array_equal(r.source_catalog, one.source_catalog)


def test_copy_to_host_orders_on_the_stream():
    """dgpu_copy_to_host copies device bytes into pinned host memory after the
    stream's queued work (ragged sizes included) and rejects pageable
    destinations."""
    import ctypes

    import torch

    from delta_b200 import _device, _lib

    ctx = _device._ctx_on_torch_stream()
    for n in (0, 16, 1000, 4 * 1024 * 1024 + 3, 3 * (4 << 20) + 5):
        src = torch.randint(0, 256, (n,), dtype=torch.uint8, device="cuda")
        src.add_(1)  # queued on the stream just before the copy, which must see it
        dst = torch.zeros(n, dtype=torch.uint8, pin_memory=True)
        _lib.check(_lib.lib().dgpu_copy_to_host(ctx.handle, ctypes.c_void_p(dst.data_ptr()),
                                                ctypes.c_void_p(src.data_ptr()), ctypes.c_int64(n)), ctx.handle)
        torch.cuda.current_stream().synchronize()
        assert torch.equal(dst, src.cpu())
    src = torch.ones(64, dtype=torch.float32, device="cuda")
    pageable = np.zeros(64, np.float32)
    with pytest.raises(ValueError):
        _lib.check(_lib.lib().dgpu_copy_to_host(ctx.handle, ctypes.c_void_p(pageable.ctypes.data),
                                                ctypes.c_void_p(src.data_ptr()), ctypes.c_int64(256)), ctx.handle)


def test_mixed_precision_falls_back_on_an_ill_conditioned_fit():
    """A frame whose PSFs nearly match drives beta to its 0.5 floor: the fit's
    theta then carries large cancelling terms (|theta| ~ 600 for a unit
    kernel), and the BF16x3 normal equations cannot resolve it. The mixed fit
    must fall back to FP64 and give the FP64 pipeline's products bit for bit."""
    import bench

    sp = bench.uneven_specs(0)[4]  # 2048 x 2048, science FWHM 2.1 px vs 2.5 px reference, 2.2% masked
    p = validation.synthetic_pair(sp["width"], sp["height"], sp["n_stars"], sp["seed"], sci_fwhm=sp["sci_fwhm"],
                                  mask_fraction=sp["mask_fraction"])
    layers = dict(science_var=p.science_var, reference_var=p.reference_var, science_mask=p.science_mask,
                  reference_mask=p.reference_mask)
    seen = {}
    fit_kernel = _core.fit_kernel

    def spy(*a, **k):
        r = fit_kernel(*a, **k)
        seen[k.get("precision", "fp64")] = r["precision_used"]
        return r

    _core.fit_kernel = spy
    try:
        sol_mixed = delta.Subtractor(**bench.subtract_kwargs(p, "mixed")).fit(p.science, p.reference, **layers)
    finally:
        _core.fit_kernel = fit_kernel
    assert seen == {"mixed": "fp64"}
    assert sol_mixed.beta == 0.5 and np.all(np.isfinite(sol_mixed.theta))
    a = delta.subtract(p.science, p.reference, **layers, **bench.subtract_kwargs(p, "mixed"))
    b = delta.subtract(p.science, p.reference, **layers, **bench.subtract_kwargs(p, "fp64"))
    np.testing.assert_array_equal(a.solution.theta, b.solution.theta)
    for name in ("difference", "variance", "mask", "score"):
        np.testing.assert_array_equal(getattr(a, name), getattr(b, name), err_msg=name)
    assert float(np.max(a.psf)) > 0.0 and len(a.source_catalog) == len(b.source_catalog)


def _uneven_vs_chain(spec_index):
    import bench
    from oracle import chain

    if not chain.available():
        pytest.skip("oracle/_ref is not built")
    sp = bench.uneven_specs(0)[spec_index]
    p = validation.synthetic_pair(sp["width"], sp["height"], sp["n_stars"], sp["seed"], sci_fwhm=sp["sci_fwhm"],
                                  mask_fraction=sp["mask_fraction"])
    kw = bench.subtract_kwargs(p, "fp64")
    res = delta.subtract(p.science, p.reference, science_var=p.science_var, reference_var=p.reference_var,
                         science_mask=p.science_mask, reference_mask=p.reference_mask, **kw)
    kw.pop("saturation")
    kw.pop("precision")
    want = chain.run(p.science, p.reference, p.science_var, p.reference_var, p.science_mask, p.reference_mask,
                     saturation=p.saturation, **kw)
    var = np.asarray(want["variance"], np.float64)
    pos = var > 0
    dd = np.abs(res.difference.astype(np.float64) - want["difference"])[pos] / np.sqrt(var[pos])
    return res, want, dd


@pytest.mark.parametrize("spec_index", [2, 7])
def test_uneven_frames_match_oracle_chain(spec_index):
    """Whole pipeline (FP64 fit, decorrelation, score, catalog) on frames of the
    uneven batch against the oracle chain on the same inputs: 1024 x 4096 and
    2048 x 2048. Masks bit-exact, whitened difference and score within 1e-3 of
    the local sigma, catalog sizes within one row."""
    res, want, dd = _uneven_vs_chain(spec_index)
    np.testing.assert_array_equal(res.mask, want["mask"])
    assert np.max(dd) < 1e-3
    assert np.max(np.abs(res.score.astype(np.float64) - want["score"])) < 1e-3
    assert abs(len(res.source_catalog) - len(want["catalog"]["x"])) <= 1


def test_beta_floor_frame_against_oracle_chain():
    """A frame whose fit sits at the beta floor: theta is ill-determined (about
    600 in large cancelling terms for a unit kernel), so two FP64 solvers that
    sum in different orders agree on the lambda and on |theta| to four digits
    but not on the model everywhere: measured, the difference moves by a median
    1.05e-3 sigma and at most 0.49 sigma between this solver and the oracle's.
    Masks stay bit-exact; the bounds below are 3x and 2x those figures."""
    res, want, dd = _uneven_vs_chain(4)
    np.testing.assert_array_equal(res.mask, want["mask"])
    assert np.median(dd) < 3e-3 and np.max(dd) < 1.0, (np.median(dd), np.max(dd))
    n_got, n_want = len(res.source_catalog), len(want["catalog"]["x"])
    assert abs(n_got - n_want) <= 2, (n_got, n_want)


@pytest.mark.parametrize("spec_index", [2, 7])
def test_mixed_pipeline_close_to_fp64_on_uneven_frames(spec_index):
    """The mixed-precision pipeline against the FP64 one on frames of the uneven
    batch (refinement corrections near 1e-3, so the mixed solve is kept): masks
    bit-exact, difference within 1e-3 of the local sigma, same catalog size."""
    import bench

    sp = bench.uneven_specs(0)[spec_index]
    p = validation.synthetic_pair(sp["width"], sp["height"], sp["n_stars"], sp["seed"], sci_fwhm=sp["sci_fwhm"],
                                  mask_fraction=sp["mask_fraction"])
    layers = dict(science_var=p.science_var, reference_var=p.reference_var, science_mask=p.science_mask,
                  reference_mask=p.reference_mask)
    a = delta.subtract(p.science, p.reference, **layers, **bench.subtract_kwargs(p, "mixed"))
    b = delta.subtract(p.science, p.reference, **layers, **bench.subtract_kwargs(p, "fp64"))
    assert a.solution.lam == b.solution.lam
    np.testing.assert_array_equal(a.mask, b.mask)
    pos = b.variance > 0
    dd = np.abs(a.difference.astype(np.float64) - b.difference)[pos] / np.sqrt(b.variance[pos].astype(np.float64))
    assert np.max(dd) < 1e-3, np.max(dd)
    assert len(a.source_catalog) == len(b.source_catalog)


def test_subtract_files_reads_subtracts_and_writes(tmp_path):
    """The FITS batch path: pairs read into pinned memory by their workers,
    subtracted, and written in the reference's write_fits layout; each result
    bit-identical to subtract() on the arrays read back from the files."""
    ps = [validation.synthetic_pair(384, 320, 200, s, mask_fraction=0.005) for s in (41, 42)]
    kw = dict(n_max=4, n_knots=3, stamp_radius=12, cv_folds=0, score=True, decorrelate=True, block=64,
              saturation=ps[0].saturation)
    pairs, outs = [], []
    for i, p in enumerate(ps):
        s_path, r_path = tmp_path / f"sci{i}.fits", tmp_path / f"ref{i}.fits"
        _core.write_fits(str(s_path), p.science, p.science_var, p.science_mask)
        _core.write_fits(str(r_path), p.reference, p.reference_var, p.reference_mask)
        pairs.append((s_path, r_path))
        outs.append(tmp_path / f"diff{i}.fits")
    got = delta.subtract_files(pairs, outs, max_in_flight=2, **kw)
    assert len(got) == 2
    for (s_path, r_path), o, r in zip(pairs, outs, got, strict=True):
        sci, ref = _core.read_fits(str(s_path)), _core.read_fits(str(r_path))
        one = delta.subtract(sci["data"], ref["data"], science_var=sci["variance"], reference_var=ref["variance"],
                             science_mask=sci["mask"], reference_mask=ref["mask"], **kw)
        for name in ("difference", "variance", "mask", "score"):
            np.testing.assert_array_equal(getattr(r, name), getattr(one, name), err_msg=name)
        back = _core.read_fits(str(o))
        np.testing.assert_array_equal(back["data"], r.difference)
        np.testing.assert_array_equal(back["variance"], r.variance)
        np.testing.assert_array_equal(back["mask"], r.mask)
    with pytest.raises(ValueError):
        delta.subtract_files(pairs, outs[:1], **kw)


def test_native_batch_matches_subtract_one_at_a_time():
    """dgpu_subtract_batch (the C++ scheduler: frames longest first over worker
    contexts with their own streams) gives, for frames of different sizes, the
    same bits as delta.subtract() on each frame alone: theta, lambda, the
    whitened difference, its variance, the mask, the score and the catalog."""
    ps = [validation.synthetic_pair(w, h, n, s, mask_fraction=0.005)
          for w, h, n, s in ((512, 384, 260, 61), (640, 512, 400, 62), (384, 448, 200, 63), (512, 512, 300, 64))]
    kw = dict(n_max=4, n_knots=3, stamp_radius=12, cv_folds=0, score=True, decorrelate=True, block=64,
              precision="mixed", saturation=ps[0].saturation)
    items = [dict(science=p.science, reference=p.reference, science_var=p.science_var,
                  reference_var=p.reference_var, science_mask=p.science_mask, reference_mask=p.reference_mask)
             for p in ps]
    native = _core.subtract_batch_native(items, frames_in_flight=3, catalog=True,
                                         **{k: v for k, v in kw.items() if k != "score"})
    assert len(native) == len(ps)
    for it, nat in zip(items, native, strict=True):
        one = delta.subtract(**it, **kw)
        np.testing.assert_array_equal(nat["theta"], one.solution.theta)
        assert nat["lambda"] == one.solution.lam and nat["beta"] == one.solution.beta
        assert nat["direction"] == one.solution.direction
        for name in ("difference", "variance", "mask", "score"):
            np.testing.assert_array_equal(nat[name], getattr(one, name), err_msg=name)
        for name in one.source_catalog.dtype.names:
            np.testing.assert_array_equal(nat["catalog"][name], one.source_catalog[name], err_msg=name)
    with pytest.raises(ValueError, match="no stamps selected"):
        blank = np.full((128, 128), 100.0, np.float32)
        _core.subtract_batch_native([dict(science=blank, reference=blank)], score=False, decorrelate=False)


def test_native_batch_graph_replay_gives_the_same_bits():
    """dgpu_subtract_batch with the post-fit device work recorded as CUDA graphs
    (a worker runs the first frame of a shape directly, then records and
    replays): the same bits as the direct launches, frame by frame, and the
    repeated shapes did replay."""
    shapes = ((320, 384, 51), (256, 320, 52), (320, 384, 53), (256, 320, 54), (320, 384, 55), (256, 320, 56))
    ps = [validation.synthetic_pair(w, h, 180, s, mask_fraction=0.005) for w, h, s in shapes]
    kw = dict(n_max=4, n_knots=3, stamp_radius=12, cv_folds=0, decorrelate=True, block=64, precision="mixed",
              saturation=ps[0].saturation, catalog=True)
    items = [dict(science=p.science, reference=p.reference, science_var=p.science_var,
                  reference_var=p.reference_var, science_mask=p.science_mask, reference_mask=p.reference_mask)
             for p in ps]
    direct = _core.subtract_batch_native(items, frames_in_flight=1, graphs=False, **kw)
    replay = _core.subtract_batch_native(items, frames_in_flight=1, graphs=True, **kw)
    again = _core.subtract_batch_native(items, frames_in_flight=2, graphs=True, **kw)
    assert sum(r["graph_replayed"] for r in replay) >= 2
    assert all(not r["graph_replayed"] for r in direct)
    for run in (replay, again):
        for a, b in zip(direct, run, strict=True):
            np.testing.assert_array_equal(a["theta"], b["theta"])
            for name in ("difference", "variance", "mask", "score"):
                np.testing.assert_array_equal(a[name], b[name], err_msg=name)
            for name in a["catalog"]:
                np.testing.assert_array_equal(a["catalog"][name], b["catalog"][name], err_msg=name)


def test_variance_rescale_on_the_device_matches_host_staged():
    """rescale_variance=True: the device-resident path scales Var(D) and the
    whitened variance with the library's kernel (a float32 product, as the
    reference's numpy `variance * variance_scale`), bit-identical to the
    host-staged path."""
    p = validation.synthetic_pair(384, 384, 220, 17, mask_fraction=0.005)
    kw = dict(n_max=4, radius=10, n_knots=3, stamp_radius=12, cv_folds=0, score=True, decorrelate=True, block=64,
              saturation=p.saturation, rescale_variance=True)
    layers = dict(science_var=p.science_var, reference_var=p.reference_var, science_mask=p.science_mask,
                  reference_mask=p.reference_mask)
    a = delta.subtract(p.science, p.reference, device_resident=True, **layers, **kw)
    b = delta.subtract(p.science, p.reference, device_resident=False, **layers, **kw)
    assert a.variance_scale == b.variance_scale and a.variance_scale != 1.0
    for name in ("difference", "variance", "score"):
        np.testing.assert_array_equal(getattr(a, name), getattr(b, name), err_msg=name)
