"""``delta._core`` re-created over the sm_100a C ABI (include/delta_gpu.h).

Same function names, argument names / defaults, return types and error
behaviour as the reference's nanobind module (src/bindings.cpp:902-1036,
python/delta/_core.pyi). Arrays are coerced like nanobind's
``ndarray<const T, ndim<N>, c_contig>`` casters (a C-contiguous copy in the
declared dtype); the GIL is released inside every library call (ctypes).
All image work runs on the GPU; nothing here computes pixels on the CPU.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import check, context, ptr

__version__ = "1.1.1"


def _img(a, name="array"):
    a = np.ascontiguousarray(a, dtype=np.float32)
    if a.ndim != 2:
        raise TypeError(f"{name}: expected a 2-D float32 array, got shape {a.shape}")
    return a


def _img_opt(a, name="array"):
    return None if a is None else _img(a, name)


def _mask_opt(a, name="mask"):
    if a is None:
        return None
    a = np.ascontiguousarray(a, dtype=np.uint8)
    if a.ndim != 2:
        raise TypeError(f"{name}: expected a 2-D uint8 array, got shape {a.shape}")
    return a


def _mat(a, cols=None, name="matrix"):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if a.ndim == 1 and cols is not None:
        a = a.reshape(-1, cols) if a.size % cols == 0 else a.reshape(1, -1)
    if a.ndim != 2:
        raise TypeError(f"{name}: expected a 2-D float64 array")
    return a


def _vec(a, name="vector"):
    a = np.ascontiguousarray(a, dtype=np.float64).ravel()
    return a


def _knots(knots):
    k = _mat(knots, name="knots")
    if k.shape[1] != 2:
        raise ValueError("knots must be (k, 2)")
    if k.shape[0] < 3:
        raise ValueError("need at least 3 knots")
    return k


def _points(points):
    p = _mat(points, name="points")
    if p.shape[1] != 2:
        raise ValueError("points must be (m, 2)")
    return p


def _same_shape(a, ref, what):
    if a is not None and a.shape != ref.shape:
        raise RuntimeError(what)


# ---- basis / convolve ---------------------------------------------------------


def _resolve_radius(beta, n_max, radius):
    return radius if radius > 0 else _lib.lib().dgpu_default_radius(ctypes.c_double(beta), int(n_max))


def gauss_hermite_basis1d(beta: float, n_max: int, radius: int = 0) -> np.ndarray:
    """1-D sampled Gauss-Hermite basis functions, shape (n_max+1, ksize)."""
    if n_max < 0:
        raise ValueError("n_max must be >= 0")
    r = _resolve_radius(beta, n_max, radius)
    out = np.zeros((n_max + 1, 2 * r + 1), np.float64)
    ks = ctypes.c_int()
    check(_lib.lib().dgpu_gauss_hermite_basis1d(ctypes.c_double(beta), int(n_max), int(radius), ptr(out),
                                                ctypes.byref(ks)))
    return out


def gauss_hermite_kernels(beta: float, n_max: int, radius: int = 0):
    """(orders int32 (ncomp, 2), kernels float32 (ncomp, ks, ks))."""
    if n_max < 0:
        raise ValueError("n_max must be >= 0")
    r = _resolve_radius(beta, n_max, radius)
    nc = (n_max + 1) * (n_max + 2) // 2
    ks = 2 * r + 1
    orders = np.zeros((nc, 2), np.int32)
    kernels = np.zeros((nc, ks, ks), np.float32)
    kso = ctypes.c_int()
    check(_lib.lib().dgpu_gauss_hermite_kernels(ctypes.c_double(beta), int(n_max), int(radius), ptr(orders),
                                                ptr(kernels), ctypes.byref(kso)))
    return orders, kernels


def basis_convolve(image, beta: float, n_max: int, radius: int = 0) -> np.ndarray:
    """Convolve image with each basis component; returns (ncomp, H, W)."""
    img = _img(image, "image")
    h, w = img.shape
    if n_max < 0:
        raise ValueError("n_max must be >= 0")
    nc = (n_max + 1) * (n_max + 2) // 2
    out = np.empty((nc, h, w), np.float32)
    ctx = context()
    check(_lib.lib().dgpu_basis_convolve(ctx.handle, _lib.MEM_HOST, ptr(img), ctypes.c_int64(w),
                                         ctypes.c_int64(h), ctypes.c_double(beta), int(n_max), int(radius),
                                         ptr(out)), ctx.handle)
    return out


# ---- thin-plate spline ----------------------------------------------------------


def grid_knots(x0: float, y0: float, x1: float, y1: float, nx: int, ny: int) -> np.ndarray:
    """Regular nx*ny grid of knots over [x0,x1]x[y0,y1]."""
    if nx < 1 or ny < 1:
        raise ValueError("nx, ny must be >= 1")
    out = np.zeros((nx * ny, 2), np.float64)
    check(_lib.lib().dgpu_grid_knots(ctypes.c_double(x0), ctypes.c_double(y0), ctypes.c_double(x1),
                                     ctypes.c_double(y1), int(nx), int(ny), ptr(out)))
    return out


def tps_design(knots, points) -> np.ndarray:
    """Thin-plate regression-spline design matrix (m, n_basis)."""
    k = _knots(knots)
    p = _points(points)
    out = np.zeros((p.shape[0], k.shape[0]), np.float64)
    check(_lib.lib().dgpu_tps_design(ptr(k), k.shape[0], ptr(p), ctypes.c_int64(p.shape[0]), ptr(out)))
    return out


def tps_penalty(knots) -> np.ndarray:
    """Thin-plate bending-energy penalty matrix (n_basis, n_basis)."""
    k = _knots(knots)
    out = np.zeros((k.shape[0], k.shape[0]), np.float64)
    check(_lib.lib().dgpu_tps_penalty(ptr(k), k.shape[0], ptr(out)))
    return out


def tps_fit(knots, points, values, lam: float) -> np.ndarray:
    """Unweighted penalised fit: (D^T D + lam P) theta = D^T values."""
    k = _knots(knots)
    p = _points(points)
    v = _vec(values)
    out = np.zeros(k.shape[0], np.float64)
    check(_lib.lib().dgpu_tps_fit(ptr(k), k.shape[0], ptr(p), ctypes.c_int64(p.shape[0]), ptr(v),
                                  ctypes.c_double(lam), ptr(out)))
    return out


def tps_evaluate(knots, points, coeffs) -> np.ndarray:
    """Evaluate a fitted TPS field at points: design(points) @ coeffs."""
    k = _knots(knots)
    p = _points(points)
    c = _vec(coeffs)
    out = np.zeros(p.shape[0], np.float64)
    check(_lib.lib().dgpu_tps_evaluate(ptr(k), k.shape[0], ptr(p), ctypes.c_int64(p.shape[0]), ptr(c), ptr(out)))
    return out


# ---- subtraction ---------------------------------------------------------------------


def _model(knots, theta, beta, n_max, radius):
    k = _knots(knots)
    th = _vec(theta)
    m = _lib.Model(k.ctypes.data, k.shape[0], th.ctypes.data, th.size, float(beta), int(n_max), int(radius))
    return m, (k, th)


def subtract(science, reference, knots, theta, beta: float, n_max: int, radius: int = 0,
             saturation: float = 0.0, science_var=None, reference_var=None, science_mask=None,
             reference_mask=None) -> dict:
    """Full-frame spatially-varying subtraction with variance/mask propagation.

    Returns {'difference','variance','mask','timing'} (src/bindings.cpp:603-638).
    """
    sci = _img(science, "science")
    ref = _img(reference, "reference")
    svar = _img_opt(science_var, "science_var")
    rvar = _img_opt(reference_var, "reference_var")
    smask = _mask_opt(science_mask, "science_mask")
    rmask = _mask_opt(reference_mask, "reference_mask")
    _same_shape(svar, sci, "variance shape does not match data")
    _same_shape(smask, sci, "mask shape does not match data")
    _same_shape(rvar, ref, "variance shape does not match data")
    _same_shape(rmask, ref, "mask shape does not match data")
    if sci.shape != ref.shape:
        raise RuntimeError("subtract: science/reference shape mismatch")
    if n_max < 0:
        raise ValueError("n_max must be >= 0")
    h, w = sci.shape
    model, keep = _model(knots, theta, beta, n_max, radius)
    diff = np.empty((h, w), np.float32)
    var = np.empty((h, w), np.float32) if (svar is not None or rvar is not None) else None
    mask = np.empty((h, w), np.uint8) if (smask is not None or rmask is not None or saturation > 0) else None
    hv, hm = ctypes.c_int(), ctypes.c_int()
    ctx = context()
    check(_lib.lib().dgpu_subtract(ctx.handle, _lib.MEM_HOST, ctypes.c_int64(w), ctypes.c_int64(h), ptr(sci),
                                   ptr(ref), ptr(svar), ptr(rvar), ptr(smask), ptr(rmask), ctypes.byref(model),
                                   ctypes.c_double(saturation), ptr(diff), ptr(var), ptr(mask),
                                   ctypes.byref(hv), ctypes.byref(hm)), ctx.handle)
    return {"timing": _lib.drain_timing(ctx), "difference": diff, "variance": var if hv.value else None,
            "mask": mask if hm.value else None}


def kernel_chi2(science, reference, weights, knots, theta, beta: float, n_max: int, radius: int = 0,
                dx: float = 0.0, dy: float = 0.0, scale: float = 1.0, reference_mask=None, grad: bool = True,
                grad_reference: bool = False) -> dict:
    """Weighted chi^2 of the kernel model shifted by (dx, dy) and scaled by
    ``scale`` (include/delta_gpu.h, dgpu_kernel_chi2; no reference counterpart)
    and, with ``grad``, its gradients with respect to theta, (dx, dy) and the
    scale; with ``grad_reference`` also with respect to the reference image.
    Returns {'chi2', 'grad_theta', 'grad_shift', 'grad_scale', 'grad_reference'}."""
    sci = _img(science, "science")
    ref = _img(reference, "reference")
    wt = _img(weights, "weights")
    rmask = _mask_opt(reference_mask, "reference_mask")
    if sci.shape != ref.shape or wt.shape != sci.shape:
        raise ValueError("kernel_chi2: science, reference and weights must share a shape")
    _same_shape(rmask, ref, "mask shape does not match data")
    h, w = sci.shape
    model, keep = _model(knots, theta, beta, n_max, radius)
    n_theta = int(np.asarray(theta).size)
    chi2 = ctypes.c_double()
    g_theta = np.empty(n_theta) if grad else None
    g_shift = np.empty(2) if grad else None
    g_scale = ctypes.c_double()
    g_ref = np.empty((h, w), np.float32) if grad_reference else None
    ctx = context()
    check(_lib.lib().dgpu_kernel_chi2(ctx.handle, _lib.MEM_HOST, ctypes.c_int64(w), ctypes.c_int64(h), ptr(sci),
                                      ptr(ref), ptr(rmask), ptr(wt), ctypes.byref(model), ctypes.c_double(dx),
                                      ctypes.c_double(dy), ctypes.c_double(scale), ctypes.byref(chi2), ptr(g_theta),
                                      ptr(g_shift), ctypes.byref(g_scale) if grad else None, ptr(g_ref)),
          ctx.handle)
    return {"chi2": chi2.value, "grad_theta": g_theta, "grad_shift": g_shift,
            "grad_scale": g_scale.value if grad else None, "grad_reference": g_ref}


def stamp_gcv(science, reference, knots, stamp_x, stamp_y, stamp_radius: int, beta: float, n_max: int,
              log_lambda: float, dx: float = 0.0, dy: float = 0.0, scale: float = 1.0, radius: int = 0,
              science_var=None, reference_var=None, science_mask=None, reference_mask=None,
              grad: bool = True) -> dict:
    """GCV score and weighted RSS of the stamp fit at lambda = exp(log_lambda)
    with the basis shifted by (dx, dy) and scaled by ``scale``, and (``grad``)
    their gradients with respect to (log_lambda, dx, dy, scale)
    (include/delta_gpu.h, dgpu_stamp_gcv; no reference counterpart)."""
    sci = _img(science, "science")
    ref = _img(reference, "reference")
    svar = _img_opt(science_var, "science_var")
    rvar = _img_opt(reference_var, "reference_var")
    smask = _mask_opt(science_mask, "science_mask")
    rmask = _mask_opt(reference_mask, "reference_mask")
    if sci.shape != ref.shape:
        raise RuntimeError("fit_kernel: science/reference shape mismatch")
    k = _knots(knots)
    sx = np.ascontiguousarray(stamp_x, np.int32)
    sy = np.ascontiguousarray(stamp_y, np.int32)
    if sx.size != sy.size:
        raise RuntimeError("fit_kernel: stamp_x/stamp_y length mismatch")
    h, w = sci.shape
    nc = (n_max + 1) * (n_max + 2) // 2
    vals = np.zeros(4)
    theta = np.zeros((nc + 1) * k.shape[0])
    g_gcv = np.zeros(4) if grad else None
    g_rss = np.zeros(4) if grad else None
    ctx = context()
    check(_lib.lib().dgpu_stamp_gcv(
        ctx.handle, _lib.MEM_HOST, ctypes.c_int64(w), ctypes.c_int64(h), ptr(sci), ptr(ref), ptr(svar), ptr(rvar),
        ptr(smask), ptr(rmask), ptr(k), k.shape[0], ptr(sx), ptr(sy), int(sx.size), int(stamp_radius),
        ctypes.c_double(beta), int(n_max), int(radius), ctypes.c_double(log_lambda), ctypes.c_double(dx),
        ctypes.c_double(dy), ctypes.c_double(scale), ptr(vals), ptr(theta), ptr(g_gcv), ptr(g_rss)), ctx.handle)
    return {"gcv": float(vals[0]), "rss": float(vals[1]), "effective_dof": float(vals[2]), "n_pixels": int(vals[3]),
            "theta": theta, "grad_gcv": g_gcv, "grad_rss": g_rss}


def subtract_batch_native(items, *, n_max: int = 6, n_knots: int = 5, radius: int = 0, stamp_radius: int = 15,
                          threshold_sigma: float = 5.0, max_stamps: int = 200, saturation: float = 0.0,
                          fwhm_radius: int = 0, match_radius: int = 2, lambda_grid=None, clip_sigma: float = 4.0,
                          clip_iterations: int = 5, min_stamps: int = 5, cv_folds: int = 5, precision: str = "fp64",
                          decorrelate: bool = True, block: int = 256, score: bool = True, catalog: bool = True,
                          catalog_threshold_sigma: float = 5.0, frames_in_flight: int = 4,
                          catalog_capacity: int = 4096, graphs: bool = True, alloc=None) -> list[dict]:
    """dgpu_subtract_batch on host frames: ``items`` are dicts of science,
    reference and the optional science_var / reference_var / science_mask /
    reference_mask layers. Returns per frame {difference, variance, mask,
    score, theta, lambda, beta, direction, n_stamps_used, catalog, seconds,
    graph_replayed}. ``graphs``: run the post-fit device work of a frame as a
    recorded CUDA graph once its worker has seen the frame's shape and layers.
    ``alloc(shape, dtype)``, when given, makes the image outputs (e.g. pinned
    host memory, which the products are copied into at full link speed)."""
    grid = np.ascontiguousarray(np.logspace(-6, 6, 25) if lambda_grid is None else lambda_grid, np.float64)
    cfg = _lib.BatchConfig(n_max, n_knots, radius, stamp_radius, threshold_sigma, max_stamps, saturation,
                           fwhm_radius, match_radius, grid.ctypes.data, grid.size, clip_sigma, clip_iterations,
                           min_stamps, cv_folds, PRECISIONS[precision], int(decorrelate), block, int(score),
                           int(catalog), catalog_threshold_sigma, frames_in_flight, _lib._default_device(),
                           int(bool(graphs)))
    n = len(items)
    frames = (_lib.Frame * max(n, 1))()
    results = (_lib.FrameResult * max(n, 1))()
    keep, outs = [], []
    nc = (n_max + 1) * (n_max + 2) // 2
    for i, it in enumerate(items):
        sci, ref = _img(it["science"], "science"), _img(it["reference"], "reference")
        layers = [_img_opt(it.get("science_var"), "science_var"), _img_opt(it.get("reference_var"), "reference_var"),
                  _mask_opt(it.get("science_mask"), "science_mask"),
                  _mask_opt(it.get("reference_mask"), "reference_mask")]
        keep.append((sci, ref, *layers))
        h, w = sci.shape
        frames[i] = _lib.Frame(w, h, sci.ctypes.data, ref.ctypes.data,
                               *[None if a is None else a.ctypes.data for a in layers])
        mk = alloc or np.empty
        o = {"difference": mk((h, w), np.float32), "variance": mk((h, w), np.float32),
             "mask": mk((h, w), np.uint8), "score": mk((h, w), np.float32) if score else None,
             "theta": np.empty((nc + 1) * n_knots * n_knots),
             "cols": {name: np.empty(catalog_capacity, dt) for name, dt in _lib.CATALOG_COLUMNS}}
        outs.append(o)
        r = results[i]
        r.difference, r.variance, r.mask = (o["difference"].ctypes.data, o["variance"].ctypes.data,
                                            o["mask"].ctypes.data)
        r.score = None if o["score"] is None else o["score"].ctypes.data
        r.theta = o["theta"].ctypes.data
        r.catalog = _lib.CatalogColumns(*[o["cols"][name].ctypes.data for name, _ in _lib.CATALOG_COLUMNS])
        r.catalog_capacity = catalog_capacity
    check(_lib.lib().dgpu_subtract_batch(ctypes.byref(cfg), _lib.MEM_HOST, n, frames, results))
    out = []
    for i, o in enumerate(outs):
        r = results[i]
        cat = None
        if catalog and score:
            if not r.catalog_fetched:
                raise RuntimeError(f"subtract_batch: frame {i} has {r.catalog_count} catalog rows, above the capacity")
            cat = {name: v[: r.catalog_count].copy() for name, v in o["cols"].items()}
        out.append({"difference": o["difference"], "variance": o["variance"] if r.has_variance else None,
                    "mask": o["mask"] if r.has_mask else None, "score": o["score"], "theta": o["theta"],
                    "lambda": r.lambda_, "beta": r.beta,
                    "direction": "reference" if r.direction_is_reference else "science",
                    "n_stamps_used": r.n_stamps_used, "catalog": cat, "seconds": r.seconds,
                    "graph_replayed": bool(r.graph_replayed)})
    return out


def photometric_scale(knots, theta, component_sums, height: int, width: int) -> np.ndarray:
    """Per-pixel photometric scale field sum_n a_n(x,y) S_n, shape (H,W)."""
    k = _knots(knots)
    th = _vec(theta)
    s = _vec(component_sums)
    out = np.empty((height, width), np.float32)
    ctx = context()
    check(_lib.lib().dgpu_photometric_scale(ctx.handle, _lib.MEM_HOST, ptr(k), k.shape[0], ptr(th),
                                            ctypes.c_int64(th.size), ptr(s), int(s.size), ctypes.c_int64(height),
                                            ctypes.c_int64(width), ptr(out)), ctx.handle)
    return out


def photometric_scale_at(knots, theta, component_sums, points) -> np.ndarray:
    """Photometric scale evaluated at points, shape (m,)."""
    k = _knots(knots)
    th = _vec(theta)
    s = _vec(component_sums)
    p = _points(points)
    out = np.zeros(p.shape[0], np.float64)
    check(_lib.lib().dgpu_photometric_scale_at(ptr(k), k.shape[0], ptr(th), ctypes.c_int64(th.size), ptr(s),
                                               int(s.size), ptr(p), ctypes.c_int64(p.shape[0]), ptr(out)))
    return out


# ---- penalised GLS + stamp fit ----------------------------------------------------------

# Normal-equation arithmetic of fit_kernel / solve_gls* (the solve itself is
# FP64 in every mode): "fp64" (default, accuracy reference), "fp32" (plain
# FP32 SIMT), "mixed" (BF16x3 tensor-core split products + one FP64 refinement step),
# "tf32" (one TF32 tensor-core product + the same refinement step).
PRECISIONS = {"fp64": _lib.PREC_FP64, "fp32": _lib.PREC_FP32, "mixed": _lib.PREC_MIXED, "tf32": _lib.PREC_TF32}
_PREC_NAMES = {v: k for k, v in PRECISIONS.items()}
_default_precision = "fp64"


def set_default_precision(name: str) -> None:
    """Select the normal-equation arithmetic used when a call does not pass one."""
    global _default_precision
    if name not in PRECISIONS:
        raise ValueError(f"precision must be one of {sorted(PRECISIONS)}")
    _default_precision = name


def _prec(precision):
    return PRECISIONS[precision or _default_precision]


def _gls_struct(P, n_lambda, nc, n_stamps=0):
    bufs = {
        "theta": np.zeros(P, np.float64),
        "lambda_grid": np.zeros(max(n_lambda, 1), np.float64),
        "gcv_curve": np.zeros(max(n_lambda, 1), np.float64),
        "component_sums": np.zeros(max(nc, 1), np.float64),
        "stamp_x": np.zeros(max(n_stamps, 1), np.int32),
        "stamp_y": np.zeros(max(n_stamps, 1), np.int32),
        "stamp_chi2": np.zeros(max(n_stamps, 1), np.float64),
        "stamp_accepted": np.zeros(max(n_stamps, 1), np.uint8),
    }
    res = _lib.GlsResult()
    for name, arr in bufs.items():
        setattr(res, name, arr.ctypes.data)
    return res, bufs


def _gls_dict(res, bufs) -> dict:
    nl = res.n_lambda_out
    return {
        "theta": bufs["theta"],
        "n_components": int(res.n_components),
        "n_spatial": int(res.n_spatial),
        "lambda": float(res.__getattribute__("lambda")),
        "gcv": float(res.gcv),
        "effective_dof": float(res.effective_dof),
        "rss": float(res.rss),
        "lambda_grid": bufs["lambda_grid"][:nl].copy(),
        "gcv_curve": bufs["gcv_curve"][:nl].copy(),
        # extensions: the arithmetic that produced theta and the last mixed
        # refinement correction (see dgpu_gls_result)
        "precision_used": _PREC_NAMES.get(int(res.precision_used), str(int(res.precision_used))),
        "refine_correction": float(res.refine_correction),
        "used_ldlt": bool(res.used_ldlt),
    }


def _solve_inputs(knots, points, target, weights, bn):
    k = _knots(knots)
    p = _points(points)
    t = _vec(target)
    w = _vec(weights)
    b = np.ascontiguousarray(bn, dtype=np.float64)
    if b.ndim == 1:
        b = b.reshape(-1, 1)
    m = p.shape[0]
    if t.size != m or w.size != m or b.shape[0] != m:
        raise RuntimeError("solve_gls: row counts of design/target/weights/bn disagree")
    return k, p, t, w, b


def solve_gls(knots, points, target, weights, bn, lam: float, precision: str | None = None) -> dict:
    """Penalised GLS at fixed lambda over the factorized A&L model."""
    k, p, t, w, b = _solve_inputs(knots, points, target, weights, bn)
    nc = b.shape[1]
    res, bufs = _gls_struct((nc + 1) * k.shape[0], 0, nc)
    ctx = context()
    check(_lib.lib().dgpu_solve_gls(ctx.handle, ptr(k), k.shape[0], ptr(p), ctypes.c_int64(p.shape[0]), ptr(t),
                                    ptr(w), ptr(b), int(nc), ctypes.c_double(lam), _prec(precision),
                                    ctypes.byref(res)), ctx.handle)
    return _gls_dict(res, bufs)


def solve_gls_gcv(knots, points, target, weights, bn, lambda_grid, precision: str | None = None) -> dict:
    """Penalised GLS selecting lambda by GCV over lambda_grid."""
    k, p, t, w, b = _solve_inputs(knots, points, target, weights, bn)
    grid = _vec(lambda_grid)
    nc = b.shape[1]
    res, bufs = _gls_struct((nc + 1) * k.shape[0], grid.size, nc)
    ctx = context()
    check(_lib.lib().dgpu_solve_gls_gcv(ctx.handle, ptr(k), k.shape[0], ptr(p), ctypes.c_int64(p.shape[0]), ptr(t),
                                        ptr(w), ptr(b), int(nc), ptr(grid), int(grid.size), _prec(precision),
                                        ctypes.byref(res)), ctx.handle)
    return _gls_dict(res, bufs)


def solve_gls_cv(knots, points, target, weights, bn, lambda_grid, group, n_groups: int,
                 precision: str | None = None) -> dict:
    """Penalised GLS selecting lambda by k-fold group cross-validation."""
    k, p, t, w, b = _solve_inputs(knots, points, target, weights, bn)
    grid = _vec(lambda_grid)
    g = np.ascontiguousarray(group, dtype=np.int32).ravel()
    if g.size != p.shape[0]:
        raise RuntimeError("solve_gls_cv: group.size() must match points.rows()")
    nc = b.shape[1]
    res, bufs = _gls_struct((nc + 1) * k.shape[0], grid.size, nc)
    ctx = context()
    check(_lib.lib().dgpu_solve_gls_cv(ctx.handle, ptr(k), k.shape[0], ptr(p), ctypes.c_int64(p.shape[0]), ptr(t),
                                       ptr(w), ptr(b), int(nc), ptr(grid), int(grid.size), ptr(g), int(n_groups),
                                       _prec(precision), ctypes.byref(res)), ctx.handle)
    return _gls_dict(res, bufs)


def fit_kernel(science, reference, knots, stamp_x, stamp_y, stamp_radius: int, beta: float, n_max: int,
               lambda_grid, radius: int = 0, clip_sigma: float = 4.0, clip_iterations: int = 5,
               min_stamps: int = 5, cv_folds: int = 0, science_var=None, reference_var=None, science_mask=None,
               reference_mask=None, precision: str | None = None) -> dict:
    """Fit the matching kernel + background from stamp pixels via penalised GLS
    with iterative per-stamp sigma clipping (src/bindings.cpp:643-693)."""
    sci = _img(science, "science")
    ref = _img(reference, "reference")
    svar = _img_opt(science_var, "science_var")
    rvar = _img_opt(reference_var, "reference_var")
    smask = _mask_opt(science_mask, "science_mask")
    rmask = _mask_opt(reference_mask, "reference_mask")
    _same_shape(svar, sci, "variance shape does not match data")
    _same_shape(smask, sci, "mask shape does not match data")
    _same_shape(rvar, ref, "variance shape does not match data")
    _same_shape(rmask, ref, "mask shape does not match data")
    if sci.shape != ref.shape:
        raise RuntimeError("fit_kernel: science/reference shape mismatch")
    sx = np.ascontiguousarray(stamp_x, dtype=np.int32).ravel()
    sy = np.ascontiguousarray(stamp_y, dtype=np.int32).ravel()
    if sx.size != sy.size:
        raise RuntimeError("fit_kernel: stamp_x/stamp_y length mismatch")
    k = _knots(knots)
    grid = _vec(lambda_grid)
    if n_max < 0:
        raise ValueError("n_max must be >= 0")
    nc = (n_max + 1) * (n_max + 2) // 2
    h, w = sci.shape
    res, bufs = _gls_struct((nc + 1) * k.shape[0], grid.size, nc, sx.size)
    ctx = context()
    check(_lib.lib().dgpu_fit_kernel(
        ctx.handle, _lib.MEM_HOST, ctypes.c_int64(w), ctypes.c_int64(h), ptr(sci), ptr(ref), ptr(svar), ptr(rvar),
        ptr(smask), ptr(rmask), ptr(k), k.shape[0], ptr(sx), ptr(sy), int(sx.size), int(stamp_radius),
        ctypes.c_double(beta), int(n_max), int(radius), ptr(grid), int(grid.size), ctypes.c_double(clip_sigma),
        int(clip_iterations), int(min_stamps), int(cv_folds), _prec(precision), ctypes.byref(res)), ctx.handle)
    out = _gls_dict(res, bufs)
    nt = int(res.n_stamps_total)
    out["timing"] = _lib.drain_timing(ctx)
    out["component_sums"] = bufs["component_sums"][:nc].copy()
    out["n_pixels"] = int(res.n_pixels)
    out["n_stamps_used"] = int(res.n_stamps_used)
    out["n_stamps_total"] = nt
    out["n_stamps_rejected"] = int(res.n_stamps_rejected)
    out["reduced_chi2"] = float(res.reduced_chi2)
    out["cv_exact_design_bytes"] = int(res.cv_exact_design_bytes)
    out["stamp_x"] = bufs["stamp_x"][:nt].copy()
    out["stamp_y"] = bufs["stamp_y"][:nt].copy()
    out["stamp_chi2"] = bufs["stamp_chi2"][:nt].copy()
    out["stamp_accepted"] = bufs["stamp_accepted"][:nt].copy()
    return out


# ---- stamp selection -----------------------------------------------------------------


def _detect_params(stamp_radius, threshold_sigma, max_stamps, saturation, isolation_radius, border, fwhm_radius,
                   match_radius):
    return _lib.DetectParams(int(stamp_radius), float(threshold_sigma), int(max_stamps), float(saturation),
                             int(isolation_radius), int(border), int(fwhm_radius), int(match_radius))


# ---- FITS I/O ------------------------------------------------------------------------


def _fits_check(rc: int) -> None:
    if rc == _lib.DGPU_OK:
        return
    msg = _lib.lib().dgpu_last_error(None).decode(errors="replace")
    if rc == _lib.DGPU_ERR_INVALID:
        raise ValueError(msg)
    raise RuntimeError(msg)


def read_fits(path: str, *, alloc=None) -> dict:
    """Read a FITS file into {'data', 'variance', 'mask'} arrays (src/bindings.cpp:128-145):
    the primary image, or the DIFFERENCE extension when the primary holds no
    2-D image, plus the optional VARIANCE / MASK extensions (None when absent).

    ``alloc(shape, dtype)`` (an extension) supplies the output arrays, e.g.
    pinned host memory for a fast upload; the default is ``np.empty``."""
    p = str(path).encode()
    w, h = ctypes.c_int64(), ctypes.c_int64()
    hv, hm = ctypes.c_int(), ctypes.c_int()
    L = _lib.lib()
    _fits_check(L.dgpu_fits_probe(p, ctypes.byref(w), ctypes.byref(h), ctypes.byref(hv), ctypes.byref(hm)))
    make = alloc or (lambda shape, dtype: np.empty(shape, dtype))
    shape = (int(h.value), int(w.value))
    data = make(shape, np.float32)
    var = make(shape, np.float32) if hv.value else None
    mask = make(shape, np.uint8) if hm.value else None
    _fits_check(L.dgpu_fits_read(p, w, h, ptr(data), ptr(var), ptr(mask)))
    return {"data": data, "variance": var, "mask": mask}


def write_fits(path: str, data, variance=None, mask=None, overwrite: bool = False) -> None:
    """Write data plus optional variance / mask layers to a FITS file
    (src/bindings.cpp:147-166); raises if the file exists unless overwrite=True."""
    d = np.ascontiguousarray(data, dtype=np.float32)
    if d.ndim != 2:
        raise TypeError(f"data: expected a 2-D float32 array, got shape {d.shape}")
    h, w = d.shape
    v = None if variance is None else np.ascontiguousarray(variance, dtype=np.float32)
    m = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint8)
    if v is not None and v.shape != d.shape:
        raise RuntimeError("variance shape does not match data")
    if m is not None and m.shape != d.shape:
        raise RuntimeError("mask shape does not match data")
    _fits_check(_lib.lib().dgpu_fits_write(str(path).encode(), ctypes.c_int64(w), ctypes.c_int64(h), ptr(d), ptr(v),
                                           ptr(m), int(bool(overwrite))))


def weighted_mean(data, variance, mask) -> float:
    """Inverse-variance weighted mean over unmasked pixels."""
    d = np.ascontiguousarray(data, np.float32)
    v = np.ascontiguousarray(variance, np.float32)
    m = np.ascontiguousarray(mask, np.uint8)
    out = ctypes.c_double()
    ctx = context()
    check(_lib.lib().dgpu_weighted_mean(ctx.handle, _lib.MEM_HOST, ctypes.c_int64(d.size), ptr(d), ptr(v), ptr(m),
                                        ctypes.byref(out)), ctx.handle)
    return out.value


def estimate_background(data, mask=None):
    """Robust (median, MAD-sigma) background over unmasked pixels."""
    d = _img(data, "data")
    m = _mask_opt(mask)
    if m is not None and m.shape != d.shape:
        raise RuntimeError("mask shape does not match data")
    h, w = d.shape
    med, sig = ctypes.c_double(), ctypes.c_double()
    ctx = context()
    check(_lib.lib().dgpu_estimate_background(ctx.handle, _lib.MEM_HOST, ctypes.c_int64(w), ctypes.c_int64(h),
                                              ptr(d), ptr(m), ctypes.byref(med), ctypes.byref(sig)), ctx.handle)
    return med.value, sig.value


def detect_stamps(data, mask=None, stamp_radius: int = 15, threshold_sigma: float = 5.0, max_stamps: int = 200,
                  saturation: float = 0.0, isolation_radius: int = 0, border: int = 0, fwhm_radius: int = 0,
                  match_radius: int = 2) -> dict:
    """Detect bright, isolated, unsaturated point-source stamps."""
    d = _img(data, "data")
    m = _mask_opt(mask)
    if m is not None and m.shape != d.shape:
        raise RuntimeError("mask shape does not match data")
    h, w = d.shape
    p = _detect_params(stamp_radius, threshold_sigma, max_stamps, saturation, isolation_radius, border, fwhm_radius,
                       match_radius)
    cap = max(int(max_stamps), 1)
    cols = {"x": np.zeros(cap, np.int32), "y": np.zeros(cap, np.int32), "flux": np.zeros(cap),
            "snr": np.zeros(cap), "fwhm": np.zeros(cap)}
    n = ctypes.c_int()
    ctx = context()
    check(_lib.lib().dgpu_detect_stamps(ctx.handle, _lib.MEM_HOST, ctypes.c_int64(w), ctypes.c_int64(h), ptr(d),
                                        ptr(m), ctypes.byref(p), cap, *[ptr(cols[k]) for k in ("x", "y", "flux",
                                                                                              "snr", "fwhm")],
                                        ctypes.byref(n)), ctx.handle)
    return {k: v[: n.value].copy() for k, v in cols.items()}


def select_stamps(science, reference, science_mask=None, reference_mask=None, catalog_x=None, catalog_y=None,
                  stamp_radius: int = 15, threshold_sigma: float = 5.0, max_stamps: int = 200,
                  saturation: float = 0.0, isolation_radius: int = 0, border: int = 0, fwhm_radius: int = 0,
                  match_radius: int = 2) -> dict:
    """Select matched stamps across both images and the convolution direction."""
    s = _img(science, "science")
    r = _img(reference, "reference")
    sm = _mask_opt(science_mask)
    rm = _mask_opt(reference_mask)
    h, w = s.shape
    if r.shape != s.shape:
        raise RuntimeError("select_stamps: science/reference shape mismatch")
    cx = None if catalog_x is None else np.ascontiguousarray(catalog_x, np.int32).ravel()
    cy = None if catalog_y is None else np.ascontiguousarray(catalog_y, np.int32).ravel()
    if (cx is None) != (cy is None):
        cx = cy = None
    ncat = 0 if cx is None else min(cx.size, cy.size)
    p = _detect_params(stamp_radius, threshold_sigma, max_stamps, saturation, isolation_radius, border, fwhm_radius,
                       match_radius)
    cap = max(int(max_stamps), ncat, 1)
    x = np.zeros(cap, np.int32)
    y = np.zeros(cap, np.int32)
    fs = np.zeros(cap)
    fr = np.zeros(cap)
    ms, mr = ctypes.c_double(), ctypes.c_double()
    dref, n = ctypes.c_int(), ctypes.c_int()
    ctx = context()
    check(_lib.lib().dgpu_select_stamps(ctx.handle, _lib.MEM_HOST, ctypes.c_int64(w), ctypes.c_int64(h), ptr(s),
                                        ptr(r), ptr(sm), ptr(rm), ptr(cx), ptr(cy), int(ncat), ctypes.byref(p), cap,
                                        ptr(x), ptr(y), ptr(fs), ptr(fr), ctypes.byref(ms), ctypes.byref(mr),
                                        ctypes.byref(dref), ctypes.byref(n)), ctx.handle)
    k = n.value
    return {"x": x[:k].copy(), "y": y[:k].copy(), "fwhm_science": fs[:k].copy(), "fwhm_reference": fr[:k].copy(),
            "median_fwhm_science": ms.value, "median_fwhm_reference": mr.value,
            "direction": "reference" if dref.value else "science"}


def estimate_psf(image, xs, ys, radius: int) -> np.ndarray:
    """Median, unit-sum postage stamp of the listed sources (the score path's PSF);
    not part of the reference binding (the reference computes it in NumPy)."""
    img = _img(image, "image")
    h, w = img.shape
    x = np.ascontiguousarray(xs, np.int32).ravel()
    y = np.ascontiguousarray(ys, np.int32).ravel()
    side = 2 * int(radius) + 1
    out = np.empty((side, side), np.float32)
    ctx = context()
    check(_lib.lib().dgpu_estimate_psf(ctx.handle, _lib.MEM_HOST, ctypes.c_int64(w), ctypes.c_int64(h), ptr(img),
                                       ptr(x), ptr(y), int(min(x.size, y.size)), int(radius), ptr(out)), ctx.handle)
    return out


# ---- noise decorrelation -------------------------------------------------------------


def decorrelate(difference, knots, theta, beta: float, n_max: int, var_science, var_reference, block: int = 256,
                radius: int = 0, kernel_cell_blocks: int = 0) -> dict:
    """Spatially-varying noise decorrelation via apodized FFT blocks.

    Returns {'difference', 'variance', 'timing'} (src/bindings.cpp:766-792).
    """
    d = _img(difference, "difference")
    vs = _img(var_science, "var_science")
    vr = _img(var_reference, "var_reference")
    h, w = d.shape
    model, keep = _model(knots, theta, beta, n_max, radius)
    out_d = np.empty((h, w), np.float32)
    out_v = np.empty((h, w), np.float32)
    ctx = context()
    check(_lib.lib().dgpu_decorrelate(ctx.handle, _lib.MEM_HOST, ctypes.c_int64(w), ctypes.c_int64(h), ptr(d),
                                      ctypes.byref(model), ptr(vs), ptr(vr), int(block), int(kernel_cell_blocks),
                                      ptr(out_d), ptr(out_v)), ctx.handle)
    return {"difference": out_d, "variance": out_v, "timing": _lib.drain_timing(ctx)}


def whiten_score_psf(psf, knots, theta, beta: float, n_max: int, var_science, var_reference, block: int,
                     radius: int = 0) -> np.ndarray:
    """Apply the ZOGY decorrelation filter to a PSF stamp (frame-centre kernel/noise)."""
    p = _img(psf, "psf")
    if p.shape[0] != p.shape[1]:
        raise RuntimeError("whiten_score_psf: psf must be square")
    if block < p.shape[0]:
        raise RuntimeError("whiten_score_psf: block must be >= psf side")
    vs = _img(var_science, "var_science")
    vr = _img(var_reference, "var_reference")
    if vs.shape != vr.shape:
        raise RuntimeError("whiten_score_psf: variance shapes disagree")
    h, w = vs.shape
    model, keep = _model(knots, theta, beta, n_max, radius)
    out = np.empty_like(p)
    ctx = context()
    check(_lib.lib().dgpu_whiten_score_psf(ctx.handle, _lib.MEM_HOST, ptr(p), int(p.shape[0]), ctypes.byref(model),
                                           ctypes.c_int64(w), ctypes.c_int64(h), ptr(vs), ptr(vr), int(block),
                                           ptr(out)), ctx.handle)
    return out


def decorrelate_block(image, kernel, var_science: float, var_reference: float) -> np.ndarray:
    """Whiten one square block with a constant kernel/noise (FFT core)."""
    img = _img(image, "image")
    n = img.shape[0]
    if img.shape[1] != n:
        raise RuntimeError("decorrelate_block: image must be square")
    k = _img(kernel, "kernel")
    if k.shape[0] != k.shape[1]:
        raise RuntimeError("decorrelate_block: kernel must be square")
    out = np.empty((n, n), np.float32)
    ctx = context()
    check(_lib.lib().dgpu_decorrelate_block(ctx.handle, ptr(img), int(n), ptr(k), int(k.shape[0]),
                                            ctypes.c_double(var_science), ctypes.c_double(var_reference), ptr(out)),
          ctx.handle)
    return out


def decorrelation_kernel(kernel, var_science: float, var_reference: float, n: int) -> np.ndarray:
    """Real-space decorrelation kernel (centred, n x n) for QA."""
    k = _img(kernel, "kernel")
    out = np.empty((n, n), np.float32)
    ctx = context()
    check(_lib.lib().dgpu_decorrelation_kernel(ctx.handle, ptr(k), int(k.shape[0]), ctypes.c_double(var_science),
                                               ctypes.c_double(var_reference), int(n), ptr(out)), ctx.handle)
    return out


# ---- matched filter -------------------------------------------------------------------


def matched_filter(image, psf, variance) -> np.ndarray:
    """Match-filtered score image (per-pixel S/N map)."""
    img = _img(image, "image")
    p = _img(psf, "psf")
    var = _img(variance, "variance")
    if p.shape[0] != p.shape[1]:
        raise RuntimeError("matched_filter: psf must be square")
    if var.shape != img.shape:
        raise RuntimeError("matched_filter: variance must match image shape")
    h, w = img.shape
    out = np.empty((h, w), np.float32)
    ctx = context()
    check(_lib.lib().dgpu_matched_filter(ctx.handle, _lib.MEM_HOST, ctypes.c_int64(w), ctypes.c_int64(h), ptr(img),
                                         ptr(p), int(p.shape[0]), ptr(var), ptr(out)), ctx.handle)
    return out


# ---- catalog ------------------------------------------------------------------------------


def build_catalog(score, difference, mask=None, threshold_sigma: float = 5.0,
                  threshold_sigma_dipole: float = 3.0, expected_fwhm: float = 3.5,
                  fwhm_tolerance_lo: float = 0.3, fwhm_tolerance_hi: float = 3.0, aperture_radius: int = 0,
                  exclude_bad_pixels: bool = True, return_negative: bool = False, fit_psf_shape: bool = False,
                  shape_chi2_tolerance: float = 3.0, variance=None, psf=None, bright_star_radius: float = 0.0,
                  max_shape_fit: int = 5000, bright_x=None, bright_y=None) -> dict:
    """Connected-component source catalog from a match-filtered score image."""
    sc = _img(score, "score")
    df = _img(difference, "difference")
    mk = _mask_opt(mask)
    var = _img_opt(variance, "variance")
    p = _img_opt(psf, "psf")
    if df.shape != sc.shape:
        raise RuntimeError("build_catalog: difference shape must match score")
    if var is not None and var.shape != sc.shape:
        raise RuntimeError("build_catalog: variance shape must match score")
    if p is not None and p.shape[0] != p.shape[1]:
        raise RuntimeError("build_catalog: psf must be square")
    if (bright_x is None) != (bright_y is None):
        raise RuntimeError("build_catalog: supply both bright_x and bright_y, or neither")
    bx = None if bright_x is None else np.ascontiguousarray(bright_x, np.float64).ravel()
    by = None if bright_y is None else np.ascontiguousarray(bright_y, np.float64).ravel()
    if bx is not None and bx.size != by.size:
        raise RuntimeError("build_catalog: bright_x and bright_y must be the same length")
    if mk is not None and mk.shape != sc.shape:
        raise RuntimeError("mask shape does not match data")
    h, w = sc.shape
    prm = _lib.CatalogParams(float(threshold_sigma), float(threshold_sigma_dipole), float(expected_fwhm),
                             float(fwhm_tolerance_lo), float(fwhm_tolerance_hi), int(aperture_radius),
                             int(bool(exclude_bad_pixels)), int(bool(return_negative)), int(bool(fit_psf_shape)),
                             float(shape_chi2_tolerance), float(bright_star_radius), int(max_shape_fit))
    ctx = context()
    L = _lib.lib()
    n = ctypes.c_int()
    check(L.dgpu_build_catalog(ctx.handle, _lib.MEM_HOST, ctypes.c_int64(w), ctypes.c_int64(h), ptr(sc), ptr(df),
                               ptr(mk), ctypes.byref(prm), ptr(var), ptr(p), 0 if p is None else int(p.shape[0]),
                               ptr(bx), ptr(by), 0 if bx is None else int(bx.size), ctypes.byref(n)), ctx.handle)
    cols = {name: np.empty(n.value, dt) for name, dt in _lib.CATALOG_COLUMNS}
    cc = _lib.CatalogColumns(*[cols[name].ctypes.data for name, _ in _lib.CATALOG_COLUMNS])
    check(L.dgpu_catalog_fetch(ctx.handle, ctypes.byref(cc), n.value), ctx.handle)
    cols["timing"] = _lib.drain_timing(ctx)
    return cols


def catalog_labels(shape) -> np.ndarray:
    """Label image of the last build_catalog on this thread (not in the reference
    binding; exposes the labels the reference keeps internal)."""
    h, w = shape
    out = np.empty((h, w), np.int32)
    ctx = context()
    check(_lib.lib().dgpu_catalog_labels(ctx.handle, _lib.MEM_HOST, ptr(out), ctypes.c_int64(h * w)), ctx.handle)
    return out


def drain_timing():
    """Drain accumulated DELTA_TIMING sub-stage timers into a {label: seconds} dict."""
    return _lib.drain_timing(context())
