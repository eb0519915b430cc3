"""Loader for oracle/_build/liboracle.so (oracle/csrc/oracle.c) -- TEST INFRASTRUCTURE ONLY.

``subtract`` / ``matched_filter`` here reproduce the reference's float32
arithmetic (accumulation order and FMA contraction); numpy_ref supplies the
FP64 lattice, basis taps and the order statistic.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import numpy_ref as nr
from ._loader import HERE, f32, ptr, u8

_LIB_PATH = HERE / "_build" / "liboracle.so"
_lib = None


def available() -> bool:
    return _LIB_PATH.exists()


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"{_LIB_PATH} not built (make -C oracle)")
        _lib = ctypes.CDLL(str(_LIB_PATH))
    return _lib


def _field_args(fl: nr.Fields):
    """Argument tuple (exact, nf, w, h, full, lat, ncx, ncy, cellx, wx, celly, wy) + keepalive."""
    nf = fl.nc + 1
    if fl.exact:
        full = np.ascontiguousarray(np.stack([fl.field_full(f) for f in range(nf)]), np.float32)
        keep = [full]
        return (1, nf, fl.w, fl.h, ptr(full), None, 0, 0, None, None, None, None), keep
    lat = np.ascontiguousarray(fl.coarse, np.float64)
    cellx = np.ascontiguousarray(fl.cellx, np.int32)
    celly = np.ascontiguousarray(fl.celly, np.int32)
    wx = np.ascontiguousarray(fl.wx, np.float32)
    wy = np.ascontiguousarray(fl.wy, np.float32)
    keep = [lat, cellx, celly, wx, wy]
    return (0, nf, fl.w, fl.h, None, ptr(lat), fl.ncx, fl.ncy, ptr(cellx), ptr(wx), ptr(celly), ptr(wy)), keep


def field_full(fl: nr.Fields, f: int) -> np.ndarray:
    args, keep = _field_args(fl)
    out = np.zeros((fl.h, fl.w), np.float32)
    lib().oc_field_full(*args, int(f), ptr(out))
    return out


def subtract(science, reference, knots, theta, beta, n_max, radius=0, saturation=0.0,
             science_var=None, reference_var=None, science_mask=None, reference_mask=None) -> dict:
    """delta::subtract (src/subtract.cpp:429-966) with reference float32 semantics."""
    sci, ref = f32(science), f32(reference)
    h, w = sci.shape
    r = nr.resolve_radius(beta, n_max, radius)
    ks = 2 * r + 1
    b1d = nr.gauss_hermite_basis1d(beta, n_max, r)
    taps = np.ascontiguousarray(b1d.astype(np.float32))
    orders = nr.basis_orders(n_max)
    nc = len(orders)
    ord_nx = np.array([o[0] for o in orders], np.int32)
    ord_ny = np.array([o[1] for o in orders], np.int32)
    fl = nr.Fields(knots, theta, nc, w, h)
    args, keep = _field_args(fl)
    rmask = u8(reference_mask)
    fill = nr.reference_fill_value(ref, rmask)
    diff = np.zeros((h, w), np.float32)
    L = lib()
    L.oc_subtract_model(ptr(sci), ptr(ref), ptr(rmask), w, h, *args[:1], *args[1:2], *args[4:],
                        n_max, ks, ptr(taps), ptr(ord_nx), ptr(ord_ny), ctypes.c_float(fill), ptr(diff))
    out = {"difference": diff, "variance": None, "mask": None}
    vs, vr = f32(science_var), f32(reference_var)
    if vs is not None or vr is not None:
        phi = np.ascontiguousarray(np.stack([nr.kernel2d(b1d, orders, c) for c in range(nc)]), np.float32)
        var = np.zeros((h, w), np.float32)
        L.oc_variance(ptr(vs), ptr(vr), w, h, *args[:1], *args[1:2], *args[4:], r, ptr(phi), ptr(var))
        out["variance"] = var
    smask = u8(science_mask)
    if smask is not None or rmask is not None or saturation > 0.0:
        mask = np.zeros((h, w), np.uint8)
        fillv = ctypes.c_float()
        L.oc_mask(ptr(sci), ptr(ref), ptr(smask), ptr(rmask), w, h, ctypes.c_double(saturation), r,
                  ptr(diff), ptr(out["variance"]), ptr(mask), ctypes.byref(fillv))
        out["mask"] = mask
    return out


def matched_filter(image, psf, variance) -> np.ndarray:
    """src/noise.cpp:535-632 with reference float32 semantics."""
    img, psf, var = f32(image), f32(psf), f32(variance)
    h, w = img.shape
    out = np.zeros((h, w), np.float32)
    lib().oc_matched_filter(ptr(img), ptr(var), w, h, ptr(psf), psf.shape[0], ptr(out))
    return out


# ---------------------------------------------------------------------------
# Penalised GLS in C (oracle/csrc/oracle_fit.c)
# ---------------------------------------------------------------------------


def assemble(design, target, weights, bn):
    """M = Xs^T Xs, rhs, ywy (src/solve.cpp:70-145) by the OpenMP rank update."""
    d = np.ascontiguousarray(design, np.float64)
    b = np.ascontiguousarray(bn, np.float64)
    t = np.ascontiguousarray(target, np.float64)
    wt = np.ascontiguousarray(weights, np.float64)
    n, k = d.shape
    nc = b.shape[1]
    if t.size != n or wt.size != n or b.shape[0] != n:
        raise RuntimeError("solve_gls: row counts of design/target/weights/bn disagree")
    p = (nc + 1) * k
    m = np.zeros((p, p))
    rhs = np.zeros(p)
    ywy = ctypes.c_double()
    rc = lib().of_assemble(ctypes.c_int64(n), k, nc, ptr(d), ptr(b), ptr(t), ptr(wt), ptr(m), ptr(rhs),
                           ctypes.byref(ywy))
    if rc:
        raise MemoryError("of_assemble")
    return m, rhs, ywy.value


def solve_grid(s: nr.System, lambdas) -> list[dict]:
    """solve_at (src/solve.cpp:147-193) at every lambda, lambdas in parallel."""
    grid = np.ascontiguousarray(lambdas, np.float64)
    p = s.p
    f = np.ascontiguousarray(s.pen_half, np.float64)
    nf = f.shape[1] if f.size else 0
    theta = np.zeros((grid.size, p))
    edf, rss, gcv = np.zeros(grid.size), np.zeros(grid.size), np.zeros(grid.size)
    used = np.zeros(grid.size, np.int32)
    rc = lib().of_solve_grid(p, ptr(np.ascontiguousarray(s.m, np.float64)), ptr(np.ascontiguousarray(s.p0)),
                             ptr(np.ascontiguousarray(s.rhs, np.float64)), ctypes.c_double(s.ywy),
                             ctypes.c_int64(s.n), ptr(f) if nf else None, nf, ptr(grid), grid.size, ptr(theta),
                             ptr(edf), ptr(rss), ptr(gcv), ptr(used))
    if rc:
        raise MemoryError("of_solve_grid")
    return [{"theta": theta[i], "lambda": float(grid[i]), "effective_dof": float(edf[i]), "rss": float(rss[i]),
             "gcv": float(gcv[i]), "n_components": s.nc, "n_spatial": s.k, "used_ldlt": bool(used[i])}
            for i in range(grid.size)]


def gls_gcv(design, target, weights, bn, penalty, lambda_grid) -> dict:
    """solve_gls_gcv_design (src/solve.cpp:227-262) with the C assembly and solves."""
    m, rhs, ywy = assemble(design, target, weights, bn)
    k = np.shape(design)[1]
    nc = np.shape(bn)[1]
    s = nr.System.from_parts(m, rhs, ywy, int(np.shape(design)[0]), nc, k, penalty)
    res = solve_grid(s, lambda_grid)
    return nr.pick_gcv(res, lambda_grid)


def ldlt_solve(a, b) -> np.ndarray:
    """Eigen-style pivoted LDL^T solve of a symmetric system (the LLT fallback)."""
    a = np.array(a, np.float64, order="C", copy=True)
    b = np.ascontiguousarray(b, np.float64)
    x = np.zeros_like(b)
    if lib().of_ldlt_solve(a.shape[0], ptr(a), ptr(b), ptr(x)):
        raise MemoryError("of_ldlt_solve")
    return x
