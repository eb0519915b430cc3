"""FP64 NumPy restatement of the reference hot path -- TEST INFRASTRUCTURE ONLY.

Every function cites the reference file:line it restates (paths are relative to
the tkillestein/delta 1.1.1 source tree). Where the reference computes in
float32 the restatement notes it; quantities the reference keeps in float64
(basis taps, thin-plate design, lattice, solver) are float64 here.

Only tests/, __graft_entry__.smoke() and bench.py's CPU legs may import this.
"""

from __future__ import annotations

import math
import os

import numpy as np
import scipy.linalg

MASK_GOOD = 0
MASK_BAD = 1
MASK_SATURATED = 2
MASK_COSMIC = 4
MASK_NONFINITE = 8
MASK_EDGE = 16
MASK_USER = 32

FWHM_PER_SIGMA = 2.354820045030949

# ---------------------------------------------------------------------------
# Gauss-Hermite basis (src/basis.cpp)
# ---------------------------------------------------------------------------


def default_radius(beta: float, n_max: int) -> int:
    """src/basis.cpp:9-12."""
    return max(int(math.ceil(3.0 * (beta * math.sqrt(n_max + 1.0)))), 3)


def resolve_radius(beta: float, n_max: int, radius: int) -> int:
    """src/bindings.cpp:98-101."""
    return radius if radius > 0 else default_radius(beta, n_max)


def gauss_hermite_basis1d(beta: float, n_max: int, radius: int) -> np.ndarray:
    """Sampled 1-D Gauss-Hermite functions, (n_max+1, 2r+1) float64.

    src/basis.cpp:14-50 (log-normalisation + physicists' Hermite recurrence).
    """
    if beta <= 0:
        raise ValueError("beta must be > 0")
    if n_max < 0:
        raise ValueError("n_max must be >= 0")
    if radius < 1:
        raise ValueError("radius must be >= 1")
    ks = 2 * radius + 1
    ln2 = math.log(2.0)
    half_ln_pi = 0.5 * math.log(math.pi)
    ln_beta = math.log(beta)
    log_norm = [-0.5 * (n * ln2 + math.lgamma(n + 1.0) + half_ln_pi + ln_beta) for n in range(n_max + 1)]
    out = np.zeros((n_max + 1, ks))
    for i in range(ks):
        t = (i - radius) / beta
        g = math.exp(-0.5 * t * t)
        h_prev = 1.0
        out[0, i] = math.exp(log_norm[0]) * h_prev * g
        if n_max >= 1:
            h_curr = 2.0 * t
            out[1, i] = math.exp(log_norm[1]) * h_curr * g
            for n in range(2, n_max + 1):
                h_next = 2.0 * t * h_curr - 2.0 * (n - 1) * h_prev
                out[n, i] = math.exp(log_norm[n]) * h_next * g
                h_prev, h_curr = h_curr, h_next
    return out


def basis_orders(n_max: int) -> list[tuple[int, int]]:
    """Component -> (nx, ny), by total order then ny.  src/basis.cpp:53-58."""
    return [(total - ny, ny) for total in range(n_max + 1) for ny in range(total + 1)]


def kernel2d(b1d: np.ndarray, orders, c: int) -> np.ndarray:
    """float32 ks x ks footprint float(gy[iy]*gx[ix]).  src/basis.cpp:66-79."""
    nx, ny = orders[c]
    return np.outer(b1d[ny], b1d[nx]).astype(np.float32)


def component_sums(b1d: np.ndarray, orders) -> np.ndarray:
    """S_c = (sum g_nx)(sum g_ny).  src/basis.cpp:81-93."""
    s = b1d.sum(axis=1)
    return np.array([s[nx] * s[ny] for nx, ny in orders])


# ---------------------------------------------------------------------------
# Thin-plate regression spline (src/spatial.cpp)
# ---------------------------------------------------------------------------


def tps_green(r2: np.ndarray) -> np.ndarray:
    """U = 0.5 r^2 log r^2, 0 at r=0.  src/spatial.cpp:13-16."""
    r2 = np.asarray(r2, dtype=np.float64)
    out = np.zeros_like(r2)
    pos = r2 > 0
    out[pos] = 0.5 * r2[pos] * np.log(r2[pos])
    return out


class ThinPlate:
    """src/spatial.cpp:20-111 (normalisation, QR null space, penalty, design)."""

    def __init__(self, knots):
        knots = np.asarray(knots, dtype=np.float64)
        if knots.ndim != 2 or knots.shape[1] != 2:
            raise ValueError("knots must be (k, 2)")
        k = knots.shape[0]
        if k < 3:
            raise ValueError("need at least 3 knots")
        self.cx = knots[:, 0].mean()
        self.cy = knots[:, 1].mean()
        sx = np.abs(knots[:, 0] - self.cx).max()
        sy = np.abs(knots[:, 1] - self.cy).max()
        self.scale = max(sx, sy, 1e-12)
        self.kn = np.column_stack([(knots[:, 0] - self.cx) / self.scale, (knots[:, 1] - self.cy) / self.scale])
        dx = self.kn[:, 0][:, None] - self.kn[:, 0][None, :]
        dy = self.kn[:, 1][:, None] - self.kn[:, 1][None, :]
        e = tps_green(dx * dx + dy * dy)
        t = np.column_stack([np.ones(k), self.kn[:, 0], self.kn[:, 1]])
        # LAPACK's Householder QR uses the same reflector sign convention as
        # Eigen's HouseholderQR (beta = -sign(alpha)||x||), so Q (hence Z) agree.
        q, _ = np.linalg.qr(t, mode="complete")
        self.z = q[:, 3:]
        pen = np.zeros((k, k))
        if k > 3:
            pen[: k - 3, : k - 3] = self.z.T @ e @ self.z
        self.penalty = 0.5 * (pen + pen.T)
        self.k = k

    def design(self, points) -> np.ndarray:
        """[radial . Z | 1, u, v].  src/spatial.cpp:67-97."""
        points = np.asarray(points, dtype=np.float64)
        ux = (points[:, 0] - self.cx) / self.scale
        uy = (points[:, 1] - self.cy) / self.scale
        dx = ux[:, None] - self.kn[:, 0][None, :]
        dy = uy[:, None] - self.kn[:, 1][None, :]
        sigma = tps_green(dx * dx + dy * dy)
        m = points.shape[0]
        d = np.empty((m, self.k))
        nr = self.k - 3
        if nr > 0:
            d[:, :nr] = sigma @ self.z
        d[:, nr] = 1.0
        d[:, nr + 1] = ux
        d[:, nr + 2] = uy
        return d

    def min_knot_spacing(self) -> float:
        """src/spatial.cpp:99-111."""
        best = math.inf
        for i in range(self.k):
            for j in range(i + 1, self.k):
                dx = self.kn[i, 0] - self.kn[j, 0]
                dy = self.kn[i, 1] - self.kn[j, 1]
                best = min(best, dx * dx + dy * dy)
        return math.sqrt(best) * self.scale if math.isfinite(best) else 0.0


def grid_knots(x0, y0, x1, y1, nx, ny) -> np.ndarray:
    """src/spatial.cpp:113-129."""
    if nx < 1 or ny < 1:
        raise ValueError("nx, ny must be >= 1")
    out = np.empty((nx * ny, 2))
    idx = 0
    for iy in range(ny):
        fy = 0.5 if ny == 1 else iy / (ny - 1)
        y = y0 + fy * (y1 - y0)
        for ix in range(nx):
            fx = 0.5 if nx == 1 else ix / (nx - 1)
            out[idx, 0] = x0 + fx * (x1 - x0)
            out[idx, 1] = y
            idx += 1
    return out


def tps_fit(knots, points, values, lam):
    """src/spatial.cpp:131-140 (LDLT solve -> plain solve here)."""
    tp = ThinPlate(knots)
    d = tp.design(points)
    a = d.T @ d + lam * tp.penalty
    return np.linalg.solve(a, d.T @ np.asarray(values, float))


# ---------------------------------------------------------------------------
# Spatial fields: coarse lattice + float32 bilinear blend (src/subtract.cpp)
# ---------------------------------------------------------------------------

K_SAMPLES_PER_KNOT_INTERVAL = 16
K_MAX_FIELD_STRIDE = 64
K_MIN_FIELD_STRIDE = 4


def choose_field_stride(tp: ThinPlate) -> int:
    """src/subtract.cpp:119-124."""
    spacing = tp.min_knot_spacing()
    if not spacing > 0.0:
        return 1
    s = int(spacing / K_SAMPLES_PER_KNOT_INTERVAL)
    return min(max(s, 1), K_MAX_FIELD_STRIDE)


def coarse_coords(length: int, stride: int) -> list[int]:
    """src/subtract.cpp:151-156."""
    g = list(range(0, length - 1, stride))
    g.append(length - 1)
    return g


class Fields:
    """a_n(x,y), b(x,y) exactly as subtract.cpp evaluates them.

    Coarse path: FP64 lattice design*C, float32 bilinear ramp
    (src/subtract.cpp:167-316); exact path for small frames
    (src/subtract.cpp:126-147, 266-275).
    """

    def __init__(self, knots, theta, n_components: int, w: int, h: int):
        self.tp = ThinPlate(knots)
        k = self.tp.k
        nf = n_components + 1
        theta = np.asarray(theta, dtype=np.float64)
        if theta.size != k * nf:
            raise RuntimeError("subtract: theta size does not match k*(nc+1)")
        self.c = theta.reshape(nf, k).T  # (k, nf): column j = theta[j*k:(j+1)*k]
        self.nc = n_components
        self.w, self.h = w, h
        stride = choose_field_stride(self.tp)
        self.stride = stride
        self.exact = stride < K_MIN_FIELD_STRIDE or w <= 2 * stride or h <= 2 * stride
        if self.exact:
            return
        self.gx = coarse_coords(w, stride)
        self.gy = coarse_coords(h, stride)
        ncx, ncy = len(self.gx), len(self.gy)
        self.ncx, self.ncy = ncx, ncy
        pts = np.array([(float(x), float(y)) for y in self.gy for x in self.gx])
        lat = self.tp.design(pts) @ self.c  # (ncy*ncx, nf)
        self.coarse = lat.T.reshape(nf, ncy, ncx).copy()  # [f, iy, ix] float64
        self.cellx = np.minimum(np.arange(w) // stride, ncx - 2)
        gxa = np.array(self.gx)
        x0 = gxa[self.cellx]
        x1 = gxa[self.cellx + 1]
        self.wx = np.where(x1 > x0, (np.arange(w) - x0).astype(np.float32) / (x1 - x0).astype(np.float32), 0.0).astype(np.float32)
        self.celly = np.minimum(np.arange(h) // stride, ncy - 2)
        gya = np.array(self.gy)
        y0 = gya[self.celly]
        y1 = gya[self.celly + 1]
        self.wy = np.where(y1 > y0, (np.arange(h) - y0).astype(np.float32) / (y1 - y0).astype(np.float32), 0.0).astype(np.float32)

    def field_full(self, f: int) -> np.ndarray:
        """Full-resolution float32 field f (f == nc is the background)."""
        if self.exact:
            ys, xs = np.mgrid[0 : self.h, 0 : self.w]
            pts = np.column_stack([xs.ravel().astype(float), ys.ravel().astype(float)])
            vals = self.tp.design(pts) @ self.c[:, f]
            return vals.reshape(self.h, self.w).astype(np.float32)
        c = self.coarse[f].astype(np.float32)
        jy = self.celly
        jx = self.cellx
        a00 = c[jy][:, jx]
        a01 = c[jy][:, jx + 1]
        a10 = c[jy + 1][:, jx]
        a11 = c[jy + 1][:, jx + 1]
        fy = self.wy[:, None].astype(np.float64)
        # float32 blend of src/subtract.cpp:196-204, evaluated in float64 and
        # rounded (differs from the FMA-contracted float path by <= 1 ulp).
        a00d, a01d, a10d, a11d = (a.astype(np.float64) for a in (a00, a01, a10, a11))
        base = (a00d + (a10d - a00d) * fy).astype(np.float32).astype(np.float64)
        top = (a01d - a00d)
        slope = (top + ((a11d - a10d) - top) * fy).astype(np.float32).astype(np.float64)
        return (base + slope * self.wx[None, :].astype(np.float64)).astype(np.float32)

    def point(self, f: int, x: int, y: int) -> float:
        """src/subtract.cpp:187-205, in float32 arithmetic."""
        if self.exact:
            vals = self.tp.design(np.array([[float(x), float(y)]])) @ self.c[:, f]
            return np.float32(vals[0])
        f32 = np.float32
        jx, jy = self.cellx[x], self.celly[y]
        a00 = f32(self.coarse[f, jy, jx])
        a01 = f32(self.coarse[f, jy, jx + 1])
        a10 = f32(self.coarse[f, jy + 1, jx])
        a11 = f32(self.coarse[f, jy + 1, jx + 1])
        fy = self.wy[y]
        base = f32(a00 + (a10 - a00) * fy)
        top = f32(a01 - a00)
        slope = f32(top + ((a11 - a10) - top) * fy)
        return f32(base + slope * self.wx[x])


def photometric_scale(knots, theta, sums, h, w) -> np.ndarray:
    """src/fit.cpp:513-530 (evaluate_fields + sum_n S_n a_n in float32)."""
    nc = len(sums)
    fl = Fields(knots, theta, nc, w, h)
    out = np.zeros((h, w), np.float32)
    for c in range(nc):
        out = (out + np.float32(sums[c]) * fl.field_full(c)).astype(np.float32)
    return out


def photometric_scale_at(knots, theta, sums, points) -> np.ndarray:
    """src/fit.cpp:532-544."""
    tp = ThinPlate(knots)
    nc = len(sums)
    c = np.asarray(theta, float).reshape(nc + 1, tp.k).T
    fields = tp.design(points) @ c
    return fields[:, :nc] @ np.asarray(sums, float)


# ---------------------------------------------------------------------------
# Order statistics (std::nth_element upper median)
# ---------------------------------------------------------------------------


def upper_median(sample: np.ndarray):
    """sample[size/2] of the sorted sample (nth_element semantics)."""
    if sample.size == 0:
        return None
    return np.partition(sample, sample.size // 2)[sample.size // 2]


def reference_fill_value(ref: np.ndarray, ref_mask) -> np.float32:
    """Upper median of good finite R[7j].  src/subtract.cpp:20-51."""
    flat = np.ascontiguousarray(ref, dtype=np.float32).ravel()
    v = flat[::7]
    ok = np.isfinite(v)
    if ref_mask is not None:
        ok &= np.ascontiguousarray(ref_mask).ravel()[::7] == 0
    med = upper_median(v[ok])
    return np.float32(0.0) if med is None else np.float32(med)


# ---------------------------------------------------------------------------
# Convolution engine (src/convolve.cpp), float64 accumulation of float32 inputs
# ---------------------------------------------------------------------------


def convolve_x(img: np.ndarray, k: np.ndarray) -> np.ndarray:
    """out[y,x] = sum_j k[j] in[y, x+h-j], zero-padded.  src/convolve.cpp:24-52."""
    img = np.asarray(img, dtype=np.float64)
    ks = k.size
    hh = (ks - 1) // 2
    h, w = img.shape
    pad = np.zeros((h, w + 2 * hh))
    pad[:, hh : hh + w] = img
    out = np.zeros((h, w))
    for j in range(ks):
        sh = hh - j  # src index x + sh
        out += float(k[j]) * pad[:, hh + sh : hh + sh + w]
    return out


def convolve_y(img: np.ndarray, k: np.ndarray) -> np.ndarray:
    """out[y,x] = sum_j k[j] in[y+h-j, x], zero-padded.  src/convolve.cpp:57-83."""
    return convolve_x(np.asarray(img).T, k).T


def basis_convolve(image: np.ndarray, beta: float, n_max: int, radius: int = 0) -> np.ndarray:
    """(nc, H, W) B_n stack.  src/convolve.cpp:90-113 (float32 taps)."""
    r = resolve_radius(beta, n_max, radius)
    b1d = gauss_hermite_basis1d(beta, n_max, r)
    k1 = b1d.astype(np.float32)
    tx = [convolve_x(image, k1[n]) for n in range(n_max + 1)]
    return np.stack([convolve_y(tx[nx], k1[ny]) for nx, ny in basis_orders(n_max)])


# ---------------------------------------------------------------------------
# Full-frame subtraction (src/subtract.cpp:429-966)
# ---------------------------------------------------------------------------


def sanitized_reference(ref, ref_mask, fill):
    """Masked / non-finite reference pixels -> fill.  src/subtract.cpp:543-568."""
    r = np.array(ref, dtype=np.float32, copy=True)
    bad = ~np.isfinite(r)
    if ref_mask is not None:
        bad |= ref_mask != 0
    r[bad] = fill
    return r


def dilate_mask(mask: np.ndarray, r: int) -> np.ndarray:
    """Separable OR-dilation by Chebyshev radius r.  src/subtract.cpp:70-101."""
    if r <= 0:
        return mask.copy()
    h, w = mask.shape
    tmp = np.zeros_like(mask)
    for d in range(-r, r + 1):
        lo, hi = max(0, -d), min(w, w - d)
        tmp[:, lo:hi] |= mask[:, lo + d : hi + d]
    out = np.zeros_like(mask)
    for d in range(-r, r + 1):
        lo, hi = max(0, -d), min(h, h - d)
        out[lo:hi, :] |= tmp[lo + d : hi + d, :]
    return out


def _block_effective_kernel(fl: Fields, phi, nc, cpx, cpy):
    """K = sum_n a_n phi_n at (cpx,cpy), float32.  src/subtract.cpp:700-705."""
    k2 = np.zeros_like(phi[0])
    for n in range(nc):
        an = fl.point(n, cpx, cpy)
        k2 = (k2 + np.float32(an) * phi[n]).astype(np.float32)
    return k2


def variance_reference_term(fl: Fields, phi, nc, rk, var_r: np.ndarray) -> np.ndarray:
    """Block-effective K^2 (x) Var(R) with box shrink and flat shortcut.

    src/subtract.cpp:647-818 (64x64 blocks, kVarFlatTol 1e-3f, kVarBoxTol 1e-4f).
    Accumulated in float64 here.
    """
    h, w = var_r.shape
    ks = 2 * rk + 1
    out = np.zeros((h, w))
    pad = np.zeros((h + 2 * rk, w + 2 * rk), np.float32)
    pad[rk : rk + h, rk : rk + w] = var_r
    bsz = 64
    tol_box = 1.0 - float(np.float32(1e-4))
    for by in range(0, h, bsz):
        for bx in range(0, w, bsz):
            bw = min(bsz, w - bx)
            bh = min(bsz, h - by)
            cpx = min(bx + bw // 2, w - 1)
            cpy = min(by + bh // 2, h - 1)
            k2 = _block_effective_kernel(fl, phi, nc, cpx, cpy)
            kf = (k2 * k2).astype(np.float32)[::-1, ::-1]
            qsum = float(np.sum(k2.astype(np.float64) ** 2))
            hw = 0
            target = tol_box * qsum
            while hw < rk:
                lo, hi = rk - hw, rk + hw
                box = float(np.sum(kf[lo : hi + 1, lo : hi + 1].astype(np.float64)))
                if box >= target:
                    break
                hw += 1
            lo, hi = rk - hw, rk + hw
            win = pad[by : by + bh + 2 * rk, bx : bx + bw + 2 * rk]
            wmin = float(win.min())
            wmax = float(win.max())
            if wmax > 0.0 and np.float32(wmax - wmin) <= np.float32(1e-3) * np.float32(wmax):
                q = float(np.float32(qsum))
                out[by : by + bh, bx : bx + bw] = q * win[rk : rk + bh, rk : rk + bw]
                continue
            acc = np.zeros((bh, bw))
            for ly in range(lo, hi + 1):
                for lx in range(lo, hi + 1):
                    c = float(kf[ly, lx])
                    if c == 0.0:
                        continue
                    acc += c * win[ly : ly + bh, lx : lx + bw]
            out[by : by + bh, bx : bx + bw] = acc
    return out


def subtract(science, reference, knots, theta, beta, n_max, radius=0, saturation=0.0,
             science_var=None, reference_var=None, science_mask=None, reference_mask=None):
    """delta::subtract restated (src/subtract.cpp:429-966); returns the _core dict.

    Model and variance are accumulated in float64 from the float32 taps,
    fields and sanitised reference, then rounded to float32.
    """
    sci = np.ascontiguousarray(science, dtype=np.float32)
    ref = np.ascontiguousarray(reference, dtype=np.float32)
    if sci.shape != ref.shape:
        raise RuntimeError("subtract: science/reference shape mismatch")
    h, w = sci.shape
    r = resolve_radius(beta, n_max, radius)
    b1d = gauss_hermite_basis1d(beta, n_max, r)
    orders = basis_orders(n_max)
    nc = len(orders)
    fl = Fields(knots, theta, nc, w, h)
    fill = reference_fill_value(ref, reference_mask)
    clean = sanitized_reference(ref, reference_mask, fill)
    k1 = b1d.astype(np.float32)
    tx = [convolve_x(clean, k1[nx]) for nx in range(n_max + 1)]
    model = fl.field_full(nc).astype(np.float64)
    for n, (nx, ny) in enumerate(orders):
        bn = convolve_y(tx[nx], k1[ny])
        model += fl.field_full(n).astype(np.float64) * bn
    diff = sci.astype(np.float64) - model
    out = {"difference": diff.astype(np.float32), "variance": None, "mask": None}

    if reference_var is not None or science_var is not None:
        var = np.zeros((h, w))
        if reference_var is not None:
            phi = [kernel2d(b1d, orders, c) for c in range(nc)]
            var += variance_reference_term(fl, phi, nc, r, np.asarray(reference_var, np.float32))
        if science_var is not None:
            var += np.asarray(science_var, np.float64)
        out["variance"] = var.astype(np.float32)

    if reference_mask is not None or science_mask is not None or saturation > 0.0:
        d = out["difference"]
        direct = np.zeros((h, w), np.uint8)
        grow = np.zeros((h, w), np.uint8)
        exact_bad = np.zeros((h, w), bool)
        if science_mask is not None:
            sm = np.asarray(science_mask, np.uint8)
            direct |= sm
            exact_bad |= sm != 0
        if reference_mask is not None:
            rm = np.asarray(reference_mask, np.uint8)
            grow |= rm
            exact_bad |= rm != 0
        if saturation > 0.0:
            sat = np.float32(saturation)
            rs = ref >= sat
            ss = sci >= sat
            grow[rs] |= MASK_SATURATED
            direct[ss] |= MASK_SATURATED
            exact_bad |= rs | ss
        mask = direct | dilate_mask(grow, r)
        ys, xs = np.mgrid[0:h, 0:w]
        edge = (xs < r) | (xs >= w - r) | (ys < r) | (ys >= h - r)
        mask[edge] |= MASK_EDGE
        nonfin = ~np.isfinite(d)
        mask[nonfin] |= MASK_NONFINITE
        exact_bad |= nonfin
        flat_d = d.ravel()
        flat_m = mask.ravel()
        samp_d = flat_d[::7]
        samp_ok = (flat_m[::7] == 0) & np.isfinite(samp_d)
        med = upper_median(samp_d[samp_ok])
        fill_d = np.float32(0.0) if med is None else np.float32(med)
        fix = (mask != 0) & exact_bad
        d = d.copy()
        d[fix] = fill_d
        out["difference"] = d
        if out["variance"] is not None:
            v = out["variance"].copy()
            v[fix] = 0.0
            out["variance"] = v
        out["mask"] = mask
    return out


# ---------------------------------------------------------------------------
# Penalised GLS (src/solve.cpp)
# ---------------------------------------------------------------------------


def make_pen_half(pen: np.ndarray, nc: int, k: int) -> np.ndarray:
    """F with F F^T = P0, from the k x k penalty eigenpairs.  src/solve.cpp:47-65."""
    wv, v = np.linalg.eigh(pen)
    wmax = np.abs(wv).max() if wv.size else 0.0
    tol = wmax * k * np.finfo(float).eps
    keep = np.nonzero(wv > tol)[0]
    fk = v[:, keep] * np.sqrt(wv[keep])
    r = keep.size
    p = (nc + 1) * k
    f = np.zeros((p, (nc + 1) * r))
    for b in range(nc + 1):
        f[b * k : (b + 1) * k, b * r : (b + 1) * r] = fk
    return f


class System:
    """M = Xs^T Xs, rhs, ywy, P0, F.  src/solve.cpp:28-42, 70-145."""

    def __init__(self, design, target, weights, bn, penalty):
        design = np.asarray(design, float)
        target = np.asarray(target, float)
        weights = np.asarray(weights, float)
        bn = np.asarray(bn, float)
        n, k = design.shape
        nc = bn.shape[1]
        if target.size != n or weights.size != n or bn.shape[0] != n:
            raise RuntimeError("solve_gls: row counts of design/target/weights/bn disagree")
        sw = np.sqrt(weights)
        blocks = [design * (bn[:, c] * sw)[:, None] for c in range(nc)] + [design * sw[:, None]]
        xs = np.concatenate(blocks, axis=1)
        ds = sw * target
        self.m = xs.T @ xs
        self.rhs = xs.T @ ds
        self.ywy = float(np.sum(weights * target * target))
        self.n, self.nc, self.k = n, nc, k
        self.p = (nc + 1) * k
        self.p0 = np.kron(np.eye(nc + 1), penalty)
        self.pen_half = make_pen_half(penalty, nc, k)

    @classmethod
    def from_parts(cls, m, rhs, ywy, n, nc, k, penalty):
        s = cls.__new__(cls)
        s.m, s.rhs, s.ywy = m, rhs, float(ywy)
        s.n, s.nc, s.k = n, nc, k
        s.p = (nc + 1) * k
        s.p0 = np.kron(np.eye(nc + 1), penalty)
        s.pen_half = make_pen_half(penalty, nc, k)
        return s


def ldlt_factor(a):
    """Eigen 3.4's pivoted LDL^T (the reference's LLT fallback, src/solve.cpp:177-181).

    Step k swaps the remaining diagonal entry of largest magnitude (first on
    ties, read before that step's update) to position k, forms d_k and
    column k of the unit lower factor by the left-looking update, and divides
    the column by d_k only when d_k != 0. An all-zero diagonal stops at once
    with identity transpositions. Returns (factor with L below and D on the
    diagonal, transpositions)."""
    a = np.array(a, np.float64, copy=True)
    p = a.shape[0]
    perm = np.arange(p)
    for k in range(p):
        diag = np.abs(np.diagonal(a)[k:])
        piv = k + int(np.argmax(diag))
        if k == 0 and diag[piv] == 0.0:
            return a, np.arange(p)
        perm[k] = piv
        if piv != k:
            a[[k, piv], :] = a[[piv, k], :]
            a[:, [k, piv]] = a[:, [piv, k]]
        temp = np.diagonal(a)[:k] * a[k, :k]
        dk = a[k, k] - float(a[k, :k] @ temp)
        a[k, k] = dk
        col = a[k + 1 :, k] - a[k + 1 :, :k] @ temp
        a[k + 1 :, k] = col / dk if dk != 0.0 else col
    return a, perm


def ldlt_solve(fac, perm, b):
    """Solve with an ldlt_factor result; D enters by its pseudo-inverse
    (1/d where |d| > the smallest normal double, else 0), as Eigen's solve."""
    x = np.array(b, np.float64, copy=True)
    p = fac.shape[0]
    for k in range(p):
        x[[k, perm[k]]] = x[[perm[k], k]]
    low = np.tril(fac, -1) + np.eye(p)
    x = scipy.linalg.solve_triangular(low, x, lower=True, unit_diagonal=True)
    d = np.diagonal(fac)
    inv = np.where(np.abs(d) > np.finfo(np.float64).tiny, 1.0 / np.where(d == 0.0, 1.0, d), 0.0)
    x = (x.T * inv).T
    x = scipy.linalg.solve_triangular(low.T, x, lower=False, unit_diagonal=True)
    for k in range(p - 1, -1, -1):
        x[[k, perm[k]]] = x[[perm[k], k]]
    return x


def solve_at(s: System, lam: float) -> dict:
    """LLT (LDLT fallback), theta, edf, rss, gcv.  src/solve.cpp:147-193."""
    a = s.m + lam * s.p0
    try:
        chol = np.linalg.cholesky(a)
        y = np.linalg.solve(chol, s.rhs)
        theta = np.linalg.solve(chol.T, y)
        if s.pen_half.size > 0:
            lf = np.linalg.solve(chol, s.pen_half)
            edf = s.p - lam * float(np.sum(lf * lf))
        else:
            edf = float(np.trace(np.linalg.solve(a, s.m)))
    except np.linalg.LinAlgError:
        fac, perm = ldlt_factor(a)
        theta = ldlt_solve(fac, perm, s.rhs)
        edf = float(np.trace(ldlt_solve(fac, perm, s.m)))
    rss = s.ywy - 2.0 * float(theta @ s.rhs) + float(theta @ (s.m @ theta))
    rss = max(rss, 0.0)
    denom = s.n - edf
    gcv = s.n * rss / (denom * denom) if denom > 0 else math.inf
    return {"theta": theta, "lambda": lam, "effective_dof": edf, "rss": rss, "gcv": gcv,
            "n_components": s.nc, "n_spatial": s.k}


def solve_gls_gcv_system(s: System, lambda_grid) -> dict:
    """Grid search on GCV.  src/solve.cpp:227-262."""
    grid = [float(v) for v in lambda_grid]
    if not grid:
        raise RuntimeError("solve_gls_gcv: lambda_grid is empty")
    return pick_gcv([solve_at(s, lam) for lam in grid], grid)


def pick_gcv(res, lambda_grid) -> dict:
    """First minimum of the GCV curve over the grid's solutions.  src/solve.cpp:240-262."""
    grid = [float(v) for v in lambda_grid]
    curve = np.array([r["gcv"] for r in res])
    best_i = 0
    best = math.inf
    for i, g in enumerate(curve):
        if g < best:
            best, best_i = g, i
    out = dict(res[best_i])
    out["lambda_grid"] = np.array(grid)
    out["gcv_curve"] = curve
    return out


def solve_gls(knots, points, target, weights, bn, lam) -> dict:
    """src/solve.cpp:208-215."""
    tp = ThinPlate(knots)
    s = System(tp.design(points), target, weights, bn, tp.penalty)
    out = solve_at(s, float(lam))
    out["lambda_grid"] = np.zeros(0)
    out["gcv_curve"] = np.zeros(0)
    return out


def solve_gls_gcv(knots, points, target, weights, bn, lambda_grid) -> dict:
    """src/solve.cpp:217-225."""
    tp = ThinPlate(knots)
    return solve_gls_gcv_system(System(tp.design(points), target, weights, bn, tp.penalty), lambda_grid)


def cv_finish(mf, rf, ysq, n_groups, penalty, n, nc, k, lambda_grid, warm_start=-1) -> dict:
    """Group-CV lambda search + final all-data fit.  src/solve.cpp:271-417."""
    m_all = sum(mf)
    r_all = sum(rf)
    s = System.from_parts(m_all, r_all, sum(ysq), n, nc, k, penalty)
    grid = [float(v) for v in lambda_grid]
    nl = len(grid)
    curve = np.full(nl, math.inf)
    done = np.zeros(nl, bool)
    m_train = [m_all - mf[g] for g in range(n_groups)]
    r_train = [r_all - rf[g] for g in range(n_groups)]

    def evaluate(idx):
        for li in idx:
            tot = 0.0
            for g in range(n_groups):
                a = m_train[g] + grid[li] * s.p0
                try:
                    chol = np.linalg.cholesky(a)
                    th = np.linalg.solve(chol.T, np.linalg.solve(chol, r_train[g]))
                except np.linalg.LinAlgError:
                    fac, perm = ldlt_factor(a)  # src/solve.cpp:328-333
                    th = ldlt_solve(fac, perm, r_train[g])
                e = ysq[g] - 2.0 * float(th @ rf[g]) + float(th @ (mf[g] @ th))
                tot += e if e > 0.0 else 0.0
            curve[li] = tot
            done[li] = True

    def argmin_done():
        b, bc = -1, math.inf
        for li in range(nl):
            if done[li] and curve[li] < bc:
                bc, b = curve[li], li
        return b

    if 0 <= warm_start < nl:
        evaluate(list(range(max(0, warm_start - 1), min(nl - 1, warm_start + 1) + 1)))
        while True:
            b = argmin_done()
            step = []
            if b > 0 and not done[b - 1]:
                step.append(b - 1)
            if b < nl - 1 and not done[b + 1]:
                step.append(b + 1)
            if not step:
                break
            evaluate(step)
    else:
        coarse = list(range(0, nl, 2))
        if not coarse or coarse[-1] != nl - 1:
            coarse.append(nl - 1)
        evaluate(coarse)
        cb = coarse[0]
        for li in coarse:
            if curve[li] < curve[cb]:
                cb = li
        refine = [li for li in range(max(0, cb - 2), min(nl - 1, cb + 2) + 1) if not done[li]]
        if refine:
            evaluate(refine)
    best_i, best = 0, math.inf
    for li in range(nl):
        if done[li] and curve[li] < best:
            best, best_i = curve[li], li
    out = solve_at(s, grid[best_i])
    out["lambda_grid"] = np.array(grid)
    out["gcv_curve"] = curve
    return out


def solve_gls_cv_design(design, target, weights, bn, penalty, lambda_grid, group, n_groups, warm_start=-1):
    """Exact per-fold build.  src/solve.cpp:433-560."""
    design = np.asarray(design, float)
    n, k = design.shape
    group = np.asarray(group)
    if group.size != n:
        raise RuntimeError("solve_gls_cv: group.size() must match points.rows()")
    if n_groups < 2:
        return solve_gls_gcv_system(System(design, target, weights, bn, penalty), lambda_grid)
    if np.any((group < 0) | (group >= n_groups)):
        raise RuntimeError("solve_gls_cv: group id out of range")
    bn = np.asarray(bn, float)
    nc = bn.shape[1]
    mf, rf, ysq = [], [], []
    for g in range(n_groups):
        sel = group == g
        s = System(design[sel], np.asarray(target, float)[sel], np.asarray(weights, float)[sel], bn[sel], penalty)
        mf.append(s.m)
        rf.append(s.rhs)
        ysq.append(s.ywy)
    return cv_finish(mf, rf, ysq, n_groups, penalty, n, nc, k, lambda_grid, warm_start)


def solve_gls_cv(knots, points, target, weights, bn, lambda_grid, group, n_groups, warm_start=-1):
    """src/solve.cpp:421-431."""
    tp = ThinPlate(knots)
    return solve_gls_cv_design(tp.design(points), target, weights, bn, tp.penalty, lambda_grid, group, n_groups, warm_start)


def solve_gls_cv_stamped(target, weights, bn, stamp_design, stamp_id, stamp_fold, penalty, lambda_grid, n_groups, warm_start=-1):
    """Per-stamp Kronecker factorised CV.  src/solve.cpp:562-633."""
    target = np.asarray(target, float)
    weights = np.asarray(weights, float)
    bn = np.asarray(bn, float)
    n = target.size
    nc = bn.shape[1]
    nf = nc + 1
    ns, k = stamp_design.shape
    p = nf * k
    a_st = np.zeros((ns, nf, nf))
    r_st = np.zeros((ns, nf))
    ds2 = np.zeros(ns)
    b = np.concatenate([bn, np.ones((n, 1))], axis=1)
    for i in range(n):
        s = stamp_id[i]
        a_st[s] += weights[i] * np.outer(b[i], b[i])
        r_st[s] += weights[i] * target[i] * b[i]
        ds2[s] += weights[i] * target[i] * target[i]
    mf = [np.zeros((p, p)) for _ in range(n_groups)]
    rf = [np.zeros(p) for _ in range(n_groups)]
    ysq = [0.0] * n_groups
    for s in range(ns):
        g = stamp_fold[s]
        d = stamp_design[s]
        mf[g] += np.kron(a_st[s], np.outer(d, d))
        rf[g] += np.kron(r_st[s], d)
        ysq[g] += ds2[s]
    return cv_finish(mf, rf, ysq, n_groups, penalty, n, nc, k, lambda_grid, warm_start)


# ---------------------------------------------------------------------------
# Stamp fit (src/fit.cpp)
# ---------------------------------------------------------------------------


def conv_var_at(x, y, k2, ks, r, var, mask) -> float:
    """(K^2 (x) Var)(x,y), masked / non-positive skipped.  src/fit.cpp:38-59."""
    h, w = var.shape
    acc = 0.0
    for dv in range(-r, r + 1):
        sy = y - dv
        if sy < 0 or sy >= h:
            continue
        for du in range(-r, r + 1):
            sx = x - du
            if sx < 0 or sx >= w:
                continue
            if mask is not None and mask[sy, sx] != 0:
                continue
            v = var[sy, sx]
            if not (v > 0.0) or not np.isfinite(v):
                continue
            acc += float(k2[dv + r, du + r]) * float(v)
    return acc


def conv_var_window(k2, r, var, mask, x0, x1, y0, y1) -> np.ndarray:
    """conv_var_at over the window [y0..y1] x [x0..x1] at once (FP64 terms of
    the same float32 K^2 and Var samples; invalid samples contribute 0)."""
    h, w = var.shape
    ey0, ey1, ex0, ex1 = y0 - r, y1 + r, x0 - r, x1 + r
    pad = np.zeros((ey1 - ey0 + 1, ex1 - ex0 + 1), np.float64)
    sy0, sy1, sx0, sx1 = max(ey0, 0), min(ey1, h - 1), max(ex0, 0), min(ex1, w - 1)
    v = np.asarray(var[sy0 : sy1 + 1, sx0 : sx1 + 1], np.float64)
    ok = (v > 0.0) & np.isfinite(v)
    if mask is not None:
        ok &= mask[sy0 : sy1 + 1, sx0 : sx1 + 1] == 0
    pad[sy0 - ey0 : sy1 - ey0 + 1, sx0 - ex0 : sx1 - ex0 + 1] = np.where(ok, v, 0.0)
    ks = 2 * r + 1
    win = np.lib.stride_tricks.sliding_window_view(pad, (ks, ks))
    kf = np.asarray(k2, np.float64)[::-1, ::-1]
    return np.einsum("jiab,ab->ji", win, kf)


def gather_stamps(science, reference, stamp_x, stamp_y, stamp_radius, b1d, n_max, r,
                  science_var, reference_var, science_mask, reference_mask, basis_convolve_fn):
    """Stamp pixel gather + per-stamp B_n.  src/fit.cpp:83-229.

    ``basis_convolve_fn(patch) -> (nc, ph, pw)`` supplies the float32 B_n; the
    tests pass the reference-built convolve.cpp (oracle.refbuild) here.
    """
    h, w = science.shape
    have_var = science_var is not None or reference_var is not None
    have_cvar = reference_var is not None
    fill = reference_fill_value(reference, reference_mask)
    nc = len(basis_orders(n_max))
    rows = {"px": [], "py": [], "target": [], "var_t": [], "var_c": [], "bn": [], "stamp": []}
    stamp_cx, stamp_cy = [], []
    for cx, cy in zip(stamp_x, stamp_y):
        cx, cy = int(cx), int(cy)
        x0, x1 = max(0, cx - stamp_radius), min(w - 1, cx + stamp_radius)
        y0, y1 = max(0, cy - stamp_radius), min(h - 1, cy + stamp_radius)
        ex0, ex1 = max(0, x0 - r), min(w - 1, x1 + r)
        ey0, ey1 = max(0, y0 - r), min(h - 1, y1 + r)
        if ex1 < ex0 or ey1 < ey0:
            continue
        patch = sanitized_reference(reference[ey0 : ey1 + 1, ex0 : ex1 + 1],
                                    None if reference_mask is None else reference_mask[ey0 : ey1 + 1, ex0 : ex1 + 1], fill)
        bn = basis_convolve_fn(patch)
        sid = len(stamp_cx)
        # The stamp's pixels in raster order (y, then x), kept by the same tests
        # as the reference's per-pixel loop.
        ok = np.ones((y1 - y0 + 1, x1 - x0 + 1), bool)
        if science_mask is not None:
            ok &= science_mask[y0 : y1 + 1, x0 : x1 + 1] == 0
        if reference_mask is not None:
            ok &= reference_mask[y0 : y1 + 1, x0 : x1 + 1] == 0
        sv = science[y0 : y1 + 1, x0 : x1 + 1]
        ok &= np.isfinite(sv)
        vt = (np.asarray(science_var[y0 : y1 + 1, x0 : x1 + 1], np.float64) if science_var is not None
              else np.zeros(ok.shape))
        vc = (np.asarray(reference_var[y0 : y1 + 1, x0 : x1 + 1], np.float64) if have_cvar else np.zeros(ok.shape))
        if have_var:
            ok &= (vt + vc) > 0.0
        cols = bn[:, y0 - ey0 : y1 - ey0 + 1, x0 - ex0 : x1 - ex0 + 1]
        ok &= np.all(np.isfinite(cols), axis=0)
        yy, xx = np.nonzero(ok)
        used = yy.size > 0
        rows["px"].append((xx + x0).astype(np.float64))
        rows["py"].append((yy + y0).astype(np.float64))
        rows["target"].append(sv[yy, xx].astype(np.float64))
        rows["var_t"].append(vt[yy, xx])
        rows["var_c"].append(vc[yy, xx])
        rows["bn"].append(cols[:, yy, xx].T.astype(np.float64))
        rows["stamp"].append(np.full(yy.size, sid, np.int64))
        if used:
            stamp_cx.append(cx)
            stamp_cy.append(cy)
    out = {k: (np.concatenate(v) if v else np.zeros(0)) for k, v in rows.items() if k != "bn"}
    out["stamp"] = out["stamp"].astype(np.int64)
    out["bn"] = np.concatenate(rows["bn"]).reshape(-1, nc) if rows["bn"] else np.zeros((0, nc))
    out["stamp_cx"] = np.asarray(stamp_cx, int)
    out["stamp_cy"] = np.asarray(stamp_cy, int)
    return out


def fit_kernel(science, reference, knots, stamp_x, stamp_y, stamp_radius, beta, n_max, lambda_grid,
               radius=0, clip_sigma=4.0, clip_iterations=5, min_stamps=5, cv_folds=0,
               science_var=None, reference_var=None, science_mask=None, reference_mask=None,
               basis_convolve_fn=None, gcv_solver=None) -> dict:
    """delta::fit_kernel restated.  src/fit.cpp:63-511.

    ``gcv_solver(design, target, weights, bn, penalty, lambda_grid)`` replaces
    the NumPy GCV solve of each IRLS pass (the timed chain passes the C
    restatement, oracle.cref.gls_gcv)."""
    science = np.asarray(science, np.float32)
    reference = np.asarray(reference, np.float32)
    r = resolve_radius(beta, n_max, radius)
    b1d = gauss_hermite_basis1d(beta, n_max, r)
    orders = basis_orders(n_max)
    nc = len(orders)
    ks = 2 * r + 1
    if basis_convolve_fn is None:
        def basis_convolve_fn(patch):
            return basis_convolve(patch, beta, n_max, r).astype(np.float32)
    g = gather_stamps(science, reference, stamp_x, stamp_y, stamp_radius, b1d, n_max, r,
                      science_var, reference_var, science_mask, reference_mask, basis_convolve_fn)
    npix_all = g["target"].size
    if npix_all == 0:
        raise RuntimeError("fit_kernel: no usable stamp pixels")
    n_stamps = g["stamp_cx"].size
    tp = ThinPlate(knots)
    k = tp.k
    have_var = science_var is not None or reference_var is not None
    have_cvar = reference_var is not None
    phi = [kernel2d(b1d, orders, c) for c in range(nc)] if have_cvar else None
    weights = np.ones(npix_all)
    if have_var:
        weights = 1.0 / (g["var_t"] + g["var_c"])
    accepted = np.ones(n_stamps, np.uint8)
    stamp_chi2 = np.full(n_stamps, np.nan)
    clip_passes = clip_iterations if (clip_sigma > 0.0 and clip_iterations > 0) else 0
    do_iterate = 1 if clip_iterations > 0 else 0
    min_pass = 1 if (do_iterate and have_var) else 0
    hard_max = max(clip_passes, min_pass)
    floor_stamps = max(1, min(min_stamps, n_stamps))
    pts_all = np.column_stack([g["px"], g["py"]])
    design_all = tp.design(pts_all)
    warm_start = -1
    cv_exact_design_bytes = 0
    it = 0
    while True:
        rows = np.nonzero(accepted[g["stamp"]] != 0)[0]
        npix = rows.size
        if npix == 0:
            raise RuntimeError("fit_kernel: all stamp pixels clipped")
        tgt = g["target"][rows]
        wts = weights[rows]
        bn = g["bn"][rows]
        des = design_all[rows]
        if cv_folds > 1:
            spacing = tp.min_knot_spacing()
            stamp_width = 2.0 * stamp_radius + 1.0
            use_stamped = spacing > 0.0 and spacing >= 16.0 * stamp_width
            env = os.environ.get("DELTA_STAMP_APPROX")  # src/fit.cpp:327-328
            if env is not None:
                try:
                    use_stamped = int(env) != 0
                except ValueError:
                    use_stamped = False
            if use_stamped:
                gids = g["stamp"][rows]
                g2l = {}
                sx, sy, cnt, fold = [], [], [], []
                sid = np.empty(npix, int)
                for j in range(npix):
                    gid = int(gids[j])
                    if gid not in g2l:
                        g2l[gid] = len(sx)
                        sx.append(0.0)
                        sy.append(0.0)
                        cnt.append(0)
                        fold.append(gid % cv_folds)
                    loc = g2l[gid]
                    sid[j] = loc
                    sx[loc] += pts_all[rows[j], 0]
                    sy[loc] += pts_all[rows[j], 1]
                    cnt[loc] += 1
                cent = np.column_stack([np.array(sx) / np.array(cnt), np.array(sy) / np.array(cnt)])
                gls = solve_gls_cv_stamped(tgt, wts, bn, tp.design(cent), sid, fold, tp.penalty,
                                           lambda_grid, cv_folds, warm_start)
            else:
                grp = g["stamp"][rows] % cv_folds
                gls = solve_gls_cv_design(des, tgt, wts, bn, tp.penalty, lambda_grid, grp, cv_folds, warm_start)
                cv_exact_design_bytes = npix * (nc + 1) * k * 8
            warm_start = int(np.argmin(gls["gcv_curve"]))
        elif gcv_solver is not None:
            gls = gcv_solver(des, tgt, wts, bn, tp.penalty, lambda_grid)
        else:
            gls = solve_gls_gcv_system(System(des, tgt, wts, bn, tp.penalty), lambda_grid)
        c = gls["theta"].reshape(nc + 1, k).T
        fields = des @ c
        model = fields[:, nc] + np.sum(fields[:, :nc] * bn, axis=1)
        resid = tgt - model
        sids = g["stamp"][rows]
        sum_chi = np.bincount(sids, weights=wts * resid * resid, minlength=n_stamps)
        cnt = np.bincount(sids, minlength=n_stamps)
        stamp_chi2 = np.full(n_stamps, np.nan)
        nz = cnt > 0
        stamp_chi2[nz] = sum_chi[nz] / cnt[nz]
        denom = npix - gls["effective_dof"]
        reduced_chi2 = gls["rss"] / denom if denom > 0 else math.nan
        if have_var:
            if have_cvar:
                var_c_img = np.asarray(reference_var, np.float32)
                stamp_k2 = {}
                for s in range(n_stamps):
                    if not accepted[s] or cnt[s] == 0:
                        continue
                    a_s = tp.design(np.array([[float(g["stamp_cx"][s]), float(g["stamp_cy"][s])]])) @ c
                    kk = np.zeros((ks, ks), np.float32)
                    for n in range(nc):
                        kk = (kk + np.float32(a_s[0, n]) * phi[n]).astype(np.float32)
                    stamp_k2[s] = (kk * kk).astype(np.float32)
                rows_arr = np.asarray(rows)
                row_sid = g["stamp"][rows_arr]
                for s in stamp_k2:
                    js = rows_arr[row_sid == s]
                    if js.size == 0:
                        continue
                    pxs = g["px"][js].astype(int)
                    pys = g["py"][js].astype(int)
                    x0, x1, y0, y1 = pxs.min(), pxs.max(), pys.min(), pys.max()
                    cv = conv_var_window(stamp_k2[s], r, var_c_img, reference_mask, x0, x1, y0, y1)
                    rv = g["var_t"][js] + cv[pys - y0, pxs - x0]
                    pos = rv > 0.0
                    weights[js[pos]] = 1.0 / rv[pos]
            else:
                for j in rows:
                    if g["var_t"][j] > 0.0:
                        weights[j] = 1.0 / g["var_t"][j]
        to_reject = []
        if clip_passes > 0 and it < clip_passes:
            act = [s for s in range(n_stamps) if accepted[s] and cnt[s] > 0]
            n_active = len(act)
            if n_active > floor_stamps:
                vals = stamp_chi2[act]
                med = float(upper_median(np.asarray(vals)))
                mad = float(upper_median(np.abs(vals - med)))
                thr = med + clip_sigma * 1.4826 * mad
                cand = [s for s in act if stamp_chi2[s] > thr]
                cand.sort(key=lambda s: -stamp_chi2[s])
                for s in cand:
                    if n_active - len(to_reject) <= floor_stamps:
                        break
                    to_reject.append(s)
        if len(to_reject) == 0 and it >= min_pass:
            break
        if it >= hard_max:
            break
        for s in to_reject:
            accepted[s] = 0
        it += 1
    n_used = int(sum(1 for s in range(n_stamps) if accepted[s] and np.isfinite(stamp_chi2[s])))
    out = dict(gls)
    out.update({
        "component_sums": component_sums(b1d, orders),
        "n_pixels": int(npix),
        "n_stamps_used": n_used,
        "n_stamps_total": int(n_stamps),
        "n_stamps_rejected": int(n_stamps - n_used),
        "reduced_chi2": reduced_chi2,
        "cv_exact_design_bytes": int(cv_exact_design_bytes),
        "stamp_x": g["stamp_cx"].astype(np.int32),
        "stamp_y": g["stamp_cy"].astype(np.int32),
        "stamp_chi2": stamp_chi2,
        "stamp_accepted": accepted,
    })
    return out


# ---------------------------------------------------------------------------
# Noise decorrelation, whitened PSF, matched filter (src/noise.cpp)
# ---------------------------------------------------------------------------


def _embed_zero_phase(kernel: np.ndarray, n: int) -> np.ndarray:
    """src/noise.cpp:65-76."""
    ks = kernel.shape[0]
    r = ks // 2
    out = np.zeros((n, n))
    for ky in range(ks):
        gy = ((ky - r) % n + n) % n
        for kx in range(ks):
            gx = ((kx - r) % n + n) % n
            out[gy, gx] = kernel[ky, kx]
    return out


def kernel_power(kernel: np.ndarray, n: int) -> np.ndarray:
    """|Khat|^2 on the (n, n/2+1) half spectrum.  src/noise.cpp:65-84."""
    spec = np.fft.rfft2(_embed_zero_phase(np.asarray(kernel, np.float32).astype(np.float64), n))
    return spec.real**2 + spec.imag**2


def decorrelation_filter(kernel, var_science, var_reference, n) -> np.ndarray:
    """src/noise.cpp:98-117."""
    kernel = np.asarray(kernel, np.float32)
    power = kernel_power(kernel, n)
    sumk2 = float(np.sum(kernel.astype(np.float64) ** 2))
    cnum = math.sqrt(max(var_science + var_reference * sumk2, 0.0))
    denom = var_science + var_reference * power
    with np.errstate(divide="ignore", invalid="ignore"):
        filt = np.where(denom > 0.0, cnum / np.sqrt(np.where(denom > 0, denom, 1.0)), 0.0)
    return filt.astype(np.float32)


def apply_filter_fft(block, filt) -> np.ndarray:
    """src/noise.cpp:119-137 (float64 FFT here)."""
    spec = np.fft.rfft2(np.asarray(block, np.float64))
    return np.fft.irfft2(spec * filt.astype(np.float64), s=block.shape).astype(np.float32)


def decorrelation_kernel_image(filt, n) -> np.ndarray:
    """src/noise.cpp:139-161."""
    img = np.fft.irfft2(filt.astype(np.float64) + 0j, s=(n, n))
    return np.roll(np.roll(img, n // 2, axis=0), n // 2, axis=1).astype(np.float32)


def hann1d(n: int) -> np.ndarray:
    """src/noise.cpp:89-94."""
    i = np.arange(n)
    return 0.5 * (1.0 - np.cos(2.0 * np.pi * (i + 0.5) / n))


def block_variance(var, bx, by, block, w, h) -> float:
    """Subsampled median of finite positive variance.  src/noise.cpp:200-224."""
    step = max(1, block // 64)
    ys = [y for y in range(by, by + block, step) if 0 <= y < h]
    xs = [x for x in range(bx, bx + block, step) if 0 <= x < w]
    if not ys or not xs:
        return 0.0
    vals = np.asarray(var, np.float32)[np.ix_(ys, xs)].ravel()
    vals = vals[np.isfinite(vals) & (vals > 0)]
    med = upper_median(vals)
    return 0.0 if med is None else float(med)


def local_kernel(tp: ThinPlate, theta, phi, nc, cx, cy) -> np.ndarray:
    """K = sum_n float(a_n) phi_n at (cx, cy).  src/noise.cpp:167-189."""
    c = np.asarray(theta, float).reshape(nc + 1, tp.k).T
    a = tp.design(np.array([[cx, cy]])) @ c
    kern = np.zeros_like(phi[0])
    for n in range(nc):
        kern = (kern + np.float32(a[0, n]) * phi[n]).astype(np.float32)
    return kern


def block_origins(extent, blk, strd) -> list[int]:
    """src/noise.cpp:253-262."""
    if extent <= blk:
        return [0]
    o = list(range(0, extent - blk + 1, strd))
    if o[-1] + blk < extent:
        o.append(extent - blk)
    return o


def decorrelate(difference, knots, theta, beta, n_max, var_science, var_reference, block=256,
                radius=0, kernel_cell_blocks=0) -> dict:
    """Apodised overlap-add ZOGY whitening.  src/noise.cpp:228-483 (float64 FFT)."""
    d = np.asarray(difference, np.float32)
    h, w = d.shape
    if block < 8 or (block & (block - 1)) != 0:
        raise RuntimeError("decorrelate: block must be a power of two >= 8")
    r = resolve_radius(beta, n_max, radius)
    b1d = gauss_hermite_basis1d(beta, n_max, r)
    orders = basis_orders(n_max)
    nc = len(orders)
    phi = [kernel2d(b1d, orders, c) for c in range(nc)]
    tp = ThinPlate(knots)
    stride = block // 2
    oxs = block_origins(w, block, stride)
    oys = block_origins(h, block, stride)
    nox, noy = len(oxs), len(oys)
    kgroup = kernel_cell_blocks
    if kgroup <= 0:
        spacing = tp.min_knot_spacing()
        kgroup = 1
        if spacing > 0.0 and stride > 0:
            kgroup = max(1, int(round_half_away(spacing / 4 / stride)))
    ncellx = (nox + kgroup - 1) // kgroup
    ncelly = (noy + kgroup - 1) // kgroup
    cell_power = {}
    cell_sumk2 = {}
    for ci in range(ncellx * ncelly):
        cix, ciy = ci % ncellx, ci // ncellx
        repx = min(cix * kgroup + kgroup // 2, nox - 1)
        repy = min(ciy * kgroup + kgroup // 2, noy - 1)
        cx = min(max(oxs[repx] + block / 2.0, 0.0), w - 1.0)
        cy = min(max(oys[repy] + block / 2.0, 0.0), h - 1.0)
        kern = local_kernel(tp, theta, phi, nc, cx, cy)
        cell_power[ci] = kernel_power(kern, block)
        cell_sumk2[ci] = float(np.sum(kern.astype(np.float64) ** 2))
    hwin = hann1d(block)
    acc = np.zeros((h, w))
    var_acc = np.zeros((h, w))
    wx_total = np.zeros(w)
    wy_total = np.zeros(h)
    for bx in oxs:
        for i in range(block):
            if 0 <= bx + i < w:
                wx_total[bx + i] += hwin[i]
    for by in oys:
        for i in range(block):
            if 0 <= by + i < h:
                wy_total[by + i] += hwin[i]
    ybase = np.arange(block)
    for iy in range(noy):
        for ix in range(nox):
            bx, by = oxs[ix], oys[iy]
            cell = (iy // kgroup) * ncellx + (ix // kgroup)
            sy = by + ybase
            sy = np.where(sy < 0, -sy - 1, sy)
            sy = np.where(sy >= h, 2 * h - sy - 1, sy)
            sy = np.clip(sy, 0, h - 1)
            sx = bx + ybase
            sx = np.where(sx < 0, -sx - 1, sx)
            sx = np.where(sx >= w, 2 * w - sx - 1, sx)
            sx = np.clip(sx, 0, w - 1)
            buf = d[np.ix_(sy, sx)].astype(np.float64)
            vs = block_variance(var_science, bx, by, block, w, h)
            vr = block_variance(var_reference, bx, by, block, w, h)
            cnum = math.sqrt(max(vs + vr * cell_sumk2[cell], 0.0))
            denom = vs + vr * cell_power[cell]
            with np.errstate(divide="ignore", invalid="ignore"):
                filt = np.where(denom > 0.0, cnum / np.sqrt(np.where(denom > 0, denom, 1.0)), 0.0)
            filt = filt.astype(np.float32).astype(np.float64)
            out = np.fft.irfft2(np.fft.rfft2(buf) * filt, s=(block, block))
            num = cnum * cnum
            y0, y1 = by, min(by + block, h)
            x0, x1 = bx, min(bx + block, w)
            wgt = np.outer(hwin[: y1 - y0], hwin[: x1 - x0])
            acc[y0:y1, x0:x1] += wgt * out[: y1 - y0, : x1 - x0]
            var_acc[y0:y1, x0:x1] += wgt * num
    wsum = np.outer(wy_total, wx_total)
    pos = wsum > 0
    dw = np.zeros((h, w))
    vw = np.zeros((h, w))
    dw[pos] = acc[pos] / wsum[pos]
    vw[pos] = var_acc[pos] / wsum[pos]
    return {"difference": dw.astype(np.float32), "variance": vw.astype(np.float32), "timing": None}


def round_half_away(v: float) -> float:
    """std::lround semantics (half away from zero)."""
    return math.floor(v + 0.5) if v >= 0 else -math.floor(-v + 0.5)


def whiten_psf(psf, kernel, var_science, var_reference, n) -> np.ndarray:
    """src/noise.cpp:485-533."""
    psf = np.asarray(psf, np.float32)
    ps = psf.shape[0]
    if ps > n:
        raise RuntimeError("whiten_psf: psf_size must be <= FFT size n")
    filt = decorrelation_filter(kernel, var_science, var_reference, n).astype(np.float64)
    emb = _embed_zero_phase(psf.astype(np.float64), n)
    out_full = np.fft.irfft2(np.fft.rfft2(emb) * filt, s=(n, n))
    r = ps // 2
    out = np.zeros((ps, ps), np.float32)
    for py in range(ps):
        gy = ((py - r) % n + n) % n
        for px in range(ps):
            gx = ((px - r) % n + n) % n
            out[py, px] = np.float32(out_full[gy, gx])
    s = float(np.sum(out.astype(np.float64)))
    if s > 0.0:
        out = (out * np.float32(1.0 / s)).astype(np.float32)
    return out


def whiten_score_psf(psf, knots, theta, beta, n_max, var_science, var_reference, block, radius=0):
    """src/bindings.cpp:796-874."""
    psf = np.asarray(psf, np.float32)
    if psf.shape[0] != psf.shape[1]:
        raise RuntimeError("whiten_score_psf: psf must be square")
    if block < psf.shape[0]:
        raise RuntimeError("whiten_score_psf: block must be >= psf side")
    h, w = np.asarray(var_science).shape
    r = resolve_radius(beta, n_max, radius)
    b1d = gauss_hermite_basis1d(beta, n_max, r)
    orders = basis_orders(n_max)
    nc = len(orders)
    phi = [kernel2d(b1d, orders, c) for c in range(nc)]
    tp = ThinPlate(knots)
    cx = 0.5 * (w - 1)
    cy = 0.5 * (h - 1)
    kern = local_kernel(tp, theta, phi, nc, cx, cy)
    bx = max(0, w // 2 - block // 2)
    by = max(0, h // 2 - block // 2)
    vs = block_variance(var_science, bx, by, block, w, h)
    vr = block_variance(var_reference, bx, by, block, w, h)
    return whiten_psf(psf, kern, vs, vr, block)


def estimate_psf(image, xs, ys, radius: int) -> np.ndarray:
    """Median of background-subtracted, unit-sum stamps, clipped at 0 and
    renormalised.  python/delta/pipeline.py:285-302."""
    image = np.asarray(image, np.float32)
    h, w = image.shape
    stamps = []
    for x, y in zip(xs, ys, strict=True):
        if x - radius < 0 or x + radius >= w or y - radius < 0 or y + radius >= h:
            continue
        cut = image[y - radius : y + radius + 1, x - radius : x + radius + 1].astype(np.float64)
        cut = cut - np.median(cut)
        total = cut.sum()
        if total > 0:
            stamps.append(cut / total)
    if not stamps:
        raise ValueError("no usable sources for PSF estimation")
    psf = np.clip(np.median(np.stack(stamps), axis=0), 0.0, None)
    return np.ascontiguousarray(psf / psf.sum(), dtype=np.float32)


def default_beta(fwhm_a: float, fwhm_b: float) -> float:
    """max(0.8 sqrt(s_broad^2 - s_narrow^2), 0.5); 2.0 without a finite FWHM.
    python/delta/pipeline.py:267-282."""
    fwhms = [f for f in (fwhm_a, fwhm_b) if np.isfinite(f) and f > 0]
    if not fwhms:
        return 2.0
    broad, narrow = max(fwhms), min(fwhms)
    to_sigma = 1.0 / FWHM_PER_SIGMA
    diff = (broad * to_sigma) ** 2 - (narrow * to_sigma) ** 2
    return float(max(0.8 * (np.sqrt(diff) if diff > 0 else 0.0), 0.5))


def matched_filter(image, psf, variance) -> np.ndarray:
    """score = (psf corr D) / sqrt(var * sum psf^2); 0 where var <= 0.

    src/noise.cpp:535-632 (float64 accumulation here).
    """
    img = np.asarray(image, np.float32).astype(np.float64)
    psf = np.asarray(psf, np.float32)
    var = np.asarray(variance, np.float32)
    h, w = img.shape
    ks = psf.shape[0]
    r = ks // 2
    sumpsf2 = np.float32(0.0)
    for v in psf.ravel():
        sumpsf2 = np.float32(sumpsf2 + np.float32(v) * np.float32(v))
    pad = np.zeros((h + 2 * r, w + 2 * r))
    pad[r : r + h, r : r + w] = img
    acc = np.zeros((h, w))
    for ly in range(ks):
        for lx in range(ks):
            p = float(psf[ly, lx])
            if p == 0.0:
                continue
            acc += p * pad[ly : ly + h, lx : lx + w]
    out = np.zeros((h, w), np.float32)
    pos = var > 0
    out[pos] = (acc[pos] / np.sqrt(var[pos].astype(np.float64) * float(sumpsf2))).astype(np.float32)
    return out


# ---------------------------------------------------------------------------
# Connected-component catalog (src/catalog.cpp)
# ---------------------------------------------------------------------------


def seed_mask(score, threshold, polarity, mask, exclude_bad) -> np.ndarray:
    """src/catalog.cpp:61-80."""
    s = np.asarray(score, np.float32)
    thr = np.float32(threshold)
    with np.errstate(invalid="ignore"):
        p = np.isfinite(s) & ((s >= thr) if polarity > 0 else (s <= -thr))
    if exclude_bad and mask is not None:
        p &= np.asarray(mask) == 0
    return p


def label_components(seed: np.ndarray) -> tuple[np.ndarray, int]:
    """8-connected labels numbered by each component's first raster pixel.

    Equivalent to src/catalog.cpp:105-261 for any block count (the provisional
    ids are raster ordered within ordered blocks, and final ids are handed out
    in provisional order).
    """
    h, w = seed.shape
    n = h * w
    parent = np.arange(n)
    flat = seed.ravel()

    def find(i):
        root = i
        while parent[root] != root:
            root = parent[root]
        while parent[i] != root:
            parent[i], i = root, parent[i]
        return root

    def unite(a, b):
        ra, rb = find(a), find(b)
        if ra != rb:
            if ra < rb:
                parent[rb] = ra
            else:
                parent[ra] = rb

    idx = np.nonzero(flat)[0]
    for i in idx:
        y, x = divmod(int(i), w)
        if x > 0 and flat[i - 1]:
            unite(i, i - 1)
        if y > 0:
            a = i - w
            if x > 0 and flat[a - 1]:
                unite(i, a - 1)
            if flat[a]:
                unite(i, a)
            if x + 1 < w and flat[a + 1]:
                unite(i, a + 1)
    labels = np.zeros(n, np.int32)
    next_id = 1
    root_id = {}
    for i in idx:
        rt = find(int(i))
        if rt not in root_id:
            root_id[rt] = next_id
            next_id += 1
        labels[i] = root_id[rt]
    return labels.reshape(h, w), next_id - 1
