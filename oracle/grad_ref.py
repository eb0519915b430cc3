"""FP64 kernel-model chi^2 and its gradients -- TEST INFRASTRUCTURE ONLY.

The reference has no gradient code, so parity for the differentiation leg is
anchored on this FP64 CPU restatement of the forward model plus its
hand-derived adjoint, itself checked against central finite differences of the
same FP64 forward (tests/test_grad_oracle.py). The forward is the
subtraction's model (src/subtract.cpp:466-639: sanitised reference, basis
convolutions in the x-then-y order of src/convolve.cpp:24-83, lattice-blended
fields of src/subtract.cpp:167-316) with the kernel shifted by (dx, dy) and
its convolved part scaled by s:

    M = s * sum_c a_c(x) (K_c^d (*) R~)(x) + b(x),  K_c^d(u, v) = g_nx(u - dx) g_ny(v - dy)
    chi2 = sum_x W(x) (S(x) - M(x))^2   over pixels with W > 0 and a finite S

Fields are blended in FP64 (bilinear weights of the lattice geometry), the
basis is sampled in FP64 at the shifted offsets, and every sum is FP64.
"""

from __future__ import annotations

import math

import numpy as np

from . import numpy_ref as nr


def shifted_basis1d(beta: float, n_max: int, radius: int, d: float):
    """g_n(u - d) and g_n'(u - d) at u = -r..r (src/basis.cpp:14-59's functions,
    g_n'(x) = norm_n / beta (2 n H_{n-1}(t) - t H_n(t)) exp(-t^2/2), t = x/beta)."""
    ks = 2 * radius + 1
    g = np.zeros((n_max + 1, ks))
    dg = np.zeros((n_max + 1, ks))
    t = (np.arange(ks) - radius - d) / beta
    e = np.exp(-0.5 * t * t)
    hm1, hc = np.zeros(ks), np.ones(ks)
    for n in range(n_max + 1):
        norm = math.exp(-0.5 * (n * math.log(2.0) + math.lgamma(n + 1.0) + 0.5 * math.log(math.pi)
                                + math.log(beta)))
        g[n] = norm * hc * e
        dg[n] = norm / beta * (2.0 * n * hm1 - t * hc) * e
        hm1, hc = hc, 2.0 * t * hc - 2.0 * n * hm1
    return g, dg


def model_image(reference, knots, theta, beta, n_max, radius=0, dx=0.0, dy=0.0, scale=1.0, reference_mask=None):
    """M = s * sum_c a_c (K_c^d (*) R~) + b in FP64, one component at a time
    (the convolved basis images are never stacked), with the float32 lattice
    fields of subtract.cpp. Used to synthesise an exposure whose shift and
    scale are known in the model's own parametrisation."""
    ref = np.asarray(reference, np.float32)
    h, w = ref.shape
    r = nr.resolve_radius(beta, n_max, radius)
    orders = nr.basis_orders(n_max)
    nc = len(orders)
    rmask = None if reference_mask is None else np.asarray(reference_mask, np.uint8)
    fill = nr.reference_fill_value(ref, rmask)
    rs = nr.sanitized_reference(ref, rmask, fill).astype(np.float64)
    fields = nr.Fields(knots, theta, nc, w, h)
    g, _ = shifted_basis1d(beta, n_max, r, dx)
    gy, _ = shifted_basis1d(beta, n_max, r, dy)
    m = np.zeros((h, w))
    for nx in range(n_max + 1):
        xpass = nr.convolve_x(rs, g[nx])
        for c, (ox, oy) in enumerate(orders):
            if ox == nx:
                m += fields.field_full(c).astype(np.float64) * nr.convolve_y(xpass, gy[oy])
    return scale * m + fields.field_full(nc).astype(np.float64)


class KernelModel:
    """The objective on one frame: fixed S, R, W, knots and basis; the
    parameters theta, (dx, dy), s vary."""

    def __init__(self, science, reference, weights, knots, beta, n_max, radius=0, reference_mask=None):
        self.s_img = np.asarray(science, np.float64)
        self.ref_f32 = np.asarray(reference, np.float32)
        self.w_img = np.asarray(weights, np.float64)
        self.rmask = None if reference_mask is None else np.asarray(reference_mask, np.uint8)
        self.h, self.w = self.s_img.shape
        self.beta, self.n_max = float(beta), int(n_max)
        self.r = nr.resolve_radius(beta, n_max, radius)
        self.orders = nr.basis_orders(n_max)
        self.nc = len(self.orders)
        self.nf = self.nc + 1
        fill = nr.reference_fill_value(self.ref_f32, self.rmask)
        self.replaced = ~np.isfinite(self.ref_f32)
        if self.rmask is not None:
            self.replaced |= self.rmask != 0
        self.rs = nr.sanitized_reference(self.ref_f32, self.rmask, fill).astype(np.float64)
        self.good = (self.w_img > 0) & np.isfinite(self.s_img)
        self.knots = np.asarray(knots, np.float64)
        self.tp = nr.ThinPlate(self.knots)
        self.k = self.tp.k
        self.design = self._design_fields()  # (k, h, w): field j of the identity theta

    def _design_fields(self):
        fl = nr.Fields(self.knots, np.zeros(self.k), 0, self.w, self.h)  # lattice geometry only
        if fl.exact:
            ys, xs = np.mgrid[0 : self.h, 0 : self.w]
            pts = np.column_stack([xs.ravel().astype(float), ys.ravel().astype(float)])
            return self.tp.design(pts).T.reshape(self.k, self.h, self.w)
        pts = np.array([(float(x), float(y)) for y in fl.gy for x in fl.gx])
        lat = self.tp.design(pts).T.reshape(self.k, fl.ncy, fl.ncx)
        jy, jx = fl.celly, fl.cellx
        fy = fl.wy.astype(np.float64)[:, None]
        fx = fl.wx.astype(np.float64)[None, :]
        out = np.empty((self.k, self.h, self.w))
        for j in range(self.k):
            c = lat[j]
            out[j] = ((1 - fy) * (1 - fx) * c[jy][:, jx] + (1 - fy) * fx * c[jy][:, jx + 1]
                      + fy * (1 - fx) * c[jy + 1][:, jx] + fy * fx * c[jy + 1][:, jx + 1])
        return out

    def fields(self, theta):
        c = np.asarray(theta, np.float64).reshape(self.nf, self.k)
        return np.einsum("fj,jyx->fyx", c, self.design)

    def components(self, dx, dy):
        g, dgx = shifted_basis1d(self.beta, self.n_max, self.r, dx)
        gy, dgy = shifted_basis1d(self.beta, self.n_max, self.r, dy)
        xs = [nr.convolve_x(self.rs, g[q]) for q in range(self.n_max + 1)]
        xds = [nr.convolve_x(self.rs, dgx[q]) for q in range(self.n_max + 1)]
        c0, cx, cy = [], [], []
        for nx, ny in self.orders:
            c0.append(nr.convolve_y(xs[nx], gy[ny]))
            cx.append(nr.convolve_y(xds[nx], gy[ny]))
            cy.append(nr.convolve_y(xs[nx], dgy[ny]))
        return np.array(c0), np.array(cx), np.array(cy), (g, gy)

    def chi2(self, theta, dx, dy, scale) -> float:
        a = self.fields(theta)
        c0, _, _, _ = self.components(dx, dy)
        m = scale * np.sum(a[: self.nc] * c0, axis=0) + a[self.nc]
        r = np.where(self.good, self.s_img - m, 0.0)
        return float(np.sum(np.where(self.good, self.w_img, 0.0) * r * r))

    def grad(self, theta, dx, dy, scale, reference=False) -> dict:
        """chi2 and its gradients by the adjoint (FP64)."""
        a = self.fields(theta)
        c0, cx, cy, (g, gy) = self.components(dx, dy)
        m0 = np.sum(a[: self.nc] * c0, axis=0)
        m = scale * m0 + a[self.nc]
        r = np.where(self.good, self.s_img - m, 0.0)
        wt = np.where(self.good, self.w_img, 0.0)
        rb = -2.0 * wt * r
        q = np.concatenate([rb[None] * scale * c0, rb[None]])  # dchi2/da_f
        out = {"chi2": float(np.sum(wt * r * r)),
               "grad_scale": float(np.sum(rb * m0)),
               "grad_shift": np.array([-float(np.sum(rb * scale * np.sum(a[: self.nc] * cx, axis=0))),
                                       -float(np.sum(rb * scale * np.sum(a[: self.nc] * cy, axis=0)))]),
               "grad_theta": np.einsum("fyx,jyx->fj", q, self.design).ravel()}
        if reference:
            p = rb * scale
            gr = np.zeros((self.h, self.w))
            for c, (nx, ny) in enumerate(self.orders):
                gr += nr.convolve_x(nr.convolve_y(p * a[c], gy[ny][::-1]), g[nx][::-1])
            out["grad_reference"] = np.where(self.replaced, 0.0, gr)
        return out


# ---------------------------------------------------------------------------
# GCV of the stamp fit through the normal-equation map (src/solve.cpp:70-193)
# ---------------------------------------------------------------------------


def _conv_fn(tx, ty, orders):
    def conv(patch):
        p = np.asarray(patch, np.float64)
        xs = {}
        out = []
        for nx, ny in orders:
            if nx not in xs:
                xs[nx] = nr.convolve_x(p, tx[nx])
            out.append(nr.convolve_y(xs[nx], ty[ny]))
        return np.array(out)
    return conv


class StampGCV:
    """GCV and weighted RSS of the stamp fit at lambda = exp(log_lambda), the
    basis shifted by (dx, dy) and scaled by s; first-pass weights
    1 / (Var_t + Var_c), no clipping (src/fit.cpp:63-287 rows, solve_at)."""

    def __init__(self, target, convolved, target_var, convolved_var, target_mask, convolved_mask, knots, stamp_x,
                 stamp_y, stamp_radius, beta, n_max, radius=0):
        self.args = (np.asarray(target, np.float32), np.asarray(convolved, np.float32), stamp_x, stamp_y,
                     int(stamp_radius))
        self.layers = (target_var, convolved_var, target_mask, convolved_mask)
        self.beta, self.n_max = float(beta), int(n_max)
        self.r = nr.resolve_radius(beta, n_max, radius)
        self.orders = nr.basis_orders(n_max)
        self.nc = len(self.orders)
        self.tp = nr.ThinPlate(knots)
        self.k = self.tp.k
        self.have_var = target_var is not None or convolved_var is not None

    def rows(self, dx, dy, scale):
        g, dg = shifted_basis1d(self.beta, self.n_max, self.r, dx)
        gy, dgy = shifted_basis1d(self.beta, self.n_max, self.r, dy)
        t, c, sx, sy, sr = self.args
        tv, cv, tm, cm = self.layers

        def gather(tx, ty):
            return nr.gather_stamps(t, c, sx, sy, sr, None, self.n_max, self.r, tv, cv, tm, cm,
                                    _conv_fn(tx, ty, self.orders))

        main = gather(scale * g, gy)
        bnx = gather(scale * dg, gy)["bn"]
        bny = gather(scale * g, dgy)["bn"]
        design = self.tp.design(np.column_stack([main["px"], main["py"]]))
        weights = 1.0 / (main["var_t"] + main["var_c"]) if self.have_var else np.ones(main["target"].size)
        return main, bnx, bny, design, weights

    def value(self, log_lambda, dx, dy, scale) -> dict:
        """solve_at's GCV / RSS, plus 'rss_direct' = sum w (t - X theta)^2 and the
        GCV from it: the same function without the cancellation of
        ywy - 2 theta.b + theta^T M theta, for finite differences."""
        main, _, _, design, weights = self.rows(dx, dy, scale)
        s = nr.System(design, main["target"], weights, main["bn"], self.tp.penalty)
        out = nr.solve_at(s, math.exp(log_lambda))
        c = out["theta"].reshape(self.nc + 1, self.k).T
        f = design @ c
        res = main["target"] - (f[:, self.nc] + np.sum(f[:, : self.nc] * main["bn"], axis=1))
        out["rss_direct"] = float(np.sum(weights * res * res))
        out["gcv_direct"] = s.n * out["rss_direct"] / (s.n - out["effective_dof"]) ** 2
        return out

    def grad(self, log_lambda, dx, dy, scale) -> dict:
        """GCV, RSS and their gradients in (log lambda, dx, dy, s) by the adjoint."""
        main, bnx, bny, d, w = self.rows(dx, dy, scale)
        t, bn = main["target"], main["bn"]
        s = nr.System(d, t, w, bn, self.tp.penalty)
        lam = math.exp(log_lambda)
        a = s.m + lam * s.p0
        f = s.pen_half
        theta = np.linalg.solve(a, s.rhs)
        hmat = np.linalg.solve(a, f)
        ft = f.T @ theta
        gmat = f.T @ hmat
        n = float(s.n)
        rss = max(s.ywy - 2.0 * theta @ s.rhs + theta @ s.m @ theta, 0.0)
        edf = s.p - lam * np.trace(gmat)
        den = n - edf
        gcv = n * rss / den**2
        alpha, beta = n / den**2, 2.0 * n * rss / den**3
        drss = 2.0 * lam * ft @ gmat @ ft
        dedf = -np.trace(gmat) + lam * np.sum(gmat * gmat)
        z = -2.0 * lam * hmat @ ft
        u = np.column_stack([bn, np.ones(len(t))])
        x = np.concatenate([d * u[:, [c]] for c in range(self.nc + 1)], axis=1)
        m_rss = np.outer(theta, theta) - 0.5 * (np.outer(z, theta) + np.outer(theta, z))
        b_rss = -2.0 * theta + z

        def ubar(mbar, bbar):
            xbar = 2.0 * w[:, None] * (x @ mbar) + (w * t)[:, None] * bbar[None, :]
            return np.stack([np.sum(d * xbar[:, c * self.k : (c + 1) * self.k], axis=1) for c in range(self.nc)], 1)

        def back(ub):
            return np.array([-np.sum(ub * bnx), -np.sum(ub * bny), np.sum(ub * bn) / scale])

        g_rss = back(ubar(m_rss, b_rss))
        g_gcv = back(ubar(alpha * m_rss + beta * lam * hmat @ hmat.T, alpha * b_rss))
        return {"gcv": gcv, "rss": rss, "effective_dof": edf, "theta": theta,
                "grad_gcv": np.concatenate([[lam * (alpha * drss + beta * dedf)], g_gcv]),
                "grad_rss": np.concatenate([[lam * drss], g_rss])}
