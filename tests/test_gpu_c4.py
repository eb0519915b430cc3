"""Differentiation on a batch of 8 fields of 2048 x 2048, each with a random
sub-pixel misregistration (dx, dy ~ U(-0.5, 0.5)) and photometric scale
(~ U(0.8, 1.2)) of its science exposure.

Per field the kernel theta0 is fitted (the device pipeline, n_max 6, 4 x 4
knots, GCV, basis scale beta = 2 so the basis is well sampled at sub-pixel
shifts) on an aligned, unscaled exposure of the same stars; the objectives are
then evaluated on the misregistered, scaled exposure:
  * the weighted chi^2 of the full-frame model (dgpu_kernel_chi2): gradients in
    (dx, dy, s) and theta against central differences of the device forward on
    every field (five-point, h = 1e-2, for the shift and scale; chi^2 is
    quadratic in theta), and against the FP64 CPU adjoint on one field;
  * the stamp-fit GCV (dgpu_stamp_gcv): gradients in (log lambda, dx, dy, s)
    against five-point central differences on every field;
  * a few L-BFGS steps on chi^2 through the torch.autograd wrapper recover the
    injected shift and scale of an exposure synthesised from the model itself
    (the FP64 model image at the injected parameters plus noise), where the
    minimum lies at the injected values by construction. (On the rendered
    exposure the chi^2 minimum sits at about 0.7 of the rendered shift, by the
    FP64 oracle as well: the fitted kernel does not carry the rendering's
    sub-pixel displacement exactly.)
"""

from __future__ import annotations

import numpy as np
import pytest

import delta_b200 as delta
from delta_b200 import _core, validation
from oracle import grad_ref

pytestmark = pytest.mark.gpu

SIZE, N_FIELDS, N_STARS = 2048, 8, 5000
BETA = 2.0


def _params(i):
    rng = np.random.default_rng(4000 + i)
    dx, dy = rng.uniform(-0.5, 0.5, 2)
    return float(dx), float(dy), float(rng.uniform(0.8, 1.2))


@pytest.fixture(scope="module")
def fields():
    out = []
    for i in range(N_FIELDS):
        dx, dy, s = _params(i)
        kw = dict(mask_fraction=0.01)
        aligned = validation.synthetic_pair(SIZE, SIZE, N_STARS, 500 + i, **kw)
        moved = validation.synthetic_pair(SIZE, SIZE, N_STARS, 500 + i, science_shift=(dx, dy), science_scale=s,
                                          **kw)
        res = delta.subtract(aligned.science, aligned.reference, science_var=aligned.science_var,
                             reference_var=aligned.reference_var, science_mask=aligned.science_mask,
                             reference_mask=aligned.reference_mask, n_max=6, n_knots=4, cv_folds=0, score=False,
                             decorrelate=False, saturation=aligned.saturation, beta=BETA)
        sol = res.solution
        assert sol.direction == "reference"
        good = (moved.science_mask == 0) & (moved.reference_mask == 0)
        wt = np.where(good, 1.0 / (moved.science_var + moved.reference_var), 0.0).astype(np.float32)
        out.append(dict(p=moved, sol=sol, wt=wt, truth=(dx, dy, s)))
    return out


def _chi2(f, dx, dy, s, grad=False, theta=None):
    sol = f["sol"]
    return _core.kernel_chi2(f["p"].science, f["p"].reference, f["wt"], sol.knots,
                             sol.theta if theta is None else theta, sol.beta, sol.n_max, sol.radius, dx=dx, dy=dy,
                             scale=s, reference_mask=f["p"].reference_mask, grad=grad)


def _fd5(f, x, h):
    """Five-point central difference (truncation O(h^4))."""
    return (f(x - 2 * h) - 8 * f(x - h) + 8 * f(x + h) - f(x + 2 * h)) / (12 * h)


def test_chi2_gradients_match_central_differences_on_all_fields(fields):
    h = 1e-2
    for f in fields:
        g = _chi2(f, 0.0, 0.0, 1.0, grad=True)
        fd = [_fd5(lambda v: _chi2(f, v, 0.0, 1.0)["chi2"], 0.0, h),
              _fd5(lambda v: _chi2(f, 0.0, v, 1.0)["chi2"], 0.0, h),
              _fd5(lambda v: _chi2(f, 0.0, 0.0, v)["chi2"], 1.0, h)]
        got = [g["grad_shift"][0], g["grad_shift"][1], g["grad_scale"]]
        np.testing.assert_allclose(fd, got, rtol=2e-3, err_msg=str(f["truth"]))
        th = np.asarray(f["sol"].theta)
        for i in (0, 7, th.size - 3):
            e = np.zeros_like(th)
            e[i] = h * max(1.0, abs(th[i]))
            fdi = (_chi2(f, 0, 0, 1, theta=th + e)["chi2"] - _chi2(f, 0, 0, 1, theta=th - e)["chi2"]) / (2 * e[i])
            assert fdi == pytest.approx(g["grad_theta"][i], rel=5e-3, abs=1e-3 * np.abs(g["grad_theta"]).max())


def test_chi2_gradient_matches_fp64_cpu_adjoint(fields):
    f = fields[0]
    sol = f["sol"]
    got = _chi2(f, 0.1, -0.2, 1.03, grad=True)
    m = grad_ref.KernelModel(f["p"].science, f["p"].reference, f["wt"], sol.knots, sol.beta, sol.n_max, sol.radius,
                             reference_mask=f["p"].reference_mask)
    want = m.grad(np.asarray(sol.theta), 0.1, -0.2, 1.03)
    assert got["chi2"] == pytest.approx(want["chi2"], rel=1e-5)
    np.testing.assert_allclose(got["grad_shift"], want["grad_shift"], rtol=1e-4)
    assert got["grad_scale"] == pytest.approx(want["grad_scale"], rel=1e-4)
    rel = np.linalg.norm(got["grad_theta"] - want["grad_theta"]) / np.linalg.norm(want["grad_theta"])
    assert rel < 1e-4, rel


def test_stamp_gcv_gradients_match_central_differences_on_all_fields(fields):
    h = 1e-3
    for f in fields:
        p, sol = f["p"], f["sol"]
        sel = _core.select_stamps(p.science, p.reference, p.science_mask, p.reference_mask, stamp_radius=15,
                                  saturation=p.saturation)
        args = (p.science, p.reference, sol.knots, sel["x"], sel["y"], 15, sol.beta, sol.n_max)
        layers = dict(science_var=p.science_var, reference_var=p.reference_var, science_mask=p.science_mask,
                      reference_mask=p.reference_mask, radius=sol.radius)
        x0 = np.array([np.log(sol.lam), 0.0, 0.0, 1.0])
        g = _core.stamp_gcv(*args, *x0, **layers)["grad_gcv"]
        h = 1e-2
        for i in range(4):
            def gcv(v, i=i):
                x = x0.copy()
                x[i] = v
                return _core.stamp_gcv(*args, *x, grad=False, **layers)["gcv"]

            fd = _fd5(gcv, x0[i], h)
            assert fd == pytest.approx(g[i], rel=5e-3, abs=2e-3 * np.abs(g).max()), (i, fd, g[i])


def test_gradient_steps_recover_the_injected_shift_and_scale(fields):
    torch = pytest.importorskip("torch")
    from delta_b200.autograd import KernelProblem

    dev = torch.device("cuda")
    for f in fields[:4]:
        p, sol = f["p"], f["sol"]
        dx, dy, s = f["truth"]
        model = grad_ref.model_image(p.reference, sol.knots, np.asarray(sol.theta), sol.beta, sol.n_max, sol.radius,
                                     dx=dx, dy=dy, scale=s, reference_mask=p.reference_mask)
        rng = np.random.default_rng(7)
        sci = (model + rng.standard_normal(model.shape) * np.sqrt(p.science_var + p.reference_var)).astype(np.float32)
        prob = KernelProblem(torch.from_numpy(sci).to(dev), torch.from_numpy(f["wt"]).to(dev), sol.knots,
                             sol.beta, sol.n_max, sol.radius, reference_mask=torch.from_numpy(p.reference_mask).to(dev))
        theta = torch.tensor(np.asarray(sol.theta), dtype=torch.float64)
        ref = torch.from_numpy(p.reference).to(dev)
        shift = torch.zeros(2, dtype=torch.float64, requires_grad=True)
        scale = torch.ones((), dtype=torch.float64, requires_grad=True)
        chi0 = float(prob.chi2(theta, shift, scale, ref))
        opt = torch.optim.LBFGS([shift, scale], lr=1.0, max_iter=40, line_search_fn="strong_wolfe")

        def closure():
            opt.zero_grad()
            loss = prob.chi2(theta, shift, scale, ref) / chi0
            loss.backward()
            return loss

        opt.step(closure)
        got = shift.detach().numpy()
        assert abs(got[0] - dx) < 0.02 and abs(got[1] - dy) < 0.02, (got, (dx, dy))
        assert abs(float(scale) - s) < 0.005 * s, (float(scale), s)
