"""Device gradients of the kernel model: the weighted chi^2 (dgpu_kernel_chi2)
and the stamp-fit GCV (dgpu_stamp_gcv), against the FP64 CPU adjoints of
oracle/grad_ref.py (themselves pinned by central differences,
tests/test_grad_oracle.py) and against central differences (h = 1e-3) of the
device's own forward, plus the torch.autograd wrappers.

Tolerances: the device forward is float32 (the subtraction's arithmetic) with
FP64 reductions; against the FP64 oracle the gradients agree to 1e-4 of their
size, and central differences of the float32 forward to 2e-3."""

from __future__ import annotations

import numpy as np
import pytest

from delta_b200 import _core, validation
from oracle import grad_ref, refbuild
from oracle import numpy_ref as nr

pytestmark = pytest.mark.gpu


def _frame(w, h, n_stars, seed, n_max, knots_side, beta=1.4):
    p = validation.synthetic_pair(w, h, n_stars, seed, mask_fraction=0.02)
    wt = np.where(p.science_mask == 0, 1.0 / (p.science_var + p.reference_var), 0.0).astype(np.float32)
    knots = nr.grid_knots(0, 0, w - 1, h - 1, knots_side, knots_side)
    nc = (n_max + 1) * (n_max + 2) // 2
    k = knots.shape[0]
    rng = np.random.default_rng(seed + 7)
    theta = 0.02 * rng.standard_normal((nc + 1) * k)
    theta[0:k] += 1.0
    theta[nc * k : (nc + 1) * k] += 2.0  # a background offset
    return p, wt, knots, theta, beta


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("w,h,n_max,knots_side", [(96, 80, 2, 3), (320, 288, 4, 4)])
def test_kernel_chi2_matches_fp64_oracle(w, h, n_max, knots_side):
    p, wt, knots, theta, beta = _frame(w, h, 60, 3, n_max, knots_side)
    dx, dy, s = 0.23, -0.31, 1.08
    got = _core.kernel_chi2(p.science, p.reference, wt, knots, theta, beta, n_max, dx=dx, dy=dy, scale=s,
                            reference_mask=p.reference_mask, grad=True, grad_reference=True)
    m = grad_ref.KernelModel(p.science, p.reference, wt, knots, beta, n_max, reference_mask=p.reference_mask)
    want = m.grad(theta, dx, dy, s, reference=True)
    assert got["chi2"] == pytest.approx(want["chi2"], rel=1e-5)
    assert _rel(got["grad_shift"], want["grad_shift"]) < 1e-4
    assert got["grad_scale"] == pytest.approx(want["grad_scale"], rel=1e-4)
    assert _rel(got["grad_theta"], want["grad_theta"]) < 1e-4
    assert _rel(got["grad_reference"], want["grad_reference"]) < 1e-4
    assert np.all(got["grad_reference"][m.replaced] == 0.0)


def _fd5(f, x, h):
    """Five-point central difference (truncation O(h^4))."""
    return (f(x - 2 * h) - 8 * f(x - h) + 8 * f(x + h) - f(x + 2 * h)) / (12 * h)


def test_kernel_chi2_central_differences_on_device():
    """Central differences of the float32 device forward. The science is the
    FP64 model at (dx, dy, s) = (0, 0, 1) plus noise, and the derivatives are
    taken at a displaced point, where chi^2 is dominated by the model mismatch
    and moves by far more than its float32 rounding over the step."""
    p, wt, knots, theta, beta = _frame(256, 224, 50, 5, 3, 3)
    rng = np.random.default_rng(12)
    model = grad_ref.model_image(p.reference, knots, theta, beta, 3, reference_mask=p.reference_mask)
    sci = (model + rng.standard_normal(model.shape) * np.sqrt(p.science_var + p.reference_var)).astype(np.float32)
    x0 = dict(dx=0.11, dy=0.07, scale=0.93)

    def f(th=theta, **kw):
        return _core.kernel_chi2(sci, p.reference, wt, knots, th, beta, 3, reference_mask=p.reference_mask,
                                 grad=False, **{**x0, **kw})["chi2"]

    g = _core.kernel_chi2(sci, p.reference, wt, knots, theta, beta, 3, reference_mask=p.reference_mask, grad=True,
                          **x0)
    h = 1e-2
    for name, gi in (("dx", g["grad_shift"][0]), ("dy", g["grad_shift"][1]), ("scale", g["grad_scale"])):
        fd = _fd5(lambda v: f(**{name: v}), x0[name], h)
        assert fd == pytest.approx(gi, rel=2e-3), name
    for i in (0, 5, theta.size - 1):  # chi^2 is quadratic in theta: a central difference is exact
        e = np.zeros_like(theta)
        e[i] = h
        fd = (f(th=theta + e) - f(th=theta - e)) / (2 * h)
        assert fd == pytest.approx(g["grad_theta"][i], rel=2e-3, abs=2e-3 * np.abs(g["grad_theta"]).max()), i


def test_kernel_chi2_autograd_function():
    torch = pytest.importorskip("torch")
    from delta_b200.autograd import KernelProblem

    p, wt, knots, theta, beta = _frame(128, 112, 40, 6, 2, 3)
    dev = torch.device("cuda")
    prob = KernelProblem(torch.from_numpy(p.science).to(dev), torch.from_numpy(wt).to(dev), knots, beta, 2,
                         reference_mask=torch.from_numpy(p.reference_mask).to(dev))
    th = torch.tensor(theta, dtype=torch.float64, requires_grad=True)
    sh = torch.tensor([0.2, -0.1], dtype=torch.float64, requires_grad=True)
    sc = torch.tensor(1.1, dtype=torch.float64, requires_grad=True)
    ref = torch.from_numpy(p.reference).to(dev).requires_grad_(True)
    loss = 0.5 * prob.chi2(th, sh, sc, ref)
    loss.backward()
    want = _core.kernel_chi2(p.science, p.reference, wt, knots, theta, beta, 2, dx=0.2, dy=-0.1, scale=1.1,
                             reference_mask=p.reference_mask, grad=True, grad_reference=True)
    assert float(loss) == pytest.approx(0.5 * want["chi2"], rel=1e-12)
    np.testing.assert_allclose(th.grad.numpy(), 0.5 * want["grad_theta"], rtol=1e-12)
    np.testing.assert_allclose(sh.grad.numpy(), 0.5 * want["grad_shift"], rtol=1e-12)
    assert float(sc.grad) == pytest.approx(0.5 * want["grad_scale"], rel=1e-12)
    np.testing.assert_allclose(ref.grad.cpu().numpy(), 0.5 * want["grad_reference"], rtol=1e-6)


def _stamp_case(seed=4, w=180, h=160, n_max=2, knots_side=3, sr=8):
    p = validation.synthetic_pair(w, h, 50, seed, mask_fraction=0.01)
    if refbuild.available():
        sel = refbuild.select_stamps(p.science, p.reference, p.science_mask, p.reference_mask, stamp_radius=sr,
                                     saturation=p.saturation, max_stamps=12)
        sx, sy = sel["x"], sel["y"]
    else:
        sx, sy = np.array([40, 90, 130, 60, 120]), np.array([40, 60, 110, 120, 30])
    knots = nr.grid_knots(0, 0, w - 1, h - 1, knots_side, knots_side)
    return p, knots, np.asarray(sx, np.int32), np.asarray(sy, np.int32), sr, n_max


def test_stamp_gcv_matches_fp64_oracle_and_central_differences():
    p, knots, sx, sy, sr, n_max = _stamp_case()
    x0 = np.array([np.log(0.3), 0.17, -0.22, 1.05])
    layers = dict(science_var=p.science_var, reference_var=p.reference_var, science_mask=p.science_mask,
                  reference_mask=p.reference_mask)

    def dev(x, grad=True):
        return _core.stamp_gcv(p.science, p.reference, knots, sx, sy, sr, 1.5, n_max, x[0], x[1], x[2], x[3],
                               grad=grad, **layers)

    got = dev(x0)
    m = grad_ref.StampGCV(p.science, p.reference, p.science_var, p.reference_var, p.science_mask, p.reference_mask,
                          knots, sx, sy, sr, 1.5, n_max)
    want = m.grad(*x0)
    assert got["gcv"] == pytest.approx(want["gcv"], rel=1e-6)
    assert got["rss"] == pytest.approx(want["rss"], rel=1e-6)
    assert got["effective_dof"] == pytest.approx(want["effective_dof"], rel=1e-9)
    np.testing.assert_allclose(got["theta"], want["theta"], rtol=1e-5, atol=1e-7 * np.abs(want["theta"]).max())
    for key in ("grad_gcv", "grad_rss"):
        np.testing.assert_allclose(got[key], want[key], rtol=1e-4, atol=1e-4 * np.abs(want[key]).max(), err_msg=key)
    h = 1e-3
    for i in range(4):
        e = np.zeros(4)
        e[i] = h
        fd = (dev(x0 + e, False)["gcv"] - dev(x0 - e, False)["gcv"]) / (2 * h)
        assert fd == pytest.approx(got["grad_gcv"][i], rel=2e-3, abs=1e-3 * np.abs(got["grad_gcv"]).max()), i


def test_stamp_gcv_autograd_function():
    torch = pytest.importorskip("torch")
    from delta_b200.autograd import StampProblem

    p, knots, sx, sy, sr, n_max = _stamp_case(seed=9)
    d = torch.device("cuda")
    t = lambda a: None if a is None else torch.from_numpy(a).to(d)  # noqa: E731
    prob = StampProblem(t(p.science), t(p.reference), knots, sx, sy, sr, 1.5, n_max, target_var=t(p.science_var),
                        convolved_var=t(p.reference_var), target_mask=t(p.science_mask),
                        convolved_mask=t(p.reference_mask))
    ll = torch.tensor(np.log(2.0), dtype=torch.float64, requires_grad=True)
    sh = torch.tensor([0.05, 0.1], dtype=torch.float64, requires_grad=True)
    sc = torch.tensor(0.97, dtype=torch.float64, requires_grad=True)
    gcv, rss = prob.gcv(ll, sh, sc)
    (gcv + 1e-3 * rss).backward()
    want = _core.stamp_gcv(p.science, p.reference, knots, sx, sy, sr, 1.5, n_max, np.log(2.0), 0.05, 0.1, 0.97,
                           science_var=p.science_var, reference_var=p.reference_var, science_mask=p.science_mask,
                           reference_mask=p.reference_mask)
    tot = want["grad_gcv"] + 1e-3 * want["grad_rss"]
    assert float(ll.grad) == pytest.approx(tot[0], rel=1e-12)
    np.testing.assert_allclose(sh.grad.cpu().numpy(), tot[1:3], rtol=1e-12)
    assert float(sc.grad) == pytest.approx(tot[3], rel=1e-12)
