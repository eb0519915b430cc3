"""Gradients of the kernel model through hand-written device adjoints.

The reference has no gradient code; these are extensions of the same model.
Two objectives are differentiable, each a ``torch.autograd.Function`` whose
forward and backward are libdelta_gpu kernels (PyTorch supplies only the
tensors, the stream and the autograd bookkeeping):

``KernelChi2`` -- the weighted chi^2 of the full-frame kernel model
    chi2 = sum_x W(x) (S(x) - M(x))^2,
    M = scale * sum_c a_c(x) [K_c shifted by (dx, dy) (*) R~](x) + b(x),
    with respect to theta (the thin-plate coefficients of every kernel
    component and the background), the shift (dx, dy), the scale and the
    reference image R. The forward computes chi^2 only; the backward recomputes
    the convolved tiles with the derivative taps (dgpu_kernel_chi2) instead of
    keeping the N_basis convolved images.

``StampGCV`` -- the GCV score of the penalised stamp fit as a function of
    log lambda, the shift and the scale (dgpu_stamp_gcv), through the adjoint
    of the normal-equation map; it also returns the stamp chi^2 (the fit's
    weighted residual sum of squares) with the same gradients.

Inputs follow the library's layout: theta float64 of length (nc+1)*k in the
order [c_0 | ... | c_{nc-1} | b]; images float32 (H, W) CUDA tensors.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _core, _lib
from ._device import _ctx_on_torch_stream, _p

try:
    import torch
except ImportError:  # pragma: no cover - the image ships torch
    torch = None

MEM_DEVICE = _lib.MEM_DEVICE


def _f32(t):
    return t.detach().to(dtype=torch.float32).contiguous()


@dataclass
class KernelProblem:
    """The fixed data of a kernel-model objective: science S, weights W
    (0 excludes a pixel), the reference mask, knots and the Gauss-Hermite
    basis. Images are CUDA tensors (H, W)."""

    science: object
    weights: object
    knots: np.ndarray
    beta: float
    n_max: int
    radius: int = 0
    reference_mask: object = None

    def __post_init__(self):
        if torch is None or not torch.cuda.is_available():
            raise _lib.DeviceUnavailableError("KernelProblem needs a CUDA device (there is no CPU path)")
        self.science = _f32(self.science)
        self.weights = _f32(self.weights)
        if self.reference_mask is not None:
            self.reference_mask = self.reference_mask.detach().to(dtype=torch.uint8).contiguous()
        self.knots = np.ascontiguousarray(self.knots, np.float64)

    def evaluate(self, theta, shift, scale, reference, grad: bool, grad_reference: bool = False) -> dict:
        """One call of dgpu_kernel_chi2 on torch's current stream."""
        ref = _f32(reference)
        h, w = self.science.shape
        if tuple(ref.shape) != (h, w):
            raise ValueError("reference shape does not match the science frame")
        th = np.ascontiguousarray(theta.detach().cpu().numpy(), np.float64)
        sh = np.asarray(shift.detach().cpu().numpy(), np.float64).reshape(2)
        sc = float(scale.detach().cpu())
        model, keep = _core._model(self.knots, th, self.beta, self.n_max, self.radius)
        ctx = _ctx_on_torch_stream()
        chi2, g_scale = ctypes.c_double(), ctypes.c_double()
        g_theta = np.empty(th.size) if grad else None
        g_shift = np.empty(2) if grad else None
        g_ref = torch.empty_like(ref) if grad_reference else None
        _lib.check(_lib.lib().dgpu_kernel_chi2(
            ctx.handle, MEM_DEVICE, ctypes.c_int64(w), ctypes.c_int64(h), _p(self.science), _p(ref),
            _p(self.reference_mask), _p(self.weights), ctypes.byref(model), ctypes.c_double(sh[0]),
            ctypes.c_double(sh[1]), ctypes.c_double(sc), ctypes.byref(chi2), _lib.ptr(g_theta), _lib.ptr(g_shift),
            ctypes.byref(g_scale) if grad else None, _p(g_ref)), ctx.handle)
        return {"chi2": chi2.value, "grad_theta": g_theta, "grad_shift": g_shift,
                "grad_scale": g_scale.value if grad else None, "grad_reference": g_ref}

    def chi2(self, theta, shift, scale, reference):
        """Differentiable chi^2 (a float64 scalar tensor)."""
        return KernelChi2.apply(theta, shift, scale, reference, self)


class KernelChi2(torch.autograd.Function if torch is not None else object):
    """chi^2(theta, shift, scale, reference) of a KernelProblem."""

    @staticmethod
    def forward(ctx, theta, shift, scale, reference, problem):
        ctx.problem = problem
        ctx.save_for_backward(theta, shift, scale, reference)
        out = problem.evaluate(theta, shift, scale, reference, grad=False)
        return torch.tensor(out["chi2"], dtype=torch.float64, device=theta.device)

    @staticmethod
    def backward(ctx, g):
        theta, shift, scale, reference = ctx.saved_tensors
        need_ref = ctx.needs_input_grad[3]
        res = ctx.problem.evaluate(theta, shift, scale, reference, grad=True, grad_reference=need_ref)
        gg = float(g)

        def as_t(v, like):
            return torch.as_tensor(np.asarray(v) * gg, dtype=like.dtype, device=like.device).reshape(like.shape)

        g_ref = (res["grad_reference"] * gg).to(reference.dtype) if need_ref else None
        return (as_t(res["grad_theta"], theta), as_t(res["grad_shift"], shift), as_t(res["grad_scale"], scale),
                g_ref, None)


@dataclass
class StampProblem:
    """The fixed data of the stamp-fit GCV objective: the target (the frame the
    fit predicts) and the convolved frame with their variances and masks as
    CUDA tensors, the knots, the stamp centres and the basis."""

    target: object
    convolved: object
    knots: np.ndarray
    stamp_x: np.ndarray
    stamp_y: np.ndarray
    stamp_radius: int
    beta: float
    n_max: int
    radius: int = 0
    target_var: object = None
    convolved_var: object = None
    target_mask: object = None
    convolved_mask: object = None

    def __post_init__(self):
        if torch is None or not torch.cuda.is_available():
            raise _lib.DeviceUnavailableError("StampProblem needs a CUDA device (there is no CPU path)")
        self.target = _f32(self.target)
        self.convolved = _f32(self.convolved)
        self.target_var = None if self.target_var is None else _f32(self.target_var)
        self.convolved_var = None if self.convolved_var is None else _f32(self.convolved_var)
        for name in ("target_mask", "convolved_mask"):
            v = getattr(self, name)
            if v is not None:
                setattr(self, name, v.detach().to(dtype=torch.uint8).contiguous())
        self.knots = np.ascontiguousarray(self.knots, np.float64)
        self.stamp_x = np.ascontiguousarray(self.stamp_x, np.int32)
        self.stamp_y = np.ascontiguousarray(self.stamp_y, np.int32)

    def evaluate(self, log_lambda, shift, scale, grad: bool) -> dict:
        """One call of dgpu_stamp_gcv on torch's current stream."""
        h, w = self.target.shape
        nc = (self.n_max + 1) * (self.n_max + 2) // 2
        sh = np.asarray(shift.detach().cpu().numpy(), np.float64).reshape(2)
        vals = np.zeros(4)
        theta = np.zeros((nc + 1) * self.knots.shape[0])
        g_gcv = np.zeros(4) if grad else None
        g_rss = np.zeros(4) if grad else None
        ctx = _ctx_on_torch_stream()
        _lib.check(_lib.lib().dgpu_stamp_gcv(
            ctx.handle, MEM_DEVICE, ctypes.c_int64(w), ctypes.c_int64(h), _p(self.target), _p(self.convolved),
            _p(self.target_var), _p(self.convolved_var), _p(self.target_mask), _p(self.convolved_mask),
            _lib.ptr(self.knots), self.knots.shape[0], _lib.ptr(self.stamp_x), _lib.ptr(self.stamp_y),
            int(self.stamp_x.size), int(self.stamp_radius), ctypes.c_double(self.beta), int(self.n_max),
            int(self.radius), ctypes.c_double(float(log_lambda.detach().cpu())), ctypes.c_double(sh[0]),
            ctypes.c_double(sh[1]), ctypes.c_double(float(scale.detach().cpu())), _lib.ptr(vals), _lib.ptr(theta),
            _lib.ptr(g_gcv), _lib.ptr(g_rss)), ctx.handle)
        return {"gcv": vals[0], "rss": vals[1], "effective_dof": vals[2], "n_pixels": int(vals[3]), "theta": theta,
                "grad_gcv": g_gcv, "grad_rss": g_rss}

    def gcv(self, log_lambda, shift, scale):
        """Differentiable (GCV, RSS) pair (float64 scalar tensors)."""
        return StampGCV.apply(log_lambda, shift, scale, self)


class StampGCV(torch.autograd.Function if torch is not None else object):
    """(GCV, RSS)(log_lambda, shift, scale) of a StampProblem."""

    @staticmethod
    def forward(ctx, log_lambda, shift, scale, problem):
        res = problem.evaluate(log_lambda, shift, scale, grad=True)
        dev = shift.device
        ctx.save_for_backward(torch.as_tensor(res["grad_gcv"], device=dev),
                              torch.as_tensor(res["grad_rss"], device=dev))
        ctx.like = (log_lambda, shift, scale)
        return (torch.tensor(res["gcv"], dtype=torch.float64, device=dev),
                torch.tensor(res["rss"], dtype=torch.float64, device=dev))

    @staticmethod
    def backward(ctx, g_gcv, g_rss):
        gg, gr = ctx.saved_tensors
        tot = gg * g_gcv.to(gg.dtype) + gr * g_rss.to(gr.dtype)
        log_lambda, shift, scale = ctx.like
        return (tot[0].to(log_lambda.dtype).reshape(log_lambda.shape), tot[1:3].to(shift.dtype).reshape(shift.shape),
                tot[3].to(scale.dtype).reshape(scale.shape), None)
