"""Loader for the in-tree CUDA library ``libdelta_gpu.so`` (include/delta_gpu.h).

There is no CPU fallback: if the library or a CUDA device is missing, every
device entry point raises :class:`DeviceUnavailableError`.
"""

from __future__ import annotations

import ctypes
import os
import sys
import threading
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libdelta_gpu.so"

DGPU_OK = 0
DGPU_ERR_INVALID = 1
DGPU_ERR_RUNTIME = 2
DGPU_ERR_CUDA = 3
DGPU_ERR_LIMIT = 4
DGPU_ERR_CAPACITY = 5
DGPU_ERR_NO_DEVICE = 6

MEM_HOST = 0
MEM_DEVICE = 1

PREC_FP64 = 0
PREC_FP32 = 1
PREC_MIXED = 2
PREC_TF32 = 3


class DeviceUnavailableError(RuntimeError):
    """The CUDA library or a CUDA device is not available (no CPU fallback)."""


class DeviceLoopLimitError(RuntimeError):
    """A device loop hit its iteration cap and returned an error status."""


_lib = None
_lock = threading.Lock()
_tls = threading.local()


class Model(ctypes.Structure):
    _fields_ = [
        ("knots", ctypes.c_void_p),
        ("n_knots", ctypes.c_int),
        ("theta", ctypes.c_void_p),
        ("n_theta", ctypes.c_int64),
        ("beta", ctypes.c_double),
        ("n_max", ctypes.c_int),
        ("radius", ctypes.c_int),
    ]


class CatalogParams(ctypes.Structure):
    _fields_ = [
        ("threshold_sigma", ctypes.c_double),
        ("threshold_sigma_dipole", ctypes.c_double),
        ("expected_fwhm", ctypes.c_double),
        ("fwhm_tolerance_lo", ctypes.c_double),
        ("fwhm_tolerance_hi", ctypes.c_double),
        ("aperture_radius", ctypes.c_int),
        ("exclude_bad_pixels", ctypes.c_int),
        ("return_negative", ctypes.c_int),
        ("fit_psf_shape", ctypes.c_int),
        ("shape_chi2_tolerance", ctypes.c_double),
        ("bright_star_radius", ctypes.c_double),
        ("max_shape_fit", ctypes.c_int),
    ]


class DetectParams(ctypes.Structure):
    _fields_ = [
        ("stamp_radius", ctypes.c_int),
        ("threshold_sigma", ctypes.c_double),
        ("max_stamps", ctypes.c_int),
        ("saturation", ctypes.c_double),
        ("isolation_radius", ctypes.c_int),
        ("border", ctypes.c_int),
        ("fwhm_radius", ctypes.c_int),
        ("match_radius", ctypes.c_int),
    ]


class GlsResult(ctypes.Structure):
    _fields_ = [
        ("theta", ctypes.c_void_p),
        ("lambda_grid", ctypes.c_void_p),
        ("gcv_curve", ctypes.c_void_p),
        ("component_sums", ctypes.c_void_p),
        ("stamp_x", ctypes.c_void_p),
        ("stamp_y", ctypes.c_void_p),
        ("stamp_chi2", ctypes.c_void_p),
        ("stamp_accepted", ctypes.c_void_p),
        ("n_components", ctypes.c_int),
        ("n_spatial", ctypes.c_int),
        ("lambda", ctypes.c_double),
        ("gcv", ctypes.c_double),
        ("effective_dof", ctypes.c_double),
        ("rss", ctypes.c_double),
        ("reduced_chi2", ctypes.c_double),
        ("n_pixels", ctypes.c_int64),
        ("n_stamps_used", ctypes.c_int),
        ("n_stamps_total", ctypes.c_int),
        ("n_stamps_rejected", ctypes.c_int),
        ("cv_exact_design_bytes", ctypes.c_int64),
        ("n_lambda_out", ctypes.c_int),
        ("refine_correction", ctypes.c_double),
        ("precision_used", ctypes.c_int),
        ("used_ldlt", ctypes.c_int),
    ]


CATALOG_COLUMNS = [
    ("x", np.float64), ("y", np.float64), ("peak_x", np.int32), ("peak_y", np.int32),
    ("peak_snr", np.float64), ("n_pix", np.int32), ("flux", np.float64),
    ("expected_n_pix", np.float64), ("fwhm_ratio", np.float64), ("fwhm_consistent", np.uint8),
    ("mask_flags", np.uint8), ("is_dipole", np.uint8), ("quality", np.uint8),
    ("psf_chi2", np.float64), ("psf_chi2_dof", np.int32), ("psf_amplitude", np.float64),
    ("psf_amplitude_err", np.float64), ("shape_consistent", np.uint8),
    ("bright_star_dist", np.float64), ("near_bright_star", np.uint8),
]


class CatalogColumns(ctypes.Structure):
    _fields_ = [(name, ctypes.c_void_p) for name, _ in CATALOG_COLUMNS]


class Frame(ctypes.Structure):
    _fields_ = [("width", ctypes.c_int64), ("height", ctypes.c_int64), ("science", ctypes.c_void_p),
                ("reference", ctypes.c_void_p), ("science_var", ctypes.c_void_p), ("reference_var", ctypes.c_void_p),
                ("science_mask", ctypes.c_void_p), ("reference_mask", ctypes.c_void_p)]


class BatchConfig(ctypes.Structure):
    _fields_ = [("n_max", ctypes.c_int), ("n_knots", ctypes.c_int), ("radius", ctypes.c_int),
                ("stamp_radius", ctypes.c_int), ("threshold_sigma", ctypes.c_double), ("max_stamps", ctypes.c_int),
                ("saturation", ctypes.c_double), ("fwhm_radius", ctypes.c_int), ("match_radius", ctypes.c_int),
                ("lambda_grid", ctypes.c_void_p), ("n_lambda", ctypes.c_int), ("clip_sigma", ctypes.c_double),
                ("clip_iterations", ctypes.c_int), ("min_stamps", ctypes.c_int), ("cv_folds", ctypes.c_int),
                ("precision", ctypes.c_int), ("decorrelate", ctypes.c_int), ("block", ctypes.c_int),
                ("score", ctypes.c_int), ("catalog", ctypes.c_int), ("catalog_threshold_sigma", ctypes.c_double),
                ("frames_in_flight", ctypes.c_int), ("device", ctypes.c_int), ("graphs", ctypes.c_int)]


class FrameResult(ctypes.Structure):
    _fields_ = [("difference", ctypes.c_void_p), ("variance", ctypes.c_void_p), ("mask", ctypes.c_void_p),
                ("score", ctypes.c_void_p), ("theta", ctypes.c_void_p), ("catalog", CatalogColumns),
                ("catalog_capacity", ctypes.c_int), ("n_theta", ctypes.c_int64), ("lambda_", ctypes.c_double),
                ("beta", ctypes.c_double), ("direction_is_reference", ctypes.c_int), ("n_stamps_used", ctypes.c_int),
                ("has_variance", ctypes.c_int), ("has_mask", ctypes.c_int), ("catalog_count", ctypes.c_int),
                ("catalog_fetched", ctypes.c_int), ("status", ctypes.c_int), ("error", ctypes.c_char * 256),
                ("seconds", ctypes.c_double), ("graph_replayed", ctypes.c_int)]


def lib():
    """The loaded C library (raises DeviceUnavailableError if it is missing)."""
    global _lib
    if _lib is None:
        with _lock:
            if _lib is None:
                if not LIB_PATH.exists():
                    raise DeviceUnavailableError(
                        f"{LIB_PATH} is not built; run `python -c 'import __graft_entry__ as g; g.build()'`"
                        " (or make -C delta_b200/csrc)"
                    )
                L = ctypes.CDLL(str(LIB_PATH))
                L.dgpu_last_error.restype = ctypes.c_char_p
                L.dgpu_last_error.argtypes = [ctypes.c_void_p]
                L.dgpu_create.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
                L.dgpu_destroy.argtypes = [ctypes.c_void_p]
                L.dgpu_default_radius.restype = ctypes.c_int
                _lib = L
    return _lib


def ptr(a):
    """Data pointer of a C-contiguous ndarray (None -> NULL)."""
    if a is None:
        return None
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("array must be C-contiguous")
    return ctypes.c_void_p(a.ctypes.data)


def check(rc: int, ctx=None, what: str = "") -> None:
    """Map a DGPU status code to the reference's Python exception types."""
    if rc == DGPU_OK:
        return
    msg = lib().dgpu_last_error(ctx).decode(errors="replace")
    if what and not msg.startswith(what):
        msg = f"{what}: {msg}" if msg else what
    if rc == DGPU_ERR_INVALID:
        raise ValueError(msg)
    if rc == DGPU_ERR_NO_DEVICE:
        raise DeviceUnavailableError(msg)
    if rc == DGPU_ERR_LIMIT:
        raise DeviceLoopLimitError(msg)
    raise RuntimeError(msg)


class Context:
    """One CUDA context handle (stream + workspace) of the library."""

    def __init__(self, device: int = 0):
        L = lib()
        h = ctypes.c_void_p()
        rc = L.dgpu_create(int(device), ctypes.byref(h))
        if rc != DGPU_OK:
            msg = L.dgpu_last_error(None).decode(errors="replace")
            if rc == DGPU_ERR_NO_DEVICE:
                raise DeviceUnavailableError(f"no CUDA device for delta_b200: {msg}")
            raise RuntimeError(msg)
        self.handle = h
        self.device = device

    def close(self):
        if self.handle:
            lib().dgpu_destroy(self.handle)
            self.handle = None

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_handle: int | None):
        check(lib().dgpu_set_stream(self.handle, ctypes.c_void_p(stream_handle or 0)), self.handle)

    def synchronize(self):
        check(lib().dgpu_synchronize(self.handle), self.handle)

    def set_precision_fallback(self, enabled: bool):
        """Whether a MIXED / TF32 fit that its FP64 refinement shows too
        inaccurate is redone in FP64 (the default) or returned as it is."""
        check(lib().dgpu_set_precision_fallback(self.handle, int(bool(enabled))), self.handle)


def _default_device() -> int:
    env = os.environ.get("DELTA_B200_DEVICE")
    if env is not None:
        return int(env)
    torch = sys.modules.get("torch")  # follow torch's current device when the caller uses it
    if torch is not None and torch.cuda.is_initialized():
        return int(torch.cuda.current_device())
    return 0


def context() -> Context:
    """The calling thread's context on device ``DELTA_B200_DEVICE``, else torch's
    current CUDA device when torch has initialised CUDA, else device 0 (one
    context per thread and device)."""
    dev = _default_device()
    ctxs = getattr(_tls, "ctxs", None)
    if ctxs is None:
        ctxs = _tls.ctxs = {}
    ctx = ctxs.get(dev)
    if ctx is None:
        ctx = ctxs[dev] = Context(dev)
    return ctx


def timing_enabled() -> bool:
    v = os.environ.get("DELTA_TIMING", "")
    return v not in ("", "0")


def drain_timing(ctx: Context) -> dict | None:
    if not timing_enabled():
        return None
    cap = 64
    labels = (ctypes.c_char * 64 * cap)()
    secs = (ctypes.c_double * cap)()
    n = ctypes.c_int()
    check(lib().dgpu_drain_timing(ctx.handle, labels, secs, cap, ctypes.byref(n)), ctx.handle)
    return {bytes(labels[i]).split(b"\0", 1)[0].decode(): secs[i] for i in range(min(n.value, cap))}
