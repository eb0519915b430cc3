"""Input coercion (mirror of python/delta/_inputs.py): ndarray / CCDData-like
objects -> contiguous (data float32, variance float32 | None, mask uint8 | None)."""

from __future__ import annotations

import numpy as np
from numpy.typing import NDArray

Layers = tuple[NDArray[np.float32], NDArray[np.float32] | None, NDArray[np.uint8] | None]


def _split(obj):
    data = getattr(obj, "data", None)
    if data is None:
        return np.asarray(obj), None, None
    variance = None
    unc = getattr(obj, "uncertainty", None)
    if unc is not None and getattr(unc, "array", None) is not None:
        arr = np.asarray(unc.array, dtype=np.float64)
        utype = getattr(unc, "uncertainty_type", "std")
        variance = arr**2 if utype == "std" else arr
    mask = getattr(obj, "mask", None)
    if mask is np.ma.nomask:
        mask = None
    return np.asarray(data), variance, mask


def as_layers(obj, variance=None, mask=None) -> Layers:
    """Coerce to (data, variance, mask); explicit arguments override the object's
    layers; a boolean mask means True == bad (kMaskBad)."""
    data, v, m = _split(obj)
    if variance is not None:
        v = variance
    if mask is not None:
        m = mask
    data = np.ascontiguousarray(data, dtype=np.float32)
    if data.ndim != 2:
        raise ValueError(f"expected a 2-D image, got shape {data.shape}")
    if v is not None:
        v = np.ascontiguousarray(v, dtype=np.float32)
        if v.shape != data.shape:
            raise ValueError("variance shape does not match data")
    if m is not None:
        m = np.asarray(m)
        if m.dtype == bool:
            m = m.astype(np.uint8)
        m = np.ascontiguousarray(m, dtype=np.uint8)
        if m.shape != data.shape:
            raise ValueError("mask shape does not match data")
    return data, v, m


def synth_variance(data, gain: float, read_noise: float = 0.0) -> NDArray[np.float32]:
    """Var = max(data, 0) / gain + read_noise**2 (ADU)."""
    if gain <= 0.0:
        raise ValueError("gain must be > 0")
    var = np.clip(data, 0.0, None) / gain + float(read_noise) ** 2
    return np.ascontiguousarray(var, dtype=np.float32)
