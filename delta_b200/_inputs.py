"""Coercion of the images a caller hands to ``subtract`` / ``Subtractor``.

The public API accepts the same inputs as the reference's (python/delta/_inputs.py,
pinned by tests/test_inputs.py there):

* a plain array -> data only;
* a ``numpy.ma.MaskedArray`` -> data, and its mask when it has one (``nomask``
  gives no mask layer; True entries become bad pixels, value 1);
* a CCDData-like object (``.data``, optional ``.uncertainty`` with ``.array`` and
  ``.uncertainty_type``, optional ``.mask``) -> data, a variance layer (a
  standard-deviation uncertainty is squared, any other kind is taken as a
  variance) and the mask.

Explicit ``variance`` / ``mask`` arguments replace the object's own layers.
Every layer leaves as a C-contiguous array: data and variance float32, mask
uint8, all of the data's 2-D shape.
"""

from __future__ import annotations

import numpy as np
from numpy.typing import NDArray

Layers = tuple[NDArray[np.float32], NDArray[np.float32] | None, NDArray[np.uint8] | None]


def _variance_of(uncertainty):
    """Variance layer carried by a CCDData-style uncertainty, or None."""
    values = None if uncertainty is None else getattr(uncertainty, "array", None)
    if values is None:
        return None
    values = np.asarray(values, dtype=np.float64)
    kind = getattr(uncertainty, "uncertainty_type", "std")
    return np.square(values) if kind == "std" else values


def _own_layers(obj):
    """(data, variance, mask) that the object itself carries."""
    if isinstance(obj, np.ma.MaskedArray):
        own_mask = np.ma.getmask(obj)
        return np.ma.getdata(obj), None, (None if own_mask is np.ma.nomask else own_mask)
    if isinstance(obj, np.ndarray) or not hasattr(obj, "data"):
        return obj, None, None
    own_mask = getattr(obj, "mask", None)
    if own_mask is np.ma.nomask:
        own_mask = None
    return obj.data, _variance_of(getattr(obj, "uncertainty", None)), own_mask


def _matching(layer, dtype, shape, name):
    out = np.ascontiguousarray(layer, dtype=dtype)
    if out.shape != shape:
        raise ValueError(f"{name} shape {out.shape} does not match data shape {shape}")
    return out


def as_layers(obj, variance=None, mask=None) -> Layers:
    """Split ``obj`` into contiguous (data, variance, mask) layers; explicit
    ``variance`` / ``mask`` arguments take precedence over the object's."""
    data, own_var, own_mask = _own_layers(obj)
    data = np.ascontiguousarray(data, dtype=np.float32)
    if data.ndim != 2:
        raise ValueError(f"expected a 2-D image, got shape {data.shape}")
    var_layer = own_var if variance is None else variance
    mask_layer = own_mask if mask is None else mask
    if var_layer is not None:
        var_layer = _matching(var_layer, np.float32, data.shape, "variance")
    if mask_layer is not None:
        # Booleans (True == bad) and integer flags both land as uint8 bit flags.
        mask_layer = _matching(np.asarray(mask_layer).astype(np.uint8, copy=False), np.uint8, data.shape, "mask")
    return data, var_layer, mask_layer


def synth_variance(data, gain: float, read_noise: float = 0.0) -> NDArray[np.float32]:
    """Poisson + read-noise variance in ADU^2 of an image in ADU:
    max(data, 0) / gain + read_noise^2."""
    if not gain > 0.0:
        raise ValueError("gain must be > 0")
    # Computed in the image's own float width (float32 stays float32), so the
    # layer is bit-identical to the reference's for the same input.
    signal = np.maximum(np.asarray(data), 0.0)
    return np.ascontiguousarray(signal / gain + float(read_noise) ** 2, dtype=np.float32)
