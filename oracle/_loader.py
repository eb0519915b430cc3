"""ctypes helpers shared by the oracle loaders -- TEST INFRASTRUCTURE ONLY."""

from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def ptr(a, ctype=ctypes.c_void_p):
    """Raw data pointer of a C-contiguous ndarray (None -> NULL)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "array must be C-contiguous"
    return a.ctypes.data_as(ctype)


def f32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float32)


def f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


def u8(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.uint8)


def i32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.int32)
