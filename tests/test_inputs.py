"""Input coercion of the public API (python/delta/_inputs.py behaviour, as the
reference's tests/test_inputs.py pins it) -- host only."""

from __future__ import annotations

import numpy as np
import pytest

from delta_b200 import as_layers, synth_variance


class _Uncertainty:
    def __init__(self, array, kind):
        self.array = array
        self.uncertainty_type = kind


class _CCD:
    def __init__(self, data, uncertainty=None, mask=None):
        self.data = data
        self.uncertainty = uncertainty
        self.mask = mask


def test_masked_array_without_masked_values_has_no_mask():
    data, var, mask = as_layers(np.ma.MaskedArray(np.ones((4, 4), np.float32)))
    assert data.shape == (4, 4) and var is None and mask is None


def test_masked_array_marks_masked_pixels_bad():
    bad = np.zeros((4, 4), bool)
    bad[1, 2] = True
    _, _, mask = as_layers(np.ma.MaskedArray(np.ones((4, 4), np.float32), mask=bad))
    assert mask.dtype == np.uint8 and mask[1, 2] == 1 and mask.sum() == 1
    _, _, mask = as_layers(np.ma.masked_all((4, 4), dtype=np.float32))
    assert np.all(mask == 1)


def test_ccd_like_uncertainty_kinds_and_overrides():
    d = np.arange(12, dtype=np.float64).reshape(3, 4)
    s = np.full((3, 4), 2.0)
    data, var, mask = as_layers(_CCD(d, _Uncertainty(s, "std"), d > 5))
    assert data.dtype == np.float32 and data.flags.c_contiguous
    np.testing.assert_array_equal(var, np.full((3, 4), 4.0, np.float32))
    np.testing.assert_array_equal(mask, (d > 5).astype(np.uint8))
    _, var, _ = as_layers(_CCD(d, _Uncertainty(s, "var")))
    np.testing.assert_array_equal(var, s.astype(np.float32))
    _, var, mask = as_layers(_CCD(d, _Uncertainty(s, "std"), np.ma.nomask), variance=np.ones((3, 4)),
                             mask=np.full((3, 4), 3))
    np.testing.assert_array_equal(var, np.ones((3, 4), np.float32))
    np.testing.assert_array_equal(mask, np.full((3, 4), 3, np.uint8))


def test_shape_errors():
    with pytest.raises(ValueError, match="2-D"):
        as_layers(np.zeros(5))
    with pytest.raises(ValueError, match="variance"):
        as_layers(np.zeros((2, 2)), variance=np.zeros((2, 3)))
    with pytest.raises(ValueError, match="mask"):
        as_layers(np.zeros((2, 2)), mask=np.zeros((3, 2)))


def test_synth_variance_float32_arithmetic():
    d = np.array([[-3.0, 0.0, 7.5, np.nan]], np.float32)
    v = synth_variance(d, 1.5, 2.0)
    want = np.maximum(d, np.float32(0)) / np.float32(1.5) + np.float32(4.0)
    assert v.dtype == np.float32
    np.testing.assert_array_equal(v, want)
    with pytest.raises(ValueError):
        synth_variance(d, 0.0)
