"""Precision study of the normal equations at the 725-unknown shape (28
components, 5 x 5 knots) over about 4e6 stamp rows of the 4096 x 4096 field:
the FP32 SIMT, TF32 and BF16x3 tensor-core builds against the FP64 oracle's fit
of the same rows (bench.precision_study). Bars: the device FP64 path within
1e-6 of the oracle's theta; BF16x3 (after its FP64 refinement step) within
1e-4 sigma RMS in the difference image; TF32 (refined, or falling back to FP64
when its refinement step shows it too coarse) within 1e-3 sigma RMS. FP32 is
reported."""

from __future__ import annotations

import json

import pytest

import bench

pytestmark = pytest.mark.gpu


def test_precision_study_at_725_unknowns_and_4e6_rows():
    from oracle import chain

    if not chain.available():
        pytest.skip("oracle/_ref is not built")
    s = bench.precision_study()
    print(json.dumps(s, indent=1))
    assert s["P"] == 725 and s["n_rows"] > 3_000_000
    m = s["modes"]
    assert m["fp64"]["theta_rel"] < 1e-6 and m["fp64"]["lambda_equal"]
    assert m["mixed"]["diff_rms_sigma"] < 1e-4, m["mixed"]
    assert m["mixed"]["score_max_abs"] < 1e-2, m["mixed"]
    assert m["tf32"]["precision_used"] in ("tf32", "fp64")
    assert m["tf32"]["diff_rms_sigma"] < 1e-3, m["tf32"]
    assert m["fp32"]["diff_rms_sigma"] < 1.0, m["fp32"]
