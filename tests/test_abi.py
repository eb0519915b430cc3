"""CPU checks of the C ABI: the library loads, exports every entry point that
include/delta_gpu.h declares, and its host-math entry points agree with the
oracle. No GPU compute is invoked here."""

from __future__ import annotations

import ctypes
import re

import numpy as np
import pytest
from conftest import ROOT

from delta_b200 import _core, _lib
from oracle import numpy_ref as nr

HEADER = ROOT / "include" / "delta_gpu.h"


def declared_symbols() -> list[str]:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(dgpu_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    names = declared_symbols()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_no_device_fails_loudly():
    n = ctypes.c_int()
    rc = _lib.lib().dgpu_device_count(ctypes.byref(n))
    if rc == 0 and n.value > 0:
        pytest.skip("a CUDA device is present")
    with pytest.raises(_lib.DeviceUnavailableError):
        _core.basis_convolve(np.zeros((8, 8), np.float32), 1.5, 1)


def test_host_basis_matches_oracle():
    for beta, n_max, r in [(1.7, 3, 6), (0.95, 6, 0), (2.0, 4, 10)]:
        got = _core.gauss_hermite_basis1d(beta, n_max, r)
        want = nr.gauss_hermite_basis1d(beta, n_max, nr.resolve_radius(beta, n_max, r))
        np.testing.assert_allclose(got, want, atol=1e-15)
        orders, kernels = _core.gauss_hermite_kernels(beta, n_max, r)
        assert [tuple(o) for o in orders] == nr.basis_orders(n_max)
        b1d = nr.gauss_hermite_basis1d(beta, n_max, nr.resolve_radius(beta, n_max, r))
        for c in range(len(orders)):
            assert np.array_equal(kernels[c], nr.kernel2d(b1d, nr.basis_orders(n_max), c))


def test_host_tps_matches_oracle():
    knots = _core.grid_knots(0, 0, 4095, 4095, 4, 4)
    np.testing.assert_array_equal(knots, nr.grid_knots(0, 0, 4095, 4095, 4, 4))
    rng = np.random.default_rng(0)
    pts = rng.uniform(0, 4096, (200, 2))
    tp = nr.ThinPlate(knots)
    np.testing.assert_allclose(_core.tps_design(knots, pts), tp.design(pts), atol=1e-12)
    np.testing.assert_allclose(_core.tps_penalty(knots), tp.penalty, atol=1e-12)
    vals = np.sin(pts[:, 0] / 900) + pts[:, 1] / 4096
    np.testing.assert_allclose(_core.tps_fit(knots, pts, vals, 1e-2), nr.tps_fit(knots, pts, vals, 1e-2), rtol=1e-8,
                               atol=1e-10)
    c = rng.standard_normal(16)
    np.testing.assert_allclose(_core.tps_evaluate(knots, pts, c), tp.design(pts) @ c, atol=1e-12)


def test_host_errors_map_to_reference_exceptions():
    with pytest.raises(ValueError):
        _core.tps_design(np.zeros((2, 2)), np.zeros((1, 2)))
    with pytest.raises(ValueError):
        _core.gauss_hermite_basis1d(-1.0, 2)
    with pytest.raises(ValueError):
        _core.grid_knots(0, 0, 1, 1, 0, 3)


def test_photometric_scale_at_matches_oracle():
    knots = _core.grid_knots(0, 0, 399, 399, 3, 3)
    rng = np.random.default_rng(7)
    theta = 0.1 * rng.standard_normal(7 * 9)
    sums = rng.standard_normal(6)
    pts = rng.uniform(0, 400, (50, 2))
    np.testing.assert_allclose(_core.photometric_scale_at(knots, theta, sums, pts),
                               nr.photometric_scale_at(knots, theta, sums, pts), atol=1e-12)


def test_ctypes_struct_layouts_match_the_header(tmp_path):
    """The ctypes mirrors of the ABI structs have the C sizes and field offsets
    (a probe compiled against include/delta_gpu.h)."""
    import shutil
    import subprocess

    if shutil.which("gcc") is None:
        pytest.skip("gcc not available")
    src = tmp_path / "probe.c"
    src.write_text(
        "#include <stdio.h>\n#include <stddef.h>\n#include \"delta_gpu.h\"\n"
        "int main(void){printf(\"%zu %zu %zu %zu %zu %zu %zu %zu\\n\", sizeof(dgpu_frame), sizeof(dgpu_batch_config),"
        " sizeof(dgpu_frame_result), offsetof(dgpu_frame_result, n_theta), offsetof(dgpu_frame_result, error),"
        " offsetof(dgpu_frame_result, seconds), sizeof(dgpu_gls_result), offsetof(dgpu_gls_result, used_ldlt));"
        "return 0;}\n")
    exe = tmp_path / "probe"
    inc = ROOT / "include"
    subprocess.run(["gcc", f"-I{inc}", str(src), "-o", str(exe)], check=True)
    want = [int(v) for v in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    fr = _lib.FrameResult
    got = [ctypes.sizeof(_lib.Frame), ctypes.sizeof(_lib.BatchConfig), ctypes.sizeof(fr), fr.n_theta.offset,
           fr.error.offset, fr.seconds.offset, ctypes.sizeof(_lib.GlsResult), _lib.GlsResult.used_ldlt.offset]
    assert got == want
