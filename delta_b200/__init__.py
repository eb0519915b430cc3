"""delta_b200 -- B200-native (sm_100a) drop-in for tkillestein/delta's
difference-imaging hot path.

The public API mirrors ``delta`` (python/delta/__init__.py): the same
``_core`` functions, ``subtract`` / ``apply`` / ``Subtractor`` / ``DiffResult``
/ ``KernelSolution`` and the ``catalog`` / ``validation`` modules. The compute
runs in hand-written CUDA kernels behind the C ABI in include/delta_gpu.h;
there is no CPU fallback: without the library or a device every call raises
``DeviceUnavailableError``.
"""

from __future__ import annotations

from . import _core, catalog, validation
from ._core import (
    __version__,
    basis_convolve,
    decorrelate,
    decorrelate_block,
    decorrelation_kernel,
    detect_stamps,
    estimate_background,
    fit_kernel,
    gauss_hermite_basis1d,
    gauss_hermite_kernels,
    grid_knots,
    matched_filter,
    photometric_scale,
    photometric_scale_at,
    select_stamps,
    solve_gls,
    solve_gls_cv,
    solve_gls_gcv,
    tps_design,
    tps_evaluate,
    tps_fit,
    tps_penalty,
    weighted_mean,
    whiten_score_psf,
)
from ._core import read_fits, write_fits
from ._core import subtract as subtract_model
from ._inputs import as_layers, synth_variance
from ._lib import DeviceLoopLimitError, DeviceUnavailableError
from ._log import configure_logging
from .pipeline import DiffResult, Subtractor, apply, apply_batch, subtract, subtract_batch, subtract_files
from .solution import KernelSolution


__all__ = [
    "DeviceLoopLimitError", "DeviceUnavailableError", "DiffResult", "KernelSolution", "Subtractor", "__version__",
    "apply", "apply_batch", "as_layers", "basis_convolve", "catalog", "configure_logging", "decorrelate",
    "decorrelate_block", "decorrelation_kernel", "detect_stamps", "estimate_background", "fit_kernel",
    "gauss_hermite_basis1d", "gauss_hermite_kernels", "grid_knots", "matched_filter", "photometric_scale",
    "photometric_scale_at", "read_fits", "select_stamps", "solve_gls", "solve_gls_cv", "solve_gls_gcv", "subtract",
    "subtract_batch", "subtract_files", "subtract_model", "synth_variance", "tps_design", "tps_evaluate", "tps_fit",
    "tps_penalty", "validation", "weighted_mean", "whiten_score_psf", "write_fits",
]
