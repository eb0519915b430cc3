"""delta_b200 -- B200-native (sm_100a) drop-in for tkillestein/delta's
difference-imaging hot path.

The public API mirrors ``delta`` (python/delta/__init__.py): the same
``_core`` functions, ``subtract`` / ``apply`` / ``Subtractor`` / ``DiffResult``
/ ``KernelSolution`` and the ``catalog`` / ``validation`` modules. The compute
runs in hand-written CUDA kernels behind the C ABI in include/delta_gpu.h;
there is no CPU fallback.
"""

from __future__ import annotations

from . import _core
from ._core import (
    __version__,
    basis_convolve,
    build_catalog as _build_catalog_core,
    gauss_hermite_basis1d,
    gauss_hermite_kernels,
    grid_knots,
    matched_filter,
    photometric_scale,
    photometric_scale_at,
    tps_design,
    tps_evaluate,
    tps_fit,
    tps_penalty,
)
from ._core import subtract as subtract_model
from ._lib import DeviceLoopLimitError, DeviceUnavailableError

__all__ = [
    "DeviceLoopLimitError",
    "DeviceUnavailableError",
    "__version__",
    "basis_convolve",
    "gauss_hermite_basis1d",
    "gauss_hermite_kernels",
    "grid_knots",
    "matched_filter",
    "photometric_scale",
    "photometric_scale_at",
    "subtract_model",
    "tps_design",
    "tps_evaluate",
    "tps_fit",
    "tps_penalty",
]
