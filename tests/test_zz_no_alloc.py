"""The allocation-free background estimate (dgpu_estimate_background_noalloc)
against the context entry point dgpu_estimate_background on the same frames.
Kept in its own file, collected last, so it also runs after every other test
has used the library on the same device."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from delta_b200 import _lib


def _call(L, data_ptr, mask_ptr, w, h, stream):
    med, sig = ctypes.c_double(), ctypes.c_double()
    rc = L.dgpu_estimate_background_noalloc(data_ptr, mask_ptr, ctypes.c_int64(w), ctypes.c_int64(h),
                                            ctypes.c_void_p(stream), ctypes.byref(med), ctypes.byref(sig))
    return rc, med.value, sig.value


@pytest.mark.gpu
@pytest.mark.parametrize("shape,with_mask", [((300, 500), True), ((1100, 1300), True), ((2048, 2048), False)])
def test_noalloc_background_matches_context_entry_point(shape, with_mask):
    torch = pytest.importorskip("torch")
    from delta_b200 import _core

    rng = np.random.default_rng(11)
    img = rng.normal(500.0, 20.0, shape).astype(np.float32)
    img[rng.random(shape) < 0.01] = np.nan
    mask = (rng.random(shape) < 0.02).astype(np.uint8) if with_mask else None
    want = _core.estimate_background(img, mask)
    dev = torch.device("cuda", torch.cuda.current_device())
    d = torch.from_numpy(img).to(dev)
    m = None if mask is None else torch.from_numpy(mask).to(dev)
    torch.cuda.synchronize()
    L = _lib.lib()
    h, w = shape
    args = (L, ctypes.c_void_p(d.data_ptr()), None if m is None else ctypes.c_void_p(m.data_ptr()), w, h,
            torch.cuda.current_stream().cuda_stream)
    # Warm-up: the first call on a device may load the library's device code,
    # which can take device memory once; it is not the call under test.
    rc, _, _ = _call(*args)
    assert rc == _lib.DGPU_OK, L.dgpu_last_error(None)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()  # cudaMemGetInfo: device-wide, not torch's cache
    for _ in range(2):  # two calls in a row: the fixed scratch is reset by each call
        rc, med, sig = _call(*args)
        assert rc == _lib.DGPU_OK, L.dgpu_last_error(None)
        np.testing.assert_allclose([med, sig], want, rtol=1e-12, atol=0)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, f"device free memory moved by {free0 - free1} bytes across allocation-free calls"


def test_noalloc_background_rejects_bad_arguments():
    """Argument errors are reported before any device work (runs without a GPU)."""
    L = _lib.lib()
    rc, _, _ = _call(L, None, None, 64, 64, 0)
    assert rc == _lib.DGPU_ERR_INVALID
    assert b"missing argument" in L.dgpu_last_error(None)
    rc, _, _ = _call(L, ctypes.c_void_p(16), None, 0, 64, 0)
    assert rc == _lib.DGPU_ERR_INVALID
    rc, _, _ = _call(L, ctypes.c_void_p(16), None, 1 << 16, 1 << 15, 0)
    assert rc == _lib.DGPU_ERR_INVALID
    assert b"too large" in L.dgpu_last_error(None)
