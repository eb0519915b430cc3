"""CPU oracle for the difference-imaging hot path -- TEST INFRASTRUCTURE ONLY.

This package restates the reference (tkillestein/delta 1.1.1) CPU algorithms so
the CUDA path can be checked against them. It is imported only by ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference`` legs
of ``bench.py``. The product package ``delta_b200`` never imports it and has no
CPU fallback: if its CUDA library is missing it raises.

Parts:

* ``oracle.numpy_ref``  -- FP64 NumPy restatement of basis, thin-plate spline,
  coarse field lattice, subtraction (model / variance / mask), penalised GLS +
  GCV / CV, the stamp fit (IRLS + clip), ZOGY decorrelation, whitened PSF,
  matched filter, connected-component catalog.
* ``oracle.cref``       -- ctypes loader for ``oracle/csrc/oracle.c``: a C
  restatement of the float32 hot loops with the reference's accumulation order
  and FMA contraction (the timed CPU baseline, kind "port").
* ``oracle.refbuild``   -- ctypes loader for ``oracle/_ref/libdelta_ref.so``,
  built from the reference's own Eigen-free sources (basis.cpp, convolve.cpp,
  catalog.cpp, detect.cpp, timing.cpp) by ``oracle/Makefile``; it pins basis
  taps, B_n convolution, stamp detection and the CCL catalog to the reference
  itself.

Parity pins: the C-built reference (``oracle/_ref``) pins basis, convolution,
detection and catalog; the analytic known-answer tests of the reference suite
pin subtraction, variance, mask, solver and noise (see tests/). Subtraction,
solver and noise restatements are otherwise "parity pinned by known answers":
their reference sources need Eigen, which is absent here.
"""
