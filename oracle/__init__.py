"""CPU oracle for GPAW's finite-difference path -- TEST INFRASTRUCTURE ONLY.

Only the test suite, the smoke check and the CPU-baseline leg of the
benchmark import this package; the product (``gpaw_b200``) never does.

* ``oracle.geometry``   grid descriptor subset, stencil coefficients and
  transformer paddings restated from the reference's Python layer.
* ``oracle.kernels``    ctypes bindings to ``liboracle.so`` (the C
  restatement in gfd_oracle.c) and, when it was built, to
  ``_ref/libgpawref.so`` (GPAW's own bmgs/bc C code, compiled unmodified).
* ``oracle.poisson``    the multigrid Poisson solver of gpaw/poisson.py
  restated in Python 3 on top of either kernel library.
"""
