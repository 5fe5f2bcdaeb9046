"""CPU oracle for the collision contraction (TEST INFRASTRUCTURE).

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package.  It checks the CUDA path; it is never the
thing measured or shipped.

Contents
--------
* ``contraction.c`` / ``liboracle.so`` -- C restatement of the reference's
  angular-first, radial-first, naive and dense kernels (src/mex/*.cpp) plus the
  bilinear Jacobian apply.
* ``_ref/libref_exact.so`` / ``_ref/libref_fast.so`` -- the reference's own MEX
  sources compiled unmodified (oracle/Makefile) against the stub MEX host in
  ``mexhost/``.  ``exact`` uses MATLAB's default optimisation level and no FMA
  contraction, so the restatement can be pinned to it bit for bit; ``fast`` is
  the timed CPU baseline.
* ``reference.py`` -- ctypes bindings for both.
* ``rtensor.py`` -- restatement of the MATLAB driver that prepares the 26 inputs
  of the reference's ``compute_rtensor_sumfac_mex`` and applies the
  conservation rule (src/GeneralCollisionTensor.m:43-192).
"""
