"""TEST INFRASTRUCTURE ONLY: the oracle for the SCN TLM step.

Two CPU implementations of the reference's TLM time step, loaded with ctypes:

* ``Oracle`` -- ``liboracle.so``, the restatement in ``tlm_oracle.cpp``
  (float instance: bitwise the reference; double instance: the FP64 oracle).
* ``RefSolver`` -- ``_ref/libtlmref.so``, the reference's own ``TlmSolver``
  compiled headless from its sources by ``oracle/Makefile`` (present when the
  reference was available at build time; the built file travels with the tree).
* ``RefFdtd`` and ``RefEmsim`` -- the reference's ``FdtdSolver`` and its
  .emsim project writer/reader (``SaveProject`` / ``LoadProject``) from the
  same library.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this package, and only as the checker.
"""
from .wrappers import Oracle, RefEmsim, RefFdtd, RefSolver, ref_available, build_oracle  # noqa: F401
