"""CPU oracle for the bksp solver path -- TEST INFRASTRUCTURE ONLY.

Two checkers live here:

* ``oracle.ref``     -- ctypes binding of the reference C library itself
  (aldente39/bksp ``src/*.c``) compiled from its own sources by
  ``oracle/Makefile`` into ``oracle/_ref/libbksp_ref.so`` against the
  environment's OpenBLAS 0.3.15.  It also records every ``cblas_dnrm2`` the
  solvers make, which yields their recursive-residual histories.
* ``oracle.solvers`` -- a NumPy FP64 restatement of each real solver,
  line-cited against the reference, used where the compiled reference is
  unavailable and to cross-check it.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import this package, and only as the checker / the timed CPU
reference -- never on the product path.
"""
