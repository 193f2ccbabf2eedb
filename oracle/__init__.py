"""CPU oracle for the SCycle quasi-dynamic / fully-dynamic time-step path.

THIS PACKAGE IS TEST INFRASTRUCTURE.  Only ``tests/``, ``__graft_entry__.smoke()``
and the ``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import
it, and only as the checker or as the timed CPU baseline.  The product path
(``scycle_b200``) never imports, links or executes anything in here.

What it is: a plain numpy / scipy restatement of the reference algorithm
(xinzhou1006/SCycle, C++/PETSc, CPU only).  Every function cites the reference
``file:line`` it follows.  The reference itself cannot be built in this
container (it needs PETSc, MPI, boost and MUMPS, none of which are present),
so parity is pinned by:

* the reference's own known-answer residual ``TestRoots``
  (source/rootFinder.cpp:12-24),
* its manufactured solution (source/linearElastic.cpp:1049-1128), used as a
  convergence-rate check of the assembled operator,
* the SBP identities the construction is built to satisfy,
* its example inputs (examples/*.in) and the PETSc-binary vector it ships
  (examples/ex3_z) as parser / binary-format fixtures.

Beyond these anchors the numerical parity of the full time-step path is
pinned only by this restatement ("parity unpinned" against a run of the
reference itself).  The elliptic solve of the reference is a MUMPS direct
Cholesky factorisation; the oracle uses a SciPy SuperLU direct factorisation
of the same assembled matrix (direct solve to round-off).
"""
