"""CPU oracle for the em3d operator-and-Krylov path.

TEST INFRASTRUCTURE ONLY.  This package is a plain NumPy restatement of the
reference algorithms (qwerty29544/em3d v0.8.0) that the B200 library is
checked against.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import it, and
only as the checker or the timed CPU baseline.  The product package
``em3d_b200`` never imports it: its kernels run on the GPU or fail loudly.

Parity status: pinned.  Every function here is checked by
``tests/test_oracle_golden.py`` against golden vectors that
``tests/golden/make_golden.py`` produced by running the reference itself
(imported read-only) on the same seeded inputs, and against the reference's own
dense-matrix known answers (``tests/test_operator_vs_dense.py:133-168`` of the
reference).

Modules
-------
``em``        EM kernel sampling, spectrum, matvec / rmatvec, dense matrices.
``acoustic``  scalar acoustic kernel, self-cell term, matvec / rmatvec.
``solvers``   BiCGStab, SIM and TwoStep restated over a matvec callable.
"""

from . import acoustic, em, solvers  # noqa: F401
