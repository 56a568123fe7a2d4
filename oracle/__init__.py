"""CPU oracle for the normal-equations inner solve — TEST INFRASTRUCTURE ONLY.

This package restates, in NumPy/SciPy, the reference algorithm of the
StefanoCipolla/MF-PSIPM inner solve: PCG on ``H = A diag(1/theta) A' + delta I``
preconditioned by a Cholesky factor of a stable, leverage-ranked active
column core, together with the PS-IPM outer loop and the V3.1 HSD linear
algebra that call it.  Each function cites the reference ``file:line`` it
follows.

Who may use it: ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline
legs of ``bench.py`` — and only as the checker or the timed CPU baseline.  The
GPU product (``mf-psipm_b200/``) never imports it.

Factor: the reference factors the core with CHOLMOD (scikit-sparse), which is
not installed in this image.  The oracle uses SciPy's SuperLU in symmetric
mode without pivoting as a stand-in (``oracle.factor``); the same stand-in is
used when the reference itself is run to produce the golden fixtures.  So
"oracle" means "reference algorithm + SuperLU stand-in factor".  Converged
directions do not depend on the factor; PCG iteration counts do.

Parity pin: ``tests/golden/make_golden.py`` runs the unmodified reference
(with the same stand-in) on seeded instances and stores per-call inputs and
outputs; ``tests/test_oracle_pin.py`` checks this oracle against those
fixtures (bit-exact for index sets and scores, directions to round-off).
"""
