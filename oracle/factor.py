"""SuperLU stand-in for the CHOLMOD factor — test infrastructure.

The reference wraps CHOLMOD in ``_CholFactor`` (psipm_active_pool.py:655-689):
``__init__`` = symbolic + numeric factorisation, ``refactor`` = numeric only,
``solve``, ``nnz``.  CHOLMOD is unavailable here, so this class keeps that
interface on top of ``scipy.sparse.linalg.splu`` in symmetric mode with no
pivoting.  A non-positive or non-finite pivot raises ``NotPositiveDefinite``,
the condition CHOLMOD reports as "not positive definite".  The golden
fixtures were generated by the reference running on the identical stand-in
(``tests/golden/cholmod_standin``), so oracle and reference share the factor.
"""

from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla


class NotPositiveDefinite(RuntimeError):
    pass


def _factor(M):
    M = sp.csc_matrix(M)
    try:
        lu = spla.splu(
            M,
            permc_spec="MMD_AT_PLUS_A",
            diag_pivot_thresh=0.0,
            options=dict(SymmetricMode=True),
        )
    except RuntimeError as exc:
        raise NotPositiveDefinite(str(exc)) from exc
    pivots = lu.U.diagonal()
    if not np.all(np.isfinite(pivots)) or np.any(pivots <= 0.0):
        raise NotPositiveDefinite("matrix not positive definite")
    return lu


class StandInFactor:
    """``_CholFactor`` interface (psipm_active_pool.py:655-689) over SuperLU."""

    def __init__(self, M, order: str = "best"):
        del order
        self._lu = _factor(M)

    def refactor(self, M) -> None:
        self._lu = _factor(M)

    def solve(self, b):
        return self._lu.solve(np.asarray(b, dtype=float))

    @property
    def nnz(self) -> int:
        return int(self._lu.L.nnz)
