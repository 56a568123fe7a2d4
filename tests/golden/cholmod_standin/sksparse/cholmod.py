"""Test-only stand-in for ``sksparse.cholmod`` backed by SciPy's SuperLU.

The reference solvers (psipm_active_pool.py:66-81, 655-689) need CHOLMOD's
``cho_factor(M, lower=True, order=...)`` object with ``factorize(M)``,
``solve(b)`` and ``nnz``, plus the ``CholmodWarning`` and
``CholmodNotPositiveDefiniteError`` classes.  scikit-sparse is not installed
here, so this module reproduces that API subset with an LU factorisation in
symmetric mode without pivoting (``diag_pivot_thresh=0``), which for an SPD
matrix is the Cholesky factorisation up to a diagonal scaling.  A
non-positive pivot raises ``CholmodNotPositiveDefiniteError`` exactly where
CHOLMOD would report "not positive definite".

This module is used only to run the reference and the oracle as a checker;
it is never part of the GPU product.  Every parity report states that the
factor is "SuperLU stand-in, not CHOLMOD": converged Newton directions do not
depend on the factor, PCG iteration counts do.
"""

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla


class CholmodWarning(UserWarning):
    pass


class CholmodError(RuntimeError):
    pass


class CholmodNotPositiveDefiniteError(CholmodError):
    pass


def _lu(M):
    M = sp.csc_matrix(M)
    try:
        lu = spla.splu(
            M,
            permc_spec="MMD_AT_PLUS_A",
            diag_pivot_thresh=0.0,
            options=dict(SymmetricMode=True),
        )
    except RuntimeError as exc:  # exactly singular
        raise CholmodNotPositiveDefiniteError(str(exc)) from exc
    pivots = lu.U.diagonal()
    if not np.all(np.isfinite(pivots)) or np.any(pivots <= 0.0):
        raise CholmodNotPositiveDefiniteError("matrix not positive definite")
    return lu


class CholeskyFactor:
    def __init__(self, M):
        self._lu = _lu(M)

    def factorize(self, M):
        self._lu = _lu(M)

    def solve(self, b):
        return self._lu.solve(np.asarray(b, dtype=float))

    @property
    def nnz(self):
        return int(self._lu.L.nnz)


def cho_factor(M, lower=True, order="best"):
    del lower, order
    return CholeskyFactor(M)
