"""Oracle restatement of the stable / spectral active-column inner solve.

Test infrastructure (see ``oracle/__init__.py``).  Three layers, each citing
the reference code it restates:

* :class:`NormalEquationsOracle` — Jacobi-scaled factor of the assembled
  normal matrix with the diagonal shift ladder and the Woodbury low-rank
  correction (psipm_active_pool.py:691-996).
* :class:`StableOracle` — leverage scores, ``top_k``, stable core refresh,
  core assembly and the plain PCG solve (psipm_stable_preconditioner.py:97-517).
* :class:`SpectralOracle` — the spectral policy, custom PCG with residual
  replacement and Ritz estimates, retry with growth and the MINRES fallback
  (psipm_spectral_preconditioner.py:105-752).

The arithmetic follows the reference operation by operation (same NumPy /
SciPy calls in the same order), so that scores and index sets agree bit for
bit and directions to round-off.
"""

from __future__ import annotations

import time
from dataclasses import dataclass
from typing import Optional

import numpy as np
import scipy.linalg as la
import scipy.sparse as sp
import scipy.sparse.csgraph as csgraph
import scipy.sparse.linalg as spla

from .factor import StandInFactor

TINY = float(np.finfo(float).tiny)


class KKTSolveError(RuntimeError):
    """Raised where the reference raises ``KKTSolveError`` (psipm_active_pool.py)."""


def _squared(M: sp.csc_matrix) -> sp.csc_matrix:
    return sp.csc_matrix((np.square(M.data), M.indices, M.indptr), shape=M.shape, copy=False)


def low_rank_normal_columns(A, max_columns, min_nnz, clique_ratio) -> np.ndarray:
    """Columns kept out of the sparse factor (psipm_active_pool.py:691-717)."""
    if max_columns <= 0 or A.shape[1] == 0:
        return np.empty(0, dtype=np.int64)
    counts = np.diff(A.indptr).astype(float)
    edges = 0.5 * counts * np.maximum(counts - 1.0, 0.0)
    scale = max(float(A.nnz), float(A.shape[0]), 1.0)
    picked = np.flatnonzero((counts >= max(1, int(min_nnz))) & (edges >= float(clique_ratio) * scale))
    if picked.size > max_columns:
        keep = np.argpartition(edges[picked], -max_columns)[-max_columns:]
        picked = picked[keep]
    return np.sort(picked.astype(np.int64, copy=False))


def top_k(score: np.ndarray, count: int) -> np.ndarray:
    """Largest finite entries ordered by (score desc, index asc).

    Restates psipm_stable_preconditioner.py:97-110.  The reference selects with
    ``np.argpartition``; when a tie straddles the cut, which tied indices it
    keeps depends on NumPy's build (its AVX-512 argselect differs from the
    scalar introselect).  The oracle resolves ties by the rule the reference's
    own final ordering states — score first, then index — which is also the
    GPU rule.  Without a straddling tie both give the same set.
    """
    count = min(max(0, int(count)), score.size)
    if count == 0:
        return np.empty(0, dtype=np.int64)
    finite = np.flatnonzero(np.isfinite(score))
    if finite.size <= count:
        chosen = finite
    else:
        order = np.lexsort((finite, -score[finite]))
        chosen = finite[order[:count]]
    order = np.lexsort((chosen, -score[chosen]))
    return chosen[order].astype(np.int64, copy=False)


def top_k_numpy(score: np.ndarray, count: int) -> np.ndarray:
    """The reference's exact ``_top_k`` (argpartition, platform tie semantics)."""
    count = min(max(0, int(count)), score.size)
    if count == 0:
        return np.empty(0, dtype=np.int64)
    finite = np.flatnonzero(np.isfinite(score))
    if finite.size <= count:
        chosen = finite
    else:
        local = np.argpartition(score[finite], -count)[-count:]
        chosen = finite[local]
    order = np.lexsort((chosen, -score[chosen]))
    return chosen[order].astype(np.int64, copy=False)


def column_weighted_normal(A: sp.csc_matrix, weights: np.ndarray) -> sp.csc_matrix:
    """``A diag(weights) A'`` (psipm_active_pool.py:999-1006)."""
    columns = np.repeat(np.arange(A.shape[1]), np.diff(A.indptr))
    Ad = sp.csc_matrix((A.data * np.sqrt(weights)[columns], A.indices, A.indptr), shape=A.shape)
    return (Ad @ Ad.T).tocsc()


class NormalEquationsOracle:
    """Factor state of psipm_active_pool.py:720-996 (CHOLMOD replaced by the stand-in)."""

    SHIFTS = (0.0, 1e-14, 1e-12, 1e-10, 1e-8, 1e-6, 1e-4, 1e-2)

    def __init__(self, A, order="best", refine=2, refine_tol=1e-10, fail_tol=1e-6,
                 extract_low_rank=True, low_rank_max_columns=8, low_rank_min_nnz=1024,
                 low_rank_clique_ratio=2.0):
        self.A = A.tocsc()
        self.A.sum_duplicates()
        self.A.sort_indices()
        self.At = self.A.T.tocsr()
        self.m, self.n = A.shape
        self.low_rank_columns = (
            low_rank_normal_columns(self.A, int(low_rank_max_columns), int(low_rank_min_nnz),
                                    float(low_rank_clique_ratio))
            if extract_low_rank else np.empty(0, dtype=np.int64)
        )
        mask = np.ones(self.n, dtype=bool)
        mask[self.low_rank_columns] = False
        self.factor_columns = np.flatnonzero(mask)
        self.A_factor = self.A[:, self.factor_columns].tocsc()
        self.A_low_rank = self.A[:, self.low_rank_columns].tocsc()
        self.col_of_nz = np.repeat(np.arange(self.A_factor.shape[1]), np.diff(self.A_factor.indptr))
        self.I = sp.eye(self.m, format="csc")
        self._factor = None
        self._pattern = None
        self._col_of_nz_M = None
        self.order = order
        self.refine = max(0, int(refine))
        self.refine_tol = float(refine_tol)
        self.fail_tol = float(fail_tol)
        self.theta = None
        self.delta = 0.0
        self._dsc = None
        self._shift = 0.0
        self._verify = False
        self._low_rank_basis = None
        self._low_rank_chol = None
        self.n_shifted = 0
        self.n_refine = 0
        self.stats = {}
        self.n_symbolic = 0
        self.n_fact = 0
        self.n_solve = 0
        self.t_fact = 0.0
        self.t_solve = 0.0
        self.factor_attempts_failed = 0

    def _assemble(self, theta, delta):  # psipm_active_pool.py:828-837
        d = np.sqrt(1.0 / theta[self.factor_columns])
        Ad = sp.csc_matrix((self.A_factor.data * d[self.col_of_nz], self.A_factor.indices,
                            self.A_factor.indptr), shape=self.A_factor.shape)
        M = (Ad @ Ad.T + delta * self.I).tocsc()
        M.sort_indices()
        return M

    def factorize(self, theta, delta):  # psipm_active_pool.py:839-897
        t0 = time.perf_counter()
        M = self._assemble(theta, delta)
        fresh = self._factor is None or not (
            M.indptr.shape == self._pattern[0].shape
            and np.array_equal(M.indptr, self._pattern[0])
            and np.array_equal(M.indices, self._pattern[1])
        )
        if fresh:
            self._col_of_nz_M = np.repeat(np.arange(self.m), np.diff(M.indptr))
        diag = M.diagonal()
        dsc = 1.0 / np.sqrt(np.where(diag > 0.0, diag, 1.0))
        M.data *= dsc[M.indices] * dsc[self._col_of_nz_M]
        start = 0
        if self._shift > 0.0:
            start = max(0, int(np.searchsorted(self.SHIFTS, self._shift, side="left")) - 1)
        last_err = None
        for k in range(start, len(self.SHIFTS)):
            eta = self.SHIFTS[k]
            Ms = M if eta == 0.0 else (M + eta * self.I).tocsc()
            if eta:
                Ms.sort_indices()
            try:
                if fresh:
                    self._factor = StandInFactor(Ms, order=self.order)
                    self._pattern = (M.indptr.copy(), M.indices.copy())
                    self.n_symbolic += 1
                else:
                    self._factor.refactor(Ms)
            except Exception as exc:
                last_err = exc
                self.factor_attempts_failed += 1
                self._factor = None if fresh else self._factor
                continue
            self._shift = eta
            if eta:
                self.n_shifted += 1
            break
        else:
            self.t_fact += time.perf_counter() - t0
            raise KKTSolveError(f"Cholesky failed even with a 1e-2 shift ({last_err})")
        self._dsc = dsc
        self.theta = theta
        self.delta = delta
        try:
            self._prepare_low_rank_correction(theta)
        except Exception:
            self.t_fact += time.perf_counter() - t0
            raise
        self._verify = True
        self.n_fact += 1
        self.t_fact += time.perf_counter() - t0

    def _apply_base(self, r):  # psipm_active_pool.py:903-904
        return self._dsc * self._factor.solve(self._dsc * r)

    def _prepare_low_rank_correction(self, theta):  # psipm_active_pool.py:906-947
        count = self.low_rank_columns.size
        if not count:
            self._low_rank_basis = None
            self._low_rank_chol = None
            return
        basis = np.empty((self.m, count), dtype=float, order="F")
        rhs = np.zeros(self.m, dtype=float)
        for j in range(count):
            rhs.fill(0.0)
            lo, hi = self.A_low_rank.indptr[j], self.A_low_rank.indptr[j + 1]
            rhs[self.A_low_rank.indices[lo:hi]] = self.A_low_rank.data[lo:hi]
            basis[:, j] = self._apply_base(rhs)
        core = np.asarray(self.A_low_rank.T @ basis, dtype=float)
        core.flat[:: count + 1] += theta[self.low_rank_columns]
        core = 0.5 * (core + core.T)
        scale = max(float(np.max(np.abs(np.diag(core)))), 1.0)
        last_err = None
        for rel in (0.0, 1e-14, 1e-12, 1e-10, 1e-8):
            try:
                shifted = core if rel == 0.0 else core + rel * scale * np.eye(count)
                chol = np.linalg.cholesky(shifted)
            except np.linalg.LinAlgError as exc:
                last_err = exc
                continue
            self._low_rank_basis = basis
            self._low_rank_chol = chol
            return
        raise KKTSolveError(f"low-rank correction is not positive definite ({last_err})")

    def _apply(self, r):  # psipm_active_pool.py:949-956
        result = self._apply_base(r)
        if self._low_rank_chol is None:
            return result
        small = np.asarray(self.A_low_rank.T @ result).ravel()
        coef = np.linalg.solve(self._low_rank_chol, small)
        coef = np.linalg.solve(self._low_rank_chol.T, coef)
        return result - self._low_rank_basis @ coef

    @property
    def nnz_factor(self):
        return int(self._factor.nnz) if self._factor is not None else 0


class StableOracle(NormalEquationsOracle):
    """psipm_stable_preconditioner.py:113-517."""

    def __init__(self, A, protected=None, core_factor=1.0, max_core_factor=3.0, retention=0.9,
                 factor_max_age=2, core_max_age=12, refresh_cg=30, fill_weight=0.2,
                 cg_tol=1e-7, cg_tol_max=1e-2, forcing_factor=0.1, cg_maxit=200,
                 retry_growth=1.35, matching_backbone=True,
                 full_preconditioner_row_threshold=1500, full_preconditioner_clique_limit=2e8,
                 full_preconditioner_nnz_limit=10_000_000, adaptive_refresh_row_threshold=20_000,
                 **kwargs):
        if core_factor <= 0.0:
            raise ValueError("core_factor must be positive")
        if max_core_factor < core_factor:
            raise ValueError("max_core_factor must be at least core_factor")
        if not 0.0 <= retention <= 1.0:
            raise ValueError("retention must lie in [0, 1]")
        if fill_weight < 0.0:
            raise ValueError("fill_weight must be nonnegative")
        if retry_growth <= 1.0:
            raise ValueError("retry_growth must exceed one")
        if not 0.0 < cg_tol <= cg_tol_max < 1.0:
            raise ValueError("require 0 < cg_tol <= cg_tol_max < 1")
        if forcing_factor <= 0.0:
            raise ValueError("forcing_factor must be positive")
        super().__init__(A, **kwargs)
        counts_f = np.diff(self.A_factor.indptr).astype(np.int64)
        coupling = np.flatnonzero(counts_f >= 2)
        self.candidates = self.factor_columns[coupling]
        self.A_coupling = self.A_factor[:, coupling].tocsc()
        self.A2_coupling = _squared(self.A_coupling)
        self.A2_factor = _squared(self.A_factor)
        self.A2_low_rank = _squared(self.A_low_rank)
        counts = counts_f[coupling].astype(float)
        self.clique_burden = 0.5 * counts * np.maximum(counts - 1.0, 0.0)
        self.use_full_preconditioner = bool(
            self.m <= max(0, int(full_preconditioner_row_threshold))
            and self.A_factor.nnz <= max(0, int(full_preconditioner_nnz_limit))
            and float(self.clique_burden.sum()) <= float(full_preconditioner_clique_limit)
        )
        prot = np.zeros(self.n, dtype=bool)
        if protected is not None:
            supplied = np.asarray(protected, dtype=bool)
            if supplied.shape != (self.n,):
                raise ValueError("protected mask has the wrong dimension")
            prot[:] = supplied
        mandatory = self.candidates[prot[self.candidates]]
        self.matching_columns = np.empty(0, dtype=np.int64)
        if matching_backbone and not self.use_full_preconditioner and self.m and self.factor_columns.size:
            self.matching_columns = self._matching_on_candidates()
            mandatory = np.union1d(mandatory, self.matching_columns)
        self.mandatory = mandatory
        requested = max(1, int(np.ceil(float(core_factor) * self.m)))
        maximum = max(requested, int(np.ceil(float(max_core_factor) * self.m)))
        if self.use_full_preconditioner:
            requested = maximum = self.candidates.size
        self.core_target = min(self.candidates.size, max(requested, self.mandatory.size))
        self.max_core_target = min(self.candidates.size, max(maximum, self.mandatory.size))
        self.retention = float(retention)
        self.factor_max_age = 0 if self.use_full_preconditioner else max(0, int(factor_max_age))
        self.core_max_age = max(1, int(core_max_age))
        self.refresh_cg = max(1, int(refresh_cg))
        self.fill_weight = float(fill_weight)
        self.cg_tol = float(cg_tol)
        self.cg_tol_max = float(cg_tol_max)
        self.forcing_factor = float(forcing_factor)
        self.current_cg_tol = self.cg_tol
        self.cg_maxit = max(1, int(cg_maxit))
        self.retry_growth = float(retry_growth)
        self.adaptive_refresh_row_threshold = max(0, int(adaptive_refresh_row_threshold))
        self.core = np.empty(0, dtype=np.int64)
        self._weights = None
        self._diag_drop = np.zeros(self.m)
        self.factor_age = self.factor_max_age
        self.core_age = self.core_max_age
        self._initialized = False
        self._last_cg = self.refresh_cg
        self.core_sizes = []
        self.cg_iterations = []
        self.cg_failures = 0
        self.pcg_retries = 0
        self.full_fallbacks = 0
        self.refreshes = 0
        self.retained_fractions = []
        self.preconditioner_nnz = []
        self.cg_tolerances = []
        # per-call records, for parity reports
        self.core_history = []

    def _matching_on_candidates(self):
        """Structural matching columns that are candidates (psipm_stable_preconditioner.py:224-239)."""
        graph = self.A_factor.tocsr(copy=True)
        graph.data.fill(1.0)
        matched = csgraph.maximum_bipartite_matching(graph, perm_type="column")
        matched = matched[matched >= 0]
        glob = self.factor_columns[matched]
        pos = np.searchsorted(self.candidates, glob)
        valid = pos < self.candidates.size
        idx = np.flatnonzero(valid)
        valid[idx] &= self.candidates[pos[idx]] == glob[idx]
        return np.unique(glob[valid])

    def observe(self, x, z, w, s, mu):  # psipm_stable_preconditioner.py:285-291
        normalized = max(float(mu), 0.0) / (1.0 + max(float(mu), 0.0))
        self.current_cg_tol = min(self.cg_tol_max, max(self.cg_tol, float(self.forcing_factor * normalized)))

    def _scores(self, weights, delta):  # psipm_stable_preconditioner.py:293-309
        if not self.candidates.size:
            return np.empty(0)
        cw = weights[self.candidates]
        diagonal = np.asarray(self.A2_factor @ weights[self.factor_columns]).ravel()
        if self.low_rank_columns.size:
            diagonal += np.asarray(self.A2_low_rank @ weights[self.low_rank_columns]).ravel()
        diagonal += max(float(delta), TINY)
        inv = 1.0 / np.maximum(diagonal, TINY)
        leverage = cw * np.asarray(self.A2_coupling.T @ inv).ravel()
        return leverage / (1.0 + self.fill_weight * self.clique_burden)

    def _refresh_core(self, weights, delta, stable):  # psipm_stable_preconditioner.py:311-371
        if self.use_full_preconditioner:
            self.core = self.candidates.copy()
            self.retained_fractions.append(1.0)
            self.refreshes += 1
            self.core_age = 0
            self._initialized = True
            self.core_history.append(self.core.copy())
            return
        scores = self._scores(weights, delta)
        target = min(self.core_target, self.candidates.size)
        old = self.core
        parts = []
        if self.mandatory.size:
            parts.append(np.searchsorted(self.candidates, self.mandatory))
        if stable and old.size and target:
            old_local = np.searchsorted(self.candidates, old)
            keep = min(old.size, max(0, int(np.floor(self.retention * target))))
            if keep:
                parts.append(old_local[top_k(scores[old_local], keep)])
        fixed = np.unique(np.concatenate(parts)) if parts else np.empty(0, dtype=np.int64)
        if fixed.size > target:
            mcount = self.mandatory.size
            if mcount >= target:
                fixed = np.searchsorted(self.candidates, self.mandatory)[:target]
            else:
                mloc = np.searchsorted(self.candidates, self.mandatory)
                optional = fixed[~np.isin(fixed, mloc, assume_unique=True)]
                fixed = np.concatenate([mloc, optional[top_k(scores[optional], target - mcount)]])
        remaining = target - fixed.size
        if remaining > 0:
            avail = scores.copy()
            avail[fixed] = -np.inf
            fixed = np.concatenate([fixed, top_k(avail, remaining)])
        new_core = np.sort(self.candidates[np.unique(fixed)])
        retained = (float(np.intersect1d(old, new_core, assume_unique=True).size) / max(1, old.size)
                    if old.size else 1.0)
        self.core = new_core
        self.retained_fractions.append(retained)
        self.refreshes += 1
        self.core_age = 0
        self._initialized = True
        self.core_history.append(new_core.copy())

    def _assemble(self, theta, delta):  # psipm_stable_preconditioner.py:373-395
        weights = self._weights
        if self.core.size:
            Ac = self.A[:, self.core].tocsc()
            matrix = column_weighted_normal(Ac, weights[self.core])
            core_local = np.searchsorted(self.candidates, self.core)
            diag_core = np.asarray(self.A2_coupling[:, core_local] @ weights[self.core]).ravel()
        else:
            matrix = sp.csc_matrix((self.m, self.m))
            diag_core = np.zeros(self.m)
        diag_full = np.asarray(self.A2_factor @ weights[self.factor_columns]).ravel()
        self._diag_drop = np.maximum(diag_full - diag_core, 0.0)
        matrix = (matrix + sp.diags(self._diag_drop + float(delta), format="csc")).tocsc()
        matrix.sort_indices()
        return matrix

    def factorize(self, theta, delta):  # psipm_stable_preconditioner.py:397-432
        theta = np.asarray(theta, dtype=float)
        self._weights = 1.0 / theta
        poor = self._last_cg >= self.refresh_cg
        can_grow = self.core_target < self.max_core_target
        refresh = (not self._initialized or self.core_age >= self.core_max_age
                   or (poor and (can_grow or self.m <= self.adaptive_refresh_row_threshold)))
        refactor = self._factor is None or self.factor_age >= self.factor_max_age or refresh or poor
        if refresh:
            self._refresh_core(self._weights, delta, stable=bool(self.core.size))
        if refactor:
            NormalEquationsOracle.factorize(self, theta, delta)
            self.factor_age = 0
            self.preconditioner_nnz.append(self.nnz_factor)
        else:
            self.theta = theta
            self.delta = float(delta)
            self.factor_age += 1
        self.core_age += 1
        self.core_sizes.append(int(self.core.size))

    def _full_matvec(self, v):  # psipm_stable_preconditioner.py:434-438
        return np.asarray(self.A @ (self._weights * (self.At @ v)) + self.delta * v).ravel()

    def _pcg(self, rhs):  # psipm_stable_preconditioner.py:440-464 (SciPy cg)
        iterations = 0

        def count(_):
            nonlocal iterations
            iterations += 1

        op = spla.LinearOperator((self.m, self.m), matvec=self._full_matvec)
        pre = spla.LinearOperator((self.m, self.m), matvec=self._apply)
        x0 = self._apply(rhs)
        sol, info = spla.cg(op, rhs, x0=x0, M=pre, rtol=self.current_cg_tol, atol=0.0,
                            maxiter=self.cg_maxit, callback=count)
        scale = max(float(np.linalg.norm(rhs)), 1.0)
        rel = float(np.linalg.norm(rhs - self._full_matvec(sol)) / scale)
        return sol, info, iterations, rel

    def solve(self, r1, r2):  # psipm_stable_preconditioner.py:466-517
        started = time.perf_counter()
        fb = self.t_fact
        w = r1 / self.theta
        rhs = np.asarray(r2 - self.A @ w).ravel()
        dy, info, iterations, rel = self._pcg(rhs)
        self.cg_tolerances.append(self.current_cg_tol)
        acceptable = max(self.fail_tol, 2.0 * self.current_cg_tol)
        failed = info != 0 or not np.isfinite(rel) or rel > acceptable
        if failed and self.core_target < self.max_core_target:
            self.pcg_retries += 1
            grown = max(self.core_target + 1, int(np.ceil(self.retry_growth * self.core_target)))
            self.core_target = min(self.max_core_target, grown)
            self._refresh_core(self._weights, self.delta, stable=True)
            NormalEquationsOracle.factorize(self, self.theta, self.delta)
            self.factor_age = 0
            self.core_sizes.append(int(self.core.size))
            self.preconditioner_nnz.append(self.nnz_factor)
            dy, info, more, rel = self._pcg(rhs)
            iterations += more
            failed = info != 0 or not np.isfinite(rel) or rel > acceptable
        self.cg_iterations.append(iterations)
        self._last_cg = iterations
        if failed:
            self.cg_failures += 1
            self.t_solve += max(0.0, time.perf_counter() - started - (self.t_fact - fb))
            raise KKTSolveError(f"stable active-column PCG failed: info={info}, "
                                f"relative residual={rel:.2e}, iterations={iterations}")
        dx = w + (self.At @ dy) / self.theta
        self.n_solve += 1
        self.t_solve += max(0.0, time.perf_counter() - started - (self.t_fact - fb))
        return dx, dy


@dataclass
class KrylovResult:
    """psipm_spectral_preconditioner.py:105-116."""

    solution: np.ndarray
    info: int
    iterations: int
    relative_residual: float
    condition_estimate: float
    spectral_error_estimate: float
    residual: np.ndarray
    replacements: int
    residual_checks: int
    stagnated: bool
    alphas: tuple = ()
    betas: tuple = ()


def ritz_estimate(alphas, betas):
    """Extremal Ritz values of the CG Lanczos tridiagonal (psipm_spectral_preconditioner.py:119-140)."""
    count = len(alphas)
    if count == 0:
        return 1.0, 1.0, 1.0
    diagonal = np.empty(count)
    diagonal[0] = 1.0 / alphas[0]
    if count > 1:
        beta = np.asarray(betas[: count - 1])
        alpha = np.asarray(alphas)
        diagonal[1:] = 1.0 / alpha[1:] + beta / alpha[:-1]
        off = np.sqrt(np.maximum(beta, 0.0)) / alpha[:-1]
        eig = la.eigvalsh_tridiagonal(diagonal, off, check_finite=False)
    else:
        eig = diagonal
    lo, hi = float(eig[0]), float(eig[-1])
    if not np.isfinite(lo) or lo <= 0.0:
        return lo, hi, np.inf
    return lo, hi, hi / lo


class SpectralOracle(StableOracle):
    """psipm_spectral_preconditioner.py:143-752."""

    def __init__(self, A, protected=None, weighted_backbone=False, structural_backbone=True,
                 matching_max_rows=50_000, matching_max_nnz=25_000_000,
                 matching_refresh_max_rows=20_000, backbone_max_age=20, residual_score_weight=0.0,
                 swap_patience=2, condition_limit=1e12, lag_spectral_ratio=1e8,
                 residual_replacement=100, residual_gap_tolerance=0.1, stagnation_window=3,
                 stagnation_reduction=0.8, corrector_tightening=1.0, minres_fallback=True,
                 minres_maxit=400, minres_max_dimension=200_000, **kwargs):
        super().__init__(A, protected=protected, matching_backbone=False, **kwargs)
        if weighted_backbone:
            raise NotImplementedError("the weighted backbone is off in the reference defaults")
        self.weighted_backbone = False
        self.structural_backbone = bool(structural_backbone)
        self.backbone_max_age = max(1, int(backbone_max_age))
        self.residual_score_weight = max(0.0, float(residual_score_weight))
        self.swap_patience = max(1, int(swap_patience))
        self.condition_limit = max(1.0, float(condition_limit))
        self.lag_spectral_ratio = max(1.0, float(lag_spectral_ratio))
        self.residual_replacement = max(0, int(residual_replacement))
        self.residual_gap_tolerance = max(np.sqrt(np.finfo(float).eps), float(residual_gap_tolerance))
        self.stagnation_window = max(2, int(stagnation_window))
        self.stagnation_reduction = float(stagnation_reduction)
        self.corrector_tightening = min(1.0, max(0.01, float(corrector_tightening)))
        self.minres_fallback = bool(minres_fallback)
        self.minres_maxit = max(1, int(minres_maxit))
        self.minres_max_dimension = max(0, int(minres_max_dimension))
        self.protected_mandatory = self.mandatory.copy()
        self.matching_columns = np.empty(0, dtype=np.int64)
        self.mandatory = self.protected_mandatory.copy()
        self.backbone_age = self.backbone_max_age
        self.weighted_backbone_refreshes = 0
        self._enrichment_vector = None
        self._reference_weights = None
        self._reference_delta = None
        self._factor_generation = 0
        self._poor_streak = 0
        self._last_condition = 1.0
        self._last_spectral_error = 0.0
        self._last_stagnated = False
        self._rhs_index = 0
        self._nonlinear_residual = None
        self._previous_nonlinear_residual = None
        self._ew_tolerance = self.cg_tol_max
        self.condition_estimates = []
        self.spectral_error_estimates = []
        self.lag_spectral_bounds = []
        self.residual_replacements = 0
        self.residual_checks = 0
        self.stagnation_events = 0
        self.core_swaps = 0
        self.minres_fallbacks = 0
        self.minres_iterations = 0
        self.krylov_breakdowns = 0
        self.krylov_iteration_limits = 0
        self.last_result: Optional[KrylovResult] = None

    def set_ipm_context(self, res_d, res_p, res_n, tol):  # :230-250
        current = max(float(res_n), float(np.linalg.norm(res_d)), float(np.linalg.norm(res_p)), TINY)
        previous = self._nonlinear_residual
        self._previous_nonlinear_residual = previous
        self._nonlinear_residual = current
        if previous is None or not np.isfinite(previous):
            estimate = self.cg_tol_max
        else:
            estimate = 0.9 * (current / max(previous, TINY)) ** 1.5
        self._ew_tolerance = min(self.cg_tol_max, max(self.cg_tol, float(tol) * 0.1, estimate))
        self._rhs_index = 0

    def observe(self, x, z, w, s, mu):  # :252-258
        normalized = max(float(mu), 0.0) / (1.0 + max(float(mu), 0.0))
        mu_tol = self.forcing_factor * normalized
        self.current_cg_tol = min(self.cg_tol_max, max(self.cg_tol, min(mu_tol, self._ew_tolerance)))

    def _linear_tolerance(self):  # :260-265
        tol = self.current_cg_tol
        if self._rhs_index:
            tol = max(self.cg_tol, self.corrector_tightening * tol)
        self._rhs_index += 1
        return float(tol)

    def _structural_matching(self):  # :307-326
        if not self.structural_backbone or self.use_full_preconditioner or not self.m \
                or not self.factor_columns.size:
            return np.empty(0, dtype=np.int64)
        return self._matching_on_candidates()

    def _update_backbone(self, weights, force=False):  # :328-365 (structural branch)
        if self.matching_columns.size:
            return
        matching = self._structural_matching()
        if matching.size:
            self.matching_columns = matching
            self.mandatory = np.union1d(self.protected_mandatory, matching)
            self.core_target = min(self.candidates.size, max(self.core_target, self.mandatory.size))
            self.max_core_target = min(self.candidates.size, max(self.max_core_target, self.mandatory.size))
            self.weighted_backbone_refreshes += 1

    def _scores(self, weights, delta):  # :367-386 (enrichment inactive at weight 0)
        scores = super()._scores(weights, delta)
        vector = self._enrichment_vector
        if not scores.size or vector is None or vector.size != self.m or self.residual_score_weight == 0.0:
            return scores
        norm = float(np.linalg.norm(vector))
        if not np.isfinite(norm) or norm == 0.0:
            return scores
        vector = vector / norm
        products = np.asarray(self.A_coupling.T @ vector).ravel()
        diag = np.asarray(self.A2_coupling.T @ np.square(vector)).ravel()
        impact = weights[self.candidates] * np.abs(np.square(products) - diag)
        impact /= 1.0 + self.fill_weight * self.clique_burden
        sscale = float(np.max(scores, initial=0.0))
        iscale = float(np.max(impact, initial=0.0))
        if iscale > 0.0 and np.isfinite(iscale):
            scores = scores + self.residual_score_weight * max(sscale, 1.0) * (impact / iscale)
        return scores

    def _refresh_core(self, weights, delta, stable, force_backbone=False):  # :388-394
        old = self.core.copy()
        self._update_backbone(weights, force=force_backbone or not self._initialized)
        super()._refresh_core(weights, delta, stable)
        if old.size and self.core.size:
            changed = old.size - np.intersect1d(old, self.core, assume_unique=True).size
            self.core_swaps += max(0, int(changed))

    def _lag_bound(self, weights, delta):  # :396-410
        if self._reference_weights is None:
            return np.inf
        ratio = weights / np.maximum(self._reference_weights, TINY)
        finite = ratio[np.isfinite(ratio) & (ratio > 0.0)]
        if finite.size != ratio.size:
            return np.inf
        bound = max(float(finite.max()), 1.0 / float(finite.min()))
        if self._reference_delta > 0.0 and delta > 0.0:
            dr = delta / self._reference_delta
            bound = max(bound, dr, 1.0 / dr)
        elif delta != self._reference_delta:
            return np.inf
        return float(bound)

    def _factor_current(self, theta, delta):  # :412-418
        NormalEquationsOracle.factorize(self, theta, delta)
        self.factor_age = 0
        self._reference_weights = self._weights.copy()
        self._reference_delta = float(delta)
        self._factor_generation += 1
        self.preconditioner_nnz.append(self.nnz_factor)

    def factorize(self, theta, delta):  # :420-467
        theta = np.asarray(theta, dtype=float)
        self._weights = 1.0 / theta
        spectral_poor = (self._last_condition >= self.condition_limit
                         and self._last_cg >= max(10, int(0.8 * self.refresh_cg)))
        poor = self._last_cg >= self.refresh_cg or spectral_poor or self._last_stagnated
        self._poor_streak = self._poor_streak + 1 if poor else 0
        can_grow = self.core_target < self.max_core_target
        swap_due = poor and not can_grow and self._poor_streak >= self.swap_patience
        refresh = not self._initialized or self.core_age >= self.core_max_age or (poor and can_grow) or swap_due
        if refresh:
            self._refresh_core(self._weights, delta, stable=bool(self.core.size), force_backbone=swap_due)
            self._poor_streak = 0
        lag = self._lag_bound(self._weights, float(delta))
        self.lag_spectral_bounds.append(lag)
        refactor = (self._factor is None or self.factor_age >= self.factor_max_age or refresh or poor
                    or lag > self.lag_spectral_ratio)
        if refactor:
            self._factor_current(theta, float(delta))
        else:
            self.theta = theta
            self.delta = float(delta)
            self.factor_age += 1
        self.core_age += 1
        self.core_sizes.append(int(self.core.size))
        self.backbone_age += 1

    def _pcg(self, rhs, tolerance):  # :469-581
        scale = max(1.0, float(np.linalg.norm(rhs)))
        x = self._apply(rhs)
        r = np.asarray(rhs - self._full_matvec(x)).ravel()
        z = np.asarray(self._apply(r)).ravel()
        rz = float(r @ z)
        p = z.copy()
        alphas, betas = [], []
        replacements = 0
        checks = 0
        history = [float(np.linalg.norm(r)) / scale]
        info = self.cg_maxit
        it = 0
        if history[-1] <= tolerance:
            info = 0
        elif not np.isfinite(rz) or rz <= 0.0:
            info = -1
        while info > 0 and it < self.cg_maxit:
            q = np.asarray(self._full_matvec(p)).ravel()
            curv = float(p @ q)
            floor = TINY * max(1.0, float(np.linalg.norm(p)) * float(np.linalg.norm(q)))
            if not np.isfinite(curv) or curv <= floor:
                info = -2
                break
            alpha = rz / curv
            if not np.isfinite(alpha) or alpha <= 0.0:
                info = -3
                break
            x += alpha * p
            r -= alpha * q
            it += 1
            alphas.append(alpha)
            rec = float(np.linalg.norm(r)) / scale
            replace = self.residual_replacement > 0 and it % self.residual_replacement == 0
            if replace or rec <= tolerance:
                true_r = np.asarray(rhs - self._full_matvec(x)).ravel()
                checks += 1
                tnorm = float(np.linalg.norm(true_r))
                rel = tnorm / scale
                history.append(rel)
                if not np.isfinite(rel):
                    info = -4
                    break
                if rel <= tolerance:
                    r = true_r
                    info = 0
                    break
                gap = float(np.linalg.norm(true_r - r))
                if gap > self.residual_gap_tolerance * max(tnorm, tolerance * scale):
                    r = true_r
                    replacements += 1
                    z = np.asarray(self._apply(r)).ravel()
                    rz = float(r @ z)
                    if not np.isfinite(rz) or rz <= 0.0:
                        info = -5
                        break
                    p = z.copy()
                    alphas.clear()
                    betas.clear()
                    continue
            z = np.asarray(self._apply(r)).ravel()
            rz_next = float(r @ z)
            if not np.isfinite(rz_next) or rz_next <= 0.0:
                info = -6
                break
            beta = rz_next / rz
            if not np.isfinite(beta) or beta < 0.0:
                info = -7
                break
            betas.append(beta)
            p = z + beta * p
            rz = rz_next
        r = np.asarray(rhs - self._full_matvec(x)).ravel()
        rel = float(np.linalg.norm(r)) / scale
        if info > 0 and rel <= tolerance:
            info = 0
        lo, hi, cond = ritz_estimate(alphas, betas)
        w = self.stagnation_window
        stagnated = len(history) >= w and history[-1] > self.stagnation_reduction * history[-w]
        return KrylovResult(x, info, it, rel, float(cond), float(max(abs(lo - 1.0), abs(hi - 1.0))),
                            r, replacements, checks, bool(stagnated), tuple(alphas), tuple(betas))

    def _minres(self, r1, r2, tolerance):  # :583-637
        size = self.n + self.m
        iterations = 0

        def matvec(v):
            dx = v[: self.n]
            q = v[self.n:]
            return np.concatenate([self.theta * dx + self.At @ q, self.A @ dx - self.delta * q])

        def precondition(v):
            return np.concatenate([v[: self.n] / self.theta, self._apply(v[self.n:])])

        def count(_):
            nonlocal iterations
            iterations += 1

        op = spla.LinearOperator((size, size), matvec=matvec, dtype=float)
        pre = spla.LinearOperator((size, size), matvec=precondition, dtype=float)
        rhs = np.concatenate([r1, r2])
        scale = max(1.0, float(np.linalg.norm(rhs)))
        target = max(2.0 * float(tolerance), self.fail_tol)
        sol = np.zeros_like(rhs)
        for _ in range(3):
            corr_rhs = rhs - matvec(sol)
            rel = float(np.linalg.norm(corr_rhs)) / scale
            if np.isfinite(rel) and rel <= target:
                break
            corr, info = spla.minres(op, corr_rhs, M=pre, rtol=max(np.finfo(float).eps, min(float(tolerance), 1e-8)),
                                     maxiter=self.minres_maxit, callback=count, check=False)
            sol += corr
            if info < 0:
                break
        rel = float(np.linalg.norm(rhs - matvec(sol))) / scale
        accepted = np.isfinite(rel) and rel <= target
        return sol[: self.n], -sol[self.n:], accepted, iterations, rel

    def _record_krylov(self, res):  # :639-649
        self._last_cg = int(res.iterations)
        self._last_condition = float(res.condition_estimate)
        self._last_spectral_error = float(res.spectral_error_estimate)
        self._last_stagnated = bool(res.stagnated)
        self._enrichment_vector = res.residual.copy()
        self.condition_estimates.append(self._last_condition)
        self.spectral_error_estimates.append(self._last_spectral_error)
        self.residual_replacements += int(res.replacements)
        self.residual_checks += int(res.residual_checks)
        self.stagnation_events += int(res.stagnated)

    def solve(self, r1, r2):  # :651-752
        started = time.perf_counter()
        fb = self.t_fact
        wr1 = r1 / self.theta
        rhs = np.asarray(r2 - self.A @ wr1).ravel()
        tol = self._linear_tolerance()
        res = self._pcg(rhs, tol)
        total = res.iterations
        failed = res.info != 0 or not np.isfinite(res.relative_residual) or res.relative_residual > tol
        can_grow = self.core_target < self.max_core_target
        warranted = can_grow or res.info < 0 or res.stagnated
        if failed and warranted and self.candidates.size and not self.use_full_preconditioner:
            self.pcg_retries += 1
            self._enrichment_vector = res.residual.copy()
            if self.core_target < self.max_core_target:
                grown = max(self.core_target + 1, int(np.ceil(self.retry_growth * self.core_target)))
                self.core_target = min(self.max_core_target, grown)
            self._refresh_core(self._weights, self.delta, stable=True,
                               force_backbone=res.info < 0 or res.stagnated)
            self._factor_current(self.theta, self.delta)
            self.core_sizes.append(int(self.core.size))
            res = self._pcg(rhs, tol)
            total += res.iterations
            failed = res.info != 0 or not np.isfinite(res.relative_residual) or res.relative_residual > tol
        if failed and res.relative_residual <= max(2.0 * tol, self.fail_tol):
            failed = False
        self.cg_tolerances.append(tol)
        self.cg_iterations.append(total)
        self._record_krylov(res)
        self.last_result = res
        if res.info < 0:
            self.krylov_breakdowns += 1
        elif res.info > 0:
            self.krylov_iteration_limits += 1
        if not failed:
            dy = res.solution
            dx = wr1 + (self.At @ dy) / self.theta
        elif (self.minres_fallback and self.n + self.m <= self.minres_max_dimension
              and (res.info < 0 or res.stagnated)):
            self.cg_failures += 1
            self.minres_fallbacks += 1
            dx, dy, accepted, iters, rel = self._minres(r1, r2, tol)
            self.minres_iterations += iters
            self.full_fallbacks += 1
            if not accepted:
                self.t_solve += max(0.0, time.perf_counter() - started - (self.t_fact - fb))
                raise KKTSolveError(f"spectral PCG and augmented MINRES failed: pcg info={res.info}, "
                                    f"pcg residual={res.relative_residual:.2e}, minres residual={rel:.2e}")
        else:
            self.cg_failures += 1
            self.t_solve += max(0.0, time.perf_counter() - started - (self.t_fact - fb))
            raise KKTSolveError(f"spectral stable-column PCG failed: info={res.info}, "
                                f"residual={res.relative_residual:.2e}")
        self.n_solve += 1
        self.t_solve += max(0.0, time.perf_counter() - started - (self.t_fact - fb))
        return dx, dy
