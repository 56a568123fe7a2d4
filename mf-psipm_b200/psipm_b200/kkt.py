"""Drop-in KKT solvers whose arithmetic runs on the B200.

:class:`GpuSpectralStableColumnPreconditioner` has the constructor,
methods, attributes and exceptions of the reference's
``SpectralStableColumnPreconditioner`` (psipm_spectral_preconditioner.py:143-752)
and so plugs into ``psipm_solve(lp, kkt_solver=...)``
(psipm_active_pool.py:2277, 2423-2426) unchanged:

* ``factorize(theta, delta)`` — the spectral refresh / refactor policy
  (:420-467) runs here on the host; scores, core refresh, assembly and the
  Cholesky factorisation run on the device.
* ``solve(r1, r2)`` — ``(dx, dy)`` from the persistent device PCG (:469-581)
  plus the retry-with-growth logic (:651-752).
* ``observe`` / ``set_ipm_context`` — inexact-Newton forcing (:230-258).

:class:`GpuStableColumnPreconditioner` is the V3.1 HSD preconditioner
surface (psipm_v3_1_hsd.py:823-989) and :func:`pcg_rows` the device
replacement of its ``_pcg`` (:1015-1063); :mod:`psipm_b200.hsd` builds the
reduced HSD Newton system (:1066-1264) on top of both.

There is no CPU fallback: without the CUDA library every constructor raises
``GpuUnavailable``.
"""

from __future__ import annotations

import math
import time
from dataclasses import dataclass
from typing import Optional

import numpy as np
import scipy.linalg as la
import scipy.sparse as sp
import scipy.sparse.csgraph as csgraph

from . import _lib
from .device import DeviceError, NormalEquationsDevice
from .roofline import pcg_launch_bytes

TINY = float(np.finfo(float).tiny)
EPS = float(np.finfo(float).eps)
SHIFTS = (0.0, 1e-14, 1e-12, 1e-10, 1e-8, 1e-6, 1e-4, 1e-2)


class KKTSolveError(RuntimeError):
    """Same role as psipm_active_pool.KKTSolveError (psipm_active_pool.py:553)."""


class _Resident:
    """Stands for a theta that already lives on the device (psipm_ipm_theta).

    The device-resident IPM (ipm_device.py) passes it to ``factorize`` in place
    of a host array; the policy then skips the host->device copy and computes
    the lag bound on the device.
    """

    def __repr__(self) -> str:
        return "RESIDENT"


RESIDENT = _Resident()


def low_rank_normal_columns(A, max_columns, min_nnz, clique_ratio):
    """Columns a Woodbury update would carry (psipm_active_pool.py:691-717)."""
    if max_columns <= 0 or A.shape[1] == 0:
        return np.empty(0, dtype=np.int64)
    counts = np.diff(A.indptr).astype(float)
    edges = 0.5 * counts * np.maximum(counts - 1.0, 0.0)
    scale = max(float(A.nnz), float(A.shape[0]), 1.0)
    picked = np.flatnonzero((counts >= max(1, int(min_nnz))) & (edges >= float(clique_ratio) * scale))
    if picked.size > max_columns:
        picked = picked[np.argpartition(edges[picked], -max_columns)[-max_columns:]]
    return np.sort(picked.astype(np.int64, copy=False))


def ritz_estimate(alphas, betas):
    """Extremal Ritz values of the PCG Lanczos tridiagonal (psipm_spectral_preconditioner.py:119-140)."""
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


@dataclass
class KrylovResult:
    """psipm_spectral_preconditioner.py:105-116."""

    solution: np.ndarray
    info: int
    iterations: int
    relative_residual: float
    condition_estimate: float
    spectral_error_estimate: float
    residual: Optional[np.ndarray]
    replacements: int
    residual_checks: int
    stagnated: bool
    seconds: float = 0.0


class GpuStableActiveColumnPreconditioner:
    """Device version of StableActiveColumnPreconditioner (psipm_stable_preconditioner.py:113-517).

    Holds the stable-rule policy state; everything proportional to the LP's
    size (weights, diagonals, scores, top-k, assembly, factor, PCG) lives on
    the device.
    """

    def __init__(self, A, protected=None, core_factor=1.0, max_core_factor=3.0, retention=0.9,
                 factor_max_age=2, core_max_age=12, refresh_cg=30, fill_weight=0.2, cg_tol=1e-7,
                 cg_tol_max=1e-2, forcing_factor=0.1, cg_maxit=200, retry_growth=1.35,
                 matching_backbone=True, full_preconditioner_row_threshold=1500,
                 full_preconditioner_clique_limit=2e8, full_preconditioner_nnz_limit=10_000_000,
                 adaptive_refresh_row_threshold=20_000, order="best", refine=2, refine_tol=1e-10,
                 fail_tol=1e-6, extract_low_rank=True, low_rank_max_columns=8, low_rank_min_nnz=1024,
                 low_rank_clique_ratio=2.0, device=0, precision=_lib.FP64, dev=None, selector=None,
                 selector_patience=2, selector_shift=True, selector_window=0.0, deterministic=False,
                 factor_tc=3):
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
        A = sp.csc_matrix(A)
        A.sum_duplicates()
        A.sort_indices()
        self.A = A
        self.m, self.n = A.shape
        self.low_rank_columns = (low_rank_normal_columns(A, int(low_rank_max_columns), int(low_rank_min_nnz),
                                                         float(low_rank_clique_ratio))
                                 if extract_low_rank else np.empty(0, dtype=np.int64))
        if self.low_rank_columns.size and precision != _lib.FP64:
            raise NotImplementedError("Woodbury-extracted dense columns need the FP64 device factor")
        # an existing device handle for the same A may be reused (its matrix
        # upload is skipped); its core is cleared so the policy starts afresh
        self.dev = dev if dev is not None else NormalEquationsDevice(A, device=device, precision=precision)
        if dev is not None:
            if dev.A.shape != A.shape or dev.A.nnz != A.nnz:
                raise ValueError("the device handle holds a different matrix")
            dev.set_core(np.empty(0, dtype=np.int64))
        self.precision = precision
        if deterministic:  # bit-repeatable runs (slower applies)
            self.dev.set_deterministic(True)
        if factor_tc != 3:  # FP32 big fronts: 3xTF32 tensor cores (3, the default), TF32 (1), CUDA cores (0)
            self.dev.set_factor_tc(int(factor_tc))
        if self.low_rank_columns.size:
            # the factor leaves these columns out and corrects for them by
            # Woodbury (psipm_active_pool.py:786-798, 906-956)
            self.dev.set_low_rank(self.low_rank_columns)
        self.factor_columns = np.setdiff1d(np.arange(self.n, dtype=np.int64), self.low_rank_columns)
        self.candidates = self.dev.candidates
        counts = np.diff(A.indptr)[self.candidates].astype(float)
        self.clique_burden = 0.5 * counts * np.maximum(counts - 1.0, 0.0)
        factor_nnz = A.nnz - int(np.diff(A.indptr)[self.low_rank_columns].sum())
        self.use_full_preconditioner = bool(
            self.m <= max(0, int(full_preconditioner_row_threshold))
            and factor_nnz <= max(0, int(full_preconditioner_nnz_limit))
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
        if matching_backbone and not self.use_full_preconditioner and self.m and self.n:
            self.matching_columns = self._matching()
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
        self.fail_tol = float(fail_tol)
        self.order = order
        self.refine = max(0, int(refine))
        # state
        self.core = np.empty(0, dtype=np.int64)
        self._weights = None
        self.theta = None
        self.delta = 0.0
        self._has_factor = False
        self._shift = 0.0
        self.factor_age = self.factor_max_age
        self.core_age = self.core_max_age
        self._initialized = False
        self._last_cg = self.refresh_cg
        # statistics with the reference's names (psipm_active_pool.py:2683-2743)
        self.n_fact = 0
        self.n_solve = 0
        self.t_fact = 0.0
        self.t_solve = 0.0
        self.n_shifted = 0
        self.n_refine = 0
        self.n_symbolic = 0
        self.stats = {"not_pd": 0}
        self.core_sizes = []
        self.cg_iterations = []
        self.cg_failures = 0
        self.pcg_retries = 0
        self.full_fallbacks = 0
        self.refreshes = 0
        self.retained_fractions = []
        self.preconditioner_nnz = []
        self.cg_tolerances = []
        self.nnz_factor = 0
        self.last_factor_info = None
        self.device_seconds = 0.0
        self.core_history = []
        self.tie_straddles = 0
        self.memory_caps = 0  # core targets lowered because a factor did not fit in device memory
        self._largest_fit = 0  # size of the largest core factored so far
        # learned selector (no counterpart in the reference): a SelectorModel that
        # re-scores the candidates before the rule's refresh; a learned core that
        # turns out poor by the rule's own signals suspends it for
        # `selector_patience` refreshes (GpuSpectralStableColumnPreconditioner.factorize)
        self.selector = selector
        self.selector_patience = max(1, int(selector_patience))
        self.selector_shift = bool(selector_shift)
        # > 1: the network only reorders the rule's best selector_window x target candidates
        self.selector_window = float(selector_window)
        self._selector_pause = 0
        self._core_learned = False
        self._shift_vote = 0.0
        self.learned_refreshes = 0
        self.selector_fallbacks = 0
        self.mu = 1.0
        self.delta_now = 0.0
        self.trace_hook = None   # called at each refresh after the rule's scores (training traces)
        self.factor_hook = None  # called after each factorisation with the shift index used
        # device PCG launches: count, iterations, H·p products, k_pcg seconds
        self.pcg_launches = 0
        self.pcg_total_iterations = 0
        self.pcg_matvecs = 0
        self.pcg_replacements = 0
        self.pcg_bytes = 0.0  # algorithmic bytes of all PCG launches (roofline numerator)
        self.pcg_phase_seconds = np.zeros(4)  # H·p, updates, applies, other (device clock)
        self.refinement_sweeps = 0  # FP64 refinement sweeps around FP32 PCG (FP32_REFINED)
        # host<->device traffic through the C ABI (bytes)
        self.h2d_bytes = 0
        self.d2h_bytes = 0

    # ---- helpers -----------------------------------------------------------
    def _matching(self) -> np.ndarray:
        """Structural matching columns among the candidates.

        Host-side SciPy Hopcroft-Karp, exactly as the reference computes it
        (psipm_stable_preconditioner.py:224-239, psipm_spectral_preconditioner.py:307-326);
        it runs once per LP.
        """
        graph = self.A.tocsr(copy=True)
        graph.data.fill(1.0)
        matched = csgraph.maximum_bipartite_matching(graph, perm_type="column")
        matched = matched[matched >= 0].astype(np.int64)
        pos = np.searchsorted(self.candidates, matched)
        valid = pos < self.candidates.size
        idx = np.flatnonzero(valid)
        valid[idx] &= self.candidates[pos[idx]] == matched[idx]
        return np.unique(matched[valid])

    def close(self) -> None:
        self.dev.close()

    def observe(self, x, z, w, s, mu) -> None:  # psipm_stable_preconditioner.py:285-291
        self.mu = float(mu)
        normalized = max(float(mu), 0.0) / (1.0 + max(float(mu), 0.0))
        self.current_cg_tol = min(self.cg_tol_max, max(self.cg_tol, float(self.forcing_factor * normalized)))

    def _upload_weights(self, theta, delta) -> None:
        if theta is RESIDENT:
            return
        self.dev.set_theta(theta, delta)
        self.h2d_bytes += 8 * self.n

    def _scores(self, weights=None, delta=None) -> np.ndarray:
        """Leverage scores computed on the device (psipm_stable_preconditioner.py:293-309)."""
        out, _ = self.dev.scores(self.fill_weight, want=True)
        return out

    def _refresh_core(self, weights, delta, stable) -> None:  # psipm_stable_preconditioner.py:311-371
        if self.use_full_preconditioner:
            self.core = self.candidates.copy()
            self.dev.set_core(self.core)
            self.retained_fractions.append(1.0)
            self.refreshes += 1
            self.core_age = 0
            self._initialized = True
            self.core_history.append(self.core.copy())
            return
        self.dev.scores(self.fill_weight, want=False)
        if self.trace_hook is not None:
            self.trace_hook(self)
        learned = self.selector is not None and self._selector_pause == 0
        if learned:
            keep = (int(np.ceil(self.selector_window * min(self.core_target, self.candidates.size)))
                    if self.selector_window > 1.0 else 0)
            self._shift_vote = self.dev.mlp_scores(self.selector.weights_bf16, self.selector.biases, self.mu, keep)
            self.learned_refreshes += 1
        elif self._selector_pause > 0:
            self._selector_pause -= 1
        self._core_learned = learned
        target = min(self.core_target, self.candidates.size)
        mandatory_local = np.searchsorted(self.candidates, self.mandatory)
        core, retained = self.dev.refresh_core(target, self.retention, bool(stable and self.core.size),
                                               mandatory_local)
        self.core = core
        self.retained_fractions.append(retained)
        self.refreshes += 1
        self.core_age = 0
        self._initialized = True
        self.core_history.append(core.copy())
        # selections whose cut fell inside a run of equal scores (index rule decided)
        self.tie_straddles = self.dev.tie_info()["straddles"]

    def _factor_numeric(self, theta, delta) -> None:
        """Assembly + Jacobi scaling + shift ladder on the device (psipm_active_pool.py:839-897)."""
        t0 = time.perf_counter()
        start = 0
        if self._shift > 0.0:
            start = max(0, int(np.searchsorted(SHIFTS, self._shift, side="left")) - 1)
        if self._core_learned and self.selector_shift:  # the network's shift vote
            start = max(start, min(len(SHIFTS) - 1, int(self._shift_vote + 0.5)))
        try:
            used, info = self.dev.factor(float(delta), start)
        except DeviceError as exc:
            self.t_fact += time.perf_counter() - t0
            if exc.status == _lib.ERR_MEMORY and self.core.size > self.mandatory.size:
                # the factor of this core does not fit in device memory: cap the
                # core below its size and refresh at the next factorisation
                cap = max(int(self.mandatory.size), int(0.8 * self.core.size))
                if self._largest_fit < self.core.size:  # never below a core whose factor fitted
                    cap = max(cap, self._largest_fit)
                self.max_core_target = min(self.max_core_target, cap)
                self.core_target = min(self.core_target, cap)
                self._initialized = False
                self._has_factor = False
                self.memory_caps += 1
                raise KKTSolveError(f"the factor does not fit in device memory ({exc})") from exc
            if exc.status == _lib.ERR_NOT_PD:
                self.stats["not_pd"] += 8 - start
                self._has_factor = False
                raise KKTSolveError(f"Cholesky failed even with a 1e-2 shift ({exc})") from exc
            raise KKTSolveError(str(exc)) from exc
        self.stats["not_pd"] += used - start
        self._largest_fit = max(self._largest_fit, int(self.core.size))
        self._shift = SHIFTS[used]
        if used > 0:
            self.n_shifted += 1
        self.n_symbolic = int(info.symbolic_analyses)
        self.nnz_factor = int(info.nnz_factor)
        self.last_factor_info = info
        self.theta = theta
        self.delta = float(delta)
        self._has_factor = True
        self.n_fact += 1
        self.t_fact += time.perf_counter() - t0
        if self.factor_hook is not None:
            self.factor_hook(self, used)

    def factorize(self, theta, delta) -> None:  # psipm_stable_preconditioner.py:397-432
        theta = theta if theta is RESIDENT else np.asarray(theta, dtype=float)
        self.delta_now = float(delta)
        self._weights = None
        self._upload_weights(theta, delta)
        poor = self._last_cg >= self.refresh_cg
        can_grow = self.core_target < self.max_core_target
        refresh = (not self._initialized or self.core_age >= self.core_max_age
                   or (poor and (can_grow or self.m <= self.adaptive_refresh_row_threshold)))
        refactor = not self._has_factor or self.factor_age >= self.factor_max_age or refresh or poor
        if refresh:
            self._refresh_core(None, delta, stable=bool(self.core.size))
        if refactor:
            self._factor_numeric(theta, delta)
            self.factor_age = 0
            self.preconditioner_nnz.append(self.nnz_factor)
        else:
            self.theta = theta
            self.delta = float(delta)
            self.factor_age += 1
        self.core_age += 1
        self.core_sizes.append(int(self.core.size))

    def _apply(self, r):
        """P^{-1} r with the device factor (psipm_active_pool.py:949-956)."""
        return self.dev.apply(r)

    def _full_matvec(self, v):
        """H v on the device (psipm_stable_preconditioner.py:434-438)."""
        return self.dev.matvec(v)


class GpuSpectralStableColumnPreconditioner(GpuStableActiveColumnPreconditioner):
    """Device version of SpectralStableColumnPreconditioner (psipm_spectral_preconditioner.py:143-752)."""

    def __init__(self, A, protected=None, weighted_backbone=False, structural_backbone=True,
                 matching_max_rows=50_000, matching_max_nnz=25_000_000, matching_refresh_max_rows=20_000,
                 backbone_max_age=20, residual_score_weight=0.0, swap_patience=2, condition_limit=1e12,
                 lag_spectral_ratio=1e8, residual_replacement=100, residual_gap_tolerance=0.1,
                 stagnation_window=3, stagnation_reduction=0.8, corrector_tightening=1.0,
                 minres_fallback=True, minres_maxit=400, minres_max_dimension=200_000, **kwargs):
        super().__init__(A, protected=protected, matching_backbone=False, **kwargs)
        if weighted_backbone:
            raise NotImplementedError("weighted_backbone=True (off by default in the reference)")
        if residual_score_weight:
            raise NotImplementedError("residual_score_weight > 0 (0 by default in the reference)")
        self.weighted_backbone = False
        self.structural_backbone = bool(structural_backbone)
        self.backbone_max_age = max(1, int(backbone_max_age))
        self.residual_score_weight = 0.0
        self.swap_patience = max(1, int(swap_patience))
        self.condition_limit = max(1.0, float(condition_limit))
        self.lag_spectral_ratio = max(1.0, float(lag_spectral_ratio))
        self.residual_replacement = max(0, int(residual_replacement))
        self.residual_gap_tolerance = max(math.sqrt(EPS), float(residual_gap_tolerance))
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
        self._reference_theta = None
        self._reference_delta = None
        self._factor_generation = 0
        self.resident = False  # set by the device-resident IPM: lag bound from device weights
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

    def set_ipm_context(self, res_d, res_p, res_n, tol) -> None:  # :230-250
        self.set_ipm_context_norms(float(np.linalg.norm(res_d)), float(np.linalg.norm(res_p)), res_n, tol)

    def set_ipm_context_norms(self, norm_d, norm_p, res_n, tol) -> None:
        """``set_ipm_context`` given the 2-norms of res_d and res_p."""
        current = max(float(res_n), float(norm_d), float(norm_p), TINY)
        previous = self._nonlinear_residual
        self._previous_nonlinear_residual = previous
        self._nonlinear_residual = current
        if previous is None or not np.isfinite(previous):
            estimate = self.cg_tol_max
        else:
            estimate = 0.9 * (current / max(previous, TINY)) ** 1.5
        self._ew_tolerance = min(self.cg_tol_max, max(self.cg_tol, float(tol) * 0.1, estimate))
        self._rhs_index = 0

    def observe(self, x, z, w, s, mu) -> None:  # :252-258
        self.mu = float(mu)
        normalized = max(float(mu), 0.0) / (1.0 + max(float(mu), 0.0))
        mu_tol = self.forcing_factor * normalized
        self.current_cg_tol = min(self.cg_tol_max, max(self.cg_tol, min(mu_tol, self._ew_tolerance)))

    def _linear_tolerance(self) -> float:  # :260-265
        tol = self.current_cg_tol
        if self._rhs_index:
            tol = max(self.cg_tol, self.corrector_tightening * tol)
        self._rhs_index += 1
        return float(tol)

    def _update_backbone(self) -> None:  # :328-365 (structural backbone)
        if self.matching_columns.size:
            return
        if not self.structural_backbone or self.use_full_preconditioner or not self.m:
            return
        matching = self._matching()
        if matching.size:
            self.matching_columns = matching
            self.mandatory = np.union1d(self.protected_mandatory, matching)
            self.core_target = min(self.candidates.size, max(self.core_target, self.mandatory.size))
            self.max_core_target = min(self.candidates.size, max(self.max_core_target, self.mandatory.size))
            self.weighted_backbone_refreshes += 1

    def _refresh_core(self, weights, delta, stable, force_backbone=False) -> None:  # :388-394
        old = self.core.copy()
        self._update_backbone()
        super()._refresh_core(weights, delta, stable)
        if old.size and self.core.size:
            changed = old.size - np.intersect1d(old, self.core, assume_unique=True).size
            self.core_swaps += max(0, int(changed))

    def _lag_bound(self, theta, delta) -> float:  # :396-410
        if self._reference_theta is None:
            return np.inf
        if theta is RESIDENT or self.resident:
            # max/min of w / max(w_ref, tiny) on the device (psipm_lag_ratio)
            hi, lo = self.dev.lag_ratio()
            if not np.isfinite(hi) or self.n == 0:
                return np.inf
            bound = max(hi, 1.0 / lo)
        else:
            weights = 1.0 / theta
            ref = 1.0 / self._reference_theta
            ratio = weights / np.maximum(ref, TINY)
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

    def _factor_current(self, theta, delta) -> None:  # :412-418
        self._factor_numeric(theta, delta)
        if self.resident:
            self.dev.lag_reference()
        self.factor_age = 0
        self._reference_theta = theta
        self._reference_delta = float(delta)
        self._factor_generation += 1
        self.preconditioner_nnz.append(self.nnz_factor)

    def factorize(self, theta, delta) -> None:  # :420-467
        theta = theta if theta is RESIDENT else np.asarray(theta, dtype=float)
        self.delta_now = float(delta)
        self._upload_weights(theta, delta)
        spectral_poor = (self._last_condition >= self.condition_limit
                         and self._last_cg >= max(10, int(0.8 * self.refresh_cg)))
        poor = self._last_cg >= self.refresh_cg or spectral_poor or self._last_stagnated
        self._poor_streak = self._poor_streak + 1 if poor else 0
        can_grow = self.core_target < self.max_core_target
        swap_due = poor and not can_grow and self._poor_streak >= self.swap_patience
        refresh = not self._initialized or self.core_age >= self.core_max_age or (poor and can_grow) or swap_due
        # learned selector fallback: a learned core that the rule's signals call
        # poor is replaced now by the plain rule, which also keeps the next refreshes
        if poor and self._core_learned:
            self.selector_fallbacks += 1
            self._selector_pause = self.selector_patience
            refresh = True
        if refresh:
            self._refresh_core(None, delta, stable=bool(self.core.size), force_backbone=swap_due)
            self._poor_streak = 0
        lag = self._lag_bound(theta, float(delta))
        self.lag_spectral_bounds.append(lag)
        refactor = (not self._has_factor or self.factor_age >= self.factor_max_age or refresh or poor
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

    def _pcg(self, r1, r2, tolerance):
        dx, res = self.dev.solve(r1, r2, tolerance, self.cg_maxit, _lib.PCG_SPECTRAL,
                                 self.residual_replacement, self.residual_gap_tolerance)
        self.h2d_bytes += 8 * (self.n + self.m)
        self.d2h_bytes += 8 * (self.n + self.m)
        return dx, self._krylov(res)

    def _pcg_resident(self, corrector, tolerance):
        finite, res = self.dev.ipm_newton(corrector, tolerance, self.cg_maxit, _lib.PCG_SPECTRAL,
                                          self.residual_replacement, self.residual_gap_tolerance)
        return finite, self._krylov(res)

    def _krylov(self, res) -> "KrylovResult":
        lo, hi, cond = ritz_estimate(res.alphas, res.betas)
        w = self.stagnation_window
        hist = res.history
        stagnated = len(hist) >= w and hist[-1] > self.stagnation_reduction * hist[-w]
        self.device_seconds += res.seconds
        self.pcg_launches += 1
        self.pcg_total_iterations += res.iterations
        self.pcg_matvecs += res.matvecs
        self.pcg_replacements += res.replacements
        self.pcg_phase_seconds += np.asarray(res.phase_seconds)
        bv = 4 if self.precision != _lib.FP64 else 8
        self.pcg_bytes += pcg_launch_bytes(self.m, self.n, self.A.nnz, self.nnz_factor, res.iterations,
                                           res.matvecs, res.iterations + 2 + res.replacements, bv)
        self.refinement_sweeps += res.refinements
        return KrylovResult(res.x, res.info, res.iterations, res.relative_residual, float(cond),
                            float(max(abs(lo - 1.0), abs(hi - 1.0))), None, res.replacements,
                            res.residual_checks, bool(stagnated), res.seconds)

    def _record_krylov(self, res: KrylovResult) -> None:  # :639-649
        self._last_cg = int(res.iterations)
        self._last_condition = float(res.condition_estimate)
        self._last_spectral_error = float(res.spectral_error_estimate)
        self._last_stagnated = bool(res.stagnated)
        self.condition_estimates.append(self._last_condition)
        self.spectral_error_estimates.append(self._last_spectral_error)
        self.residual_replacements += int(res.replacements)
        self.residual_checks += int(res.residual_checks)
        self.stagnation_events += int(res.stagnated)

    def solve(self, r1, r2):  # :651-752
        def fallback(tol):  # augmented MINRES (:583-637) on the device
            dx, dy, accepted, its, rel = self.dev.minres(r1, r2, tol, self.minres_maxit, self.fail_tol)
            self.h2d_bytes += 8 * (self.n + self.m)
            self.d2h_bytes += 8 * (self.n + self.m)
            return (dx, dy), accepted, its, rel

        return self._solve_policy(lambda tol: self._pcg(r1, r2, tol), lambda dx, res: (dx, res.solution),
                                  fallback if self._minres_available() else None)

    def _minres_available(self) -> bool:
        return self.precision == _lib.FP64 and hasattr(self.dev, "minres")

    def solve_resident(self, corrector: bool) -> bool:
        """``solve`` on the device-resident Newton system (psipm_ipm_newton).

        ``corrector=False`` solves for D from (rd, rp, rmz, rmw), ``True`` for
        C from (0, 0, rmz, rmw); the directions stay on the device.  Same
        policy, statistics and ``KKTSolveError`` as :meth:`solve`; returns
        whether every entry of the directions is finite.
        """
        def fallback(tol):
            finite, accepted, its, rel = self.dev.ipm_minres(corrector, tol, self.minres_maxit, self.fail_tol)
            return finite, accepted, its, rel

        return self._solve_policy(lambda tol: self._pcg_resident(corrector, tol), lambda finite, res: finite,
                                  fallback if self._minres_available() else None)

    def solve_start(self, which: int) -> bool:
        """``solve(zeros, b)`` (which 0) or ``solve(zeros, A c)`` (which 1) of
        the starting point (psipm_active_pool.py:4182-4187) on the device: same
        policy, statistics and ``KKTSolveError`` as :meth:`solve`; the result
        goes straight into the device iterate (x = A^T dy, or y = dy).
        Returns whether it is finite."""
        return self._solve_policy(lambda tol: self._pcg_start(which, tol), lambda finite, res: finite, None)

    def _pcg_start(self, which, tolerance):
        finite, res = self.dev.ipm_start_solve(which, tolerance, self.cg_maxit, _lib.PCG_SPECTRAL,
                                               self.residual_replacement, self.residual_gap_tolerance)
        return finite, self._krylov(res)

    def _solve_policy(self, run, finish, fallback=None):
        started = time.perf_counter()
        fb = self.t_fact
        if not self._has_factor:
            raise KKTSolveError("solve before a successful factorize")
        tol = self._linear_tolerance()
        try:
            dx, res = run(tol)
        except DeviceError as exc:
            self.cg_failures += 1
            raise KKTSolveError(str(exc)) from exc
        total = res.iterations
        failed = res.info != 0 or not np.isfinite(res.relative_residual) or res.relative_residual > tol
        can_grow = self.core_target < self.max_core_target
        warranted = can_grow or res.info < 0 or res.stagnated
        if failed and warranted and self.candidates.size and not self.use_full_preconditioner:
            self.pcg_retries += 1
            if self.core_target < self.max_core_target:
                grown = max(self.core_target + 1, int(np.ceil(self.retry_growth * self.core_target)))
                self.core_target = min(self.max_core_target, grown)
            self._refresh_core(None, self.delta, stable=True, force_backbone=res.info < 0 or res.stagnated)
            self._factor_current(self.theta, self.delta)
            self.core_sizes.append(int(self.core.size))
            try:
                dx, res = run(tol)
            except DeviceError as exc:
                self.cg_failures += 1
                raise KKTSolveError(str(exc)) from exc
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
        if failed:
            if (fallback is not None and self.minres_fallback and self.n + self.m <= self.minres_max_dimension
                    and (res.info < 0 or res.stagnated)):  # :717-737
                self.cg_failures += 1
                self.minres_fallbacks += 1
                try:
                    result, accepted, its, rel = fallback(tol)
                except DeviceError as exc:
                    self.t_solve += max(0.0, time.perf_counter() - started - (self.t_fact - fb))
                    raise KKTSolveError(str(exc)) from exc
                self.minres_iterations += its
                self.full_fallbacks += 1
                if not accepted:
                    self.t_solve += max(0.0, time.perf_counter() - started - (self.t_fact - fb))
                    raise KKTSolveError("spectral PCG and augmented MINRES failed: "
                                        f"pcg info={res.info}, pcg residual={res.relative_residual:.2e}, "
                                        f"minres residual={rel:.2e}")
                self.n_solve += 1
                self.t_solve += max(0.0, time.perf_counter() - started - (self.t_fact - fb))
                return result
            self.cg_failures += 1
            self.t_solve += max(0.0, time.perf_counter() - started - (self.t_fact - fb))
            raise KKTSolveError(f"spectral stable-column PCG failed: info={res.info}, "
                                f"residual={res.relative_residual:.2e}")
        self.n_solve += 1
        self.t_solve += max(0.0, time.perf_counter() - started - (self.t_fact - fb))
        return finish(dx, res)


# ---------------------------------------------------------------------------
# V3.1 HSD surface
class GpuStableColumnPreconditioner:
    """HSD preconditioner protocol (psipm_v3_1_hsd.py:823-989) on the device.

    ``factor(weights, delta)`` maps ``theta = 1/max(weights, TINY)`` into the
    stable-rule policy (:902-921); ``solve(rhs)`` applies ``P^{-1}``;
    ``record_iterations`` grows the core from measured PCG/factor time
    (:954-984).  ``impl`` exposes the device object, whose ``dev`` handle
    :func:`pcg_rows` uses to run the whole HSD PCG on the device.
    """

    def __init__(self, A, options=None, stats=None, device=0, precision=_lib.FP64, **overrides):
        o = dict(core_factor=1.0, max_core_factor=3.0, retention=0.9, factor_max_age=2, core_max_age=12,
                 fill_weight=0.2, pcg_tolerance_late=1e-10, pcg_tolerance_early=1e-8,
                 pcg_max_iterations=1000, retry_growth=1.6, refresh_cg=60, growth_amortization=1.0)
        if options is not None:
            for key in list(o):
                for name in (f"generic_{key}", key):
                    if hasattr(options, name):
                        o[key] = getattr(options, name)
        o.update(overrides)
        self.options = o
        self.stats = stats
        self.impl = GpuStableActiveColumnPreconditioner(
            A, core_factor=o["core_factor"], max_core_factor=o["max_core_factor"], retention=o["retention"],
            factor_max_age=o["factor_max_age"], core_max_age=o["core_max_age"],
            refresh_cg=int(o["pcg_max_iterations"]) + 1, fill_weight=o["fill_weight"],
            cg_tol=o["pcg_tolerance_late"], cg_tol_max=o["pcg_tolerance_early"],
            cg_maxit=int(o["pcg_max_iterations"]), retry_growth=o["retry_growth"], refine=0,
            device=device, precision=precision)
        self._retry_growth = float(o["retry_growth"])
        self._growth_trigger = int(o["refresh_cg"])
        self._growth_amortization = float(o["growth_amortization"])
        self._last_numeric_factor_seconds = 0.0
        self._factor_epoch = 0
        self._last_growth_epoch = -1
        self.growth_events = 0

    @property
    def backend(self) -> str:
        return "stable-active-column-b200"

    def close(self) -> None:
        """Release the device handle (the reference's object has nothing to release)."""
        self.impl.close()

    def factor(self, weights, delta) -> float:  # :902-921
        started = time.perf_counter()
        before = int(self.impl.n_fact)
        theta = 1.0 / np.maximum(np.asarray(weights, dtype=float), TINY)
        self.impl.factorize(theta, float(delta))
        elapsed = time.perf_counter() - started
        self._factor_epoch += 1
        if self.impl.n_fact > before:
            self._last_numeric_factor_seconds = elapsed
        return elapsed

    def solve(self, rhs):  # :923-926
        return self.impl._apply(np.asarray(rhs, dtype=float))

    def record_iterations(self, iterations, elapsed=0.0, converged=True) -> None:  # :954-984
        impl = self.impl
        impl._last_cg = int(iterations)
        can_grow = impl.core_target < impl.max_core_target
        projected = 4.0 * max(float(elapsed), 0.0)
        affordable = (self._last_numeric_factor_seconds <= 0.0
                      or projected >= self._growth_amortization * self._last_numeric_factor_seconds)
        if iterations >= self._growth_trigger and affordable and self._last_growth_epoch != self._factor_epoch:
            if can_grow:
                grown = max(impl.core_target + 1, int(math.ceil(self._retry_growth * impl.core_target)))
                impl.core_target = min(impl.max_core_target, grown)
                self.growth_events += 1
            impl.core_age = impl.core_max_age
            self._last_growth_epoch = self._factor_epoch

    def record_solve(self, iterations, elapsed, converged) -> None:
        self.record_iterations(iterations, elapsed, converged)

    def solve_normal(self, r1, r2, rtol, max_iterations, deadline=np.inf):
        """``dy = H^{-1} (r2 - A D r1)`` by the HSD PCG (psipm_v3_1_hsd.py:1015-1063)
        and ``dx = D (r1 + A' dy)``, both on the device; ``D`` are the weights of
        the last :meth:`factor` call (``1/theta`` with ``theta = 1/max(D, TINY)``).

        One ``psipm_solve`` call: the right-hand side's SpMV, the PCG and the
        back-substitution run on the device; r1, r2 go in and dx, dy come out.
        Returns ``(dx, dy, iterations, matvecs, okay, elapsed)``; the deadline
        bounds the launch as in :func:`pcg_rows`.
        """
        started = time.perf_counter()
        dev = self.impl.dev
        dx, res = _under_deadline(dev, deadline, lambda: dev.solve(r1, r2, rtol, int(max_iterations), _lib.PCG_HSD))
        return dx, res.x, res.iterations, res.matvecs, bool(res.ok), time.perf_counter() - started


def pcg_rows(preconditioner: GpuStableColumnPreconditioner, rhs, rtol, max_iterations, deadline=np.inf):
    """Device replacement of the HSD ``_pcg`` (psipm_v3_1_hsd.py:1015-1063).

    Returns ``(x, iterations, matvecs, okay, elapsed)`` like the reference.
    The operator is ``A diag(D) A' + delta I`` with the weights of the last
    ``factor`` call, which is what ``HSDNewtonSystem.matvec`` applies
    (psipm_v3_1_hsd.py:1136-1137).
    """
    started = time.perf_counter()
    dev = preconditioner.impl.dev
    res = _under_deadline(dev, deadline, lambda: dev.pcg(rhs, rtol, int(max_iterations), _lib.PCG_HSD))
    return res.x, res.iterations, res.matvecs, bool(res.ok), time.perf_counter() - started


def _under_deadline(dev, deadline, call):
    """Run one device PCG call under the caller's ``time.perf_counter`` deadline.

    The reference tests the deadline after each iteration's convergence test
    and then returns the current x as not converged (psipm_v3_1_hsd.py:1054-1055);
    the device PCG does the same against a wall-clock budget
    (``psipm_set_pcg_budget``), set here to the time left (at least 1 ns, so a
    call that starts past its deadline stops after one iteration) and cleared
    afterwards.
    """
    if not np.isfinite(deadline):
        return call()
    dev.set_pcg_budget(max(deadline - time.perf_counter(), 1e-9))
    try:
        return call()
    finally:
        dev.set_pcg_budget(0.0)
