"""Oracle restatement of the V3.1 HSD linear algebra — test infrastructure.

* :func:`pcg` — the HSD preconditioned CG with true-residual replacement
  every 10 iterations (psipm_v3_1_hsd.py:1015-1063).
* :class:`StableColumnPreconditionerOracle` — the V3.1 wrapper around the
  stable active-column preconditioner (psipm_v3_1_hsd.py:823-989).
"""

from __future__ import annotations

import math
import time

import numpy as np

from .stable import StableOracle

TINY = float(np.finfo(np.float64).tiny)
EPS = float(np.finfo(np.float64).eps)


def pcg(matvec, rhs, preconditioner, rtol, max_iterations, deadline=np.inf):
    """psipm_v3_1_hsd.py:1015-1063; returns (x, iterations, matvecs, ok, elapsed)."""
    started = time.perf_counter()
    rhs_norm = float(np.linalg.norm(rhs))
    if rhs_norm == 0.0:
        return np.zeros_like(rhs), 0, 0, True, time.perf_counter() - started
    x = preconditioner.solve(rhs)
    r = rhs - matvec(x)
    matvecs = 1
    target = max(rtol * rhs_norm, 64.0 * EPS * rhs_norm)
    if float(np.linalg.norm(r)) <= target:
        return x, 0, matvecs, True, time.perf_counter() - started
    z = preconditioner.solve(r)
    p = z.copy()
    rz = float(r @ z)
    if not np.isfinite(rz) or rz <= 0.0:
        return x, 0, matvecs, False, time.perf_counter() - started
    for it in range(1, max_iterations + 1):
        q = matvec(p)
        matvecs += 1
        curv = float(p @ q)
        if not np.isfinite(curv) or curv <= 0.0:
            return x, it, matvecs, False, time.perf_counter() - started
        step = rz / curv
        x += step * p
        r -= step * q
        if it % 10 == 0:
            r = rhs - matvec(x)
            matvecs += 1
        if float(np.linalg.norm(r)) <= target:
            return x, it, matvecs, True, time.perf_counter() - started
        if time.perf_counter() >= deadline:
            return x, it, matvecs, False, time.perf_counter() - started
        z = preconditioner.solve(r)
        rz_new = float(r @ z)
        if not np.isfinite(rz_new) or rz_new <= 0.0:
            return x, it, matvecs, False, time.perf_counter() - started
        p *= rz_new / rz
        p += z
        rz = rz_new
    return x, max_iterations, matvecs, False, time.perf_counter() - started


class StableColumnPreconditionerOracle:
    """psipm_v3_1_hsd.py:823-989 with the stable preconditioner required."""

    def __init__(self, A, core_factor=1.0, max_core_factor=3.0, retention=0.9, factor_max_age=2,
                 core_max_age=12, fill_weight=0.2, pcg_tolerance_late=1e-10, pcg_tolerance_early=1e-8,
                 pcg_max_iterations=1000, retry_growth=1.6, refresh_cg=60, growth_amortization=1.0):
        self.impl = StableOracle(
            A, core_factor=core_factor, max_core_factor=max_core_factor, retention=retention,
            factor_max_age=factor_max_age, core_max_age=core_max_age,
            refresh_cg=pcg_max_iterations + 1, fill_weight=fill_weight, cg_tol=pcg_tolerance_late,
            cg_tol_max=pcg_tolerance_early, cg_maxit=pcg_max_iterations, retry_growth=retry_growth,
            refine=0)
        self._retry_growth = retry_growth
        self._growth_trigger = refresh_cg
        self._growth_amortization = growth_amortization
        self._last_numeric_factor_seconds = 0.0
        self._factor_epoch = 0
        self._last_growth_epoch = -1
        self.growth_events = 0

    def factor(self, weights, delta):  # :902-921
        started = time.perf_counter()
        before = int(self.impl.n_fact)
        theta = 1.0 / np.maximum(weights, TINY)
        self.impl.factorize(theta, float(delta))
        elapsed = time.perf_counter() - started
        self._factor_epoch += 1
        if self.impl.n_fact > before:
            self._last_numeric_factor_seconds = elapsed
        return elapsed

    def solve(self, rhs):  # :923-926
        return np.asarray(self.impl._apply(rhs)).ravel()

    def record_iterations(self, iterations, elapsed=0.0, converged=True):  # :954-984
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
