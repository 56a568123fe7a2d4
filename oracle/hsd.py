"""Oracle restatement of the V3.1 HSD linear algebra — test infrastructure.

* :func:`pcg` — the HSD preconditioned CG with true-residual replacement
  every 10 iterations (psipm_v3_1_hsd.py:1015-1063).
* :class:`StableColumnPreconditionerOracle` — the V3.1 wrapper around the
  stable active-column preconditioner (psipm_v3_1_hsd.py:823-989).
* :class:`HSDNewtonSystemOracle` — the reduced HSD Newton system
  (psipm_v3_1_hsd.py:1066-1264): border data, three normal-equations solves,
  the 2 x 2 border solve and the back-substitution.

Pinned bit-exact to the reference on the fixtures hsd_m1600 and
hsd_newton_m1600 (tests/test_hsd_oracle.py).
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


class HSDNewtonSystemOracle:
    """The reduced HSD Newton system of one active-column set
    (psipm_v3_1_hsd.py:1066-1264), restated.

    ``state`` supplies x, z, w, tau, kappa; ``embedding`` bar_b, bar_c, bar_g;
    ``options`` zeta and pcg_max_iterations; ``stats`` the LinearStats counters
    (iterations, max_iterations, solves, matvecs, failures, seconds,
    preconditioner_seconds).  The construction factors the preconditioner
    (:1098) and forms the border data (:1099-1131); ``direction`` solves
    ``f``, and on its first call also ``h`` and ``theta_row`` (:1160-1264).
    """

    def __init__(self, A, c, upper, b, D, delta, eta, state, embedding, preconditioner, pcg_tolerance,
                 options, deadline, stats):
        self.A, self.c, self.upper, self.b, self.D = A, c, upper, b, D
        self.delta, self.eta, self.state, self.embedding = delta, eta, state, embedding
        self.preconditioner, self.pcg_tolerance = preconditioner, pcg_tolerance
        self.options, self.deadline, self.stats = options, deadline, stats
        stats.preconditioner_seconds += preconditioner.factor(D, delta)
        boxed = np.isfinite(upper)
        self.boxed = boxed
        slack = np.ones_like(c)
        slack[boxed] = upper[boxed] * state.tau - state.x[boxed]
        ratio = np.zeros_like(c)
        ratio[boxed] = state.w[boxed] / slack[boxed]
        self.slack, self.upper_ratio = slack, ratio
        u0 = np.where(boxed, upper, 0.0)
        self.c_direction = c - ratio * u0
        self.c_gap = c + ratio * u0
        bar_b, bar_c = embedding.bar_b, embedding.bar_c
        self.h = b + A @ (D * self.c_direction)
        self.g = b - A @ (D * self.c_gap)
        Dc = A @ (D * bar_c)
        self.theta_row = bar_b + Dc
        self.normal_row = Dc - bar_b
        curvature = float(np.sum(ratio[boxed] * upper[boxed] * upper[boxed]))
        self.alpha = float(self.c_gap @ (D * self.c_direction)) + curvature + state.kappa / state.tau + eta
        self.beta = embedding.bar_g - float(self.c_gap @ (D * bar_c))
        self.gamma = -float(bar_c @ (D * self.c_direction)) - embedding.bar_g
        self.lambda_theta = float(bar_c @ (D * bar_c)) + options.zeta
        self._h_solution = None
        self._theta_solution = None

    def matvec(self, v):  # :1136-1137
        return self.A @ (self.D * (self.A.T @ v)) + self.delta * v

    def solve_rows(self, rhs):  # :1139-1159
        x, it, mv, ok, elapsed = pcg(self.matvec, rhs, self.preconditioner, self.pcg_tolerance,
                                     self.options.pcg_max_iterations, self.deadline)
        st = self.stats
        st.solves += 1
        st.iterations += it
        st.max_iterations = max(st.max_iterations, it)
        st.matvecs += mv
        st.seconds += elapsed
        if hasattr(self.preconditioner, "record_solve"):
            self.preconditioner.record_solve(it, elapsed, ok)
        else:
            self.preconditioner.record_iterations(it)
        if not ok:
            st.failures += 1
        return x, ok

    def direction(self, rhs_d, rhs_p, rhs_g, rhs_n, rhs_c, rhs_upper, rhs_t):  # :1160-1264
        st, boxed, D = self.state, self.boxed, self.D
        up = np.zeros_like(rhs_d)
        up[boxed] = rhs_upper[boxed] / self.slack[boxed]
        q = rhs_d + rhs_c / st.x - up
        u, ok_u = self.solve_rows(-rhs_p - self.A @ (D * q))
        ok_h = ok_t = True
        if self._h_solution is None:
            self._h_solution, ok_h = self.solve_rows(self.h)
        if self._theta_solution is None:
            self._theta_solution, ok_t = self.solve_rows(self.theta_row)
        hs, ts = self._h_solution, self._theta_solution
        bar_c = self.embedding.bar_c
        gap_rhs = (rhs_g + float(self.c_gap @ (D * q))
                   + float(self.upper[boxed] @ (rhs_upper[boxed] / self.slack[boxed]))
                   + rhs_t / st.tau - float(self.g @ u))
        normal_rhs = rhs_n - float(bar_c @ (D * q)) - float(self.normal_row @ u)
        M = np.array([[self.alpha + float(self.g @ hs), self.beta - float(self.g @ ts)],
                      [self.gamma + float(self.normal_row @ hs), self.lambda_theta - float(self.normal_row @ ts)]],
                     dtype=np.float64)
        v = np.array([gap_rhs, normal_rhs], dtype=np.float64)
        det = float(np.linalg.det(M))
        scale = max(float(np.linalg.norm(M, ord=np.inf)), 1.0)
        if not np.all(np.isfinite(M)) or not np.all(np.isfinite(v)) or abs(det) <= 64.0 * EPS * scale * scale:
            ok_u = False
            M = M + 64.0 * EPS * scale * np.eye(2)
        try:
            dtau, dtheta = np.linalg.solve(M, v)
        except np.linalg.LinAlgError:
            dtau, dtheta = np.linalg.lstsq(M, v, rcond=None)[0]
            ok_u = False
        dy = u + hs * dtau - ts * dtheta
        dx = D * (q + self.A.T @ dy - self.c_direction * dtau + bar_c * dtheta)
        dz = (rhs_c - st.z * dx) / st.x
        dw = np.zeros_like(dx)
        ds = np.zeros_like(dx)
        ds[boxed] = self.upper[boxed] * dtau - dx[boxed]
        dw[boxed] = (rhs_upper[boxed] - st.w[boxed] * ds[boxed]) / self.slack[boxed]
        dkappa = (rhs_t - st.kappa * dtau) / st.tau
        finite = all(np.all(np.isfinite(a)) for a in (dx, dy, dz, dw, np.asarray([dtau, dtheta, dkappa])))
        return dx, dy, dz, dw, float(dtau), float(dtheta), float(dkappa), bool(ok_u and ok_h and ok_t and finite)


def pricing_round(A, c, y, tau, active, pricing_tolerance, pricing_batch):
    """The pricing step of the V3.1 HSD loop (psipm_v3_1_hsd.py:2101-2103,
    2148-2156): violation over all columns and the candidate columns, ties at
    the batch cut taken by ascending index (the reference's argpartition
    leaves that choice to NumPy's build)."""
    import numpy as np

    tau_scale = max(tau, 1.0e-12)
    violation = A.T.tocsr() @ y - c * tau
    candidate = np.flatnonzero(~np.asarray(active, dtype=bool) & (violation > pricing_tolerance * tau_scale))
    if candidate.size > pricing_batch:
        order = np.lexsort((candidate, -violation[candidate]))
        candidate = np.sort(candidate[order[:pricing_batch]])
    return violation, candidate
