"""Reduced HSD Newton system on the device (psipm_v3_1_hsd.py:1066-1264).

:class:`HSDNewtonSystem` takes the reference's constructor arguments and
returns the reference's ``direction`` tuple, so the V3.1 step loop
(psipm_v3_1_hsd.py:1652-1934) can construct it in place of its own class
when the active set's preconditioner is a
:class:`psipm_b200.kkt.GpuStableColumnPreconditioner`.

The reference eliminates ``dx`` and the two HSD scalars ``dtau``, ``dtheta``
to three normal-equations solves ``H u = f``, ``H h' = h``, ``H t' = theta_row``
(``H = A D A' + delta I``) followed by a 2 x 2 border system.  Each of those
right-hand sides is ``r2 - A D r1`` for an (r1, r2) pair,

* ``f         = -rhs_p - A D q``      (r1 = q,      r2 = -rhs_p)
* ``h         = b + A D c_direction``   (r1 = -c_dir, r2 = b)
* ``theta_row = bar_b + A D bar_c``     (r1 = -bar_c, r2 = bar_b)

which is exactly what one device Newton solve (``psipm_solve``) forms before
its PCG; it also returns ``D (r1 + A' dy)``.  So ``dx`` of the reference,
``D (q + A' dy - c_dir dtau + bar_c dtheta)`` with ``dy = u + h' dtau - t' dtheta``,
is the same combination of the three returned ``dx`` parts, and no
O(nnz) product of ``direction`` runs on the host.  The border vectors ``g``
and ``normal_row`` (two SpMVs per system) and the O(n) scalar work stay on
the host, as in the reference.  ``h'`` and ``t'`` are solved once per system
and reused by later directions (:1169-1176).

Results equal the reference's to the PCG tolerance; the device forms
``A (r1 / theta)`` where the reference forms ``A (D r1)``, and sums in another
order, so they are not bit-identical.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

EPS = float(np.finfo(np.float64).eps)


@dataclass
class LinearStats:
    """Counters the Newton system updates (psipm_v3_1_hsd.py:243-251)."""

    iterations: int = 0
    max_iterations: int = 0
    solves: int = 0
    matvecs: int = 0
    failures: int = 0
    seconds: float = 0.0
    preconditioner_seconds: float = 0.0


class HSDNewtonSystem:
    """Implicit reduced HSD Newton system for one active-column set.

    Arguments as the reference (psipm_v3_1_hsd.py:1069-1085): ``A`` the active
    columns (CSC), ``c``, ``upper`` (``inf`` where unbounded), ``b``, the weights
    ``D``, ``delta``, ``eta``; ``state`` with ``x, z, w, tau, kappa``;
    ``embedding`` with ``bar_b, bar_c, bar_g``; ``preconditioner`` a
    ``GpuStableColumnPreconditioner`` over the same ``A`` (anything with
    ``factor``, ``solve_normal`` and ``record_solve``); ``pcg_tolerance``;
    ``options`` with ``zeta`` and ``pcg_max_iterations``; ``deadline``
    (``time.perf_counter`` seconds); ``stats`` a :class:`LinearStats`.
    """

    def __init__(self, A, c, upper, b, D, delta, eta, state, embedding, preconditioner, pcg_tolerance, options,
                 deadline, stats):
        if preconditioner.impl.A.shape != A.shape:
            raise ValueError("the preconditioner was built for another active-column set")
        self.A, self.c, self.upper, self.b = A, c, upper, b
        self.D = np.asarray(D, dtype=np.float64)
        self.delta, self.eta = float(delta), float(eta)
        self.state, self.embedding = state, embedding
        self.preconditioner = preconditioner
        self.pcg_tolerance = float(pcg_tolerance)
        self.options, self.deadline, self.stats = options, deadline, stats
        stats.preconditioner_seconds += preconditioner.factor(self.D, self.delta)
        D = self.D
        boxed = np.isfinite(upper)
        self.boxed = boxed
        slack = np.ones_like(c)
        slack[boxed] = upper[boxed] * state.tau - state.x[boxed]
        ratio = np.zeros_like(c)
        ratio[boxed] = state.w[boxed] / slack[boxed]
        self.slack, self.upper_ratio = slack, ratio
        upper0 = np.where(boxed, upper, 0.0)
        self.c_direction = c - ratio * upper0
        self.c_gap = c + ratio * upper0
        bar_b, bar_c = embedding.bar_b, embedding.bar_c
        self.g = b - A @ (D * self.c_gap)
        self.normal_row = A @ (D * bar_c) - bar_b
        self.alpha = (float(self.c_gap @ (D * self.c_direction)) + float(np.sum(ratio[boxed] * upper[boxed] ** 2))
                      + state.kappa / state.tau + self.eta)
        self.beta = embedding.bar_g - float(self.c_gap @ (D * bar_c))
        self.gamma = -float(bar_c @ (D * self.c_direction)) - embedding.bar_g
        self.lambda_theta = float(bar_c @ (D * bar_c)) + options.zeta
        self._h = None  # (dx part, dy) of H h' = h
        self._t = None  # (dx part, dy) of H t' = theta_row

    def _solve(self, r1, r2):
        """One device Newton solve, with the reference's bookkeeping (:1139-1159)."""
        dx, dy, it, mv, ok, elapsed = self.preconditioner.solve_normal(
            r1, r2, self.pcg_tolerance, self.options.pcg_max_iterations, self.deadline)
        st = self.stats
        st.solves += 1
        st.iterations += it
        st.max_iterations = max(st.max_iterations, it)
        st.matvecs += mv
        st.seconds += elapsed
        self.preconditioner.record_solve(it, elapsed, ok)
        if not ok:
            st.failures += 1
        return dx, dy, ok

    def direction(self, rhs_d, rhs_p, rhs_g, rhs_n, rhs_c, rhs_upper, rhs_t):
        """``(dx, dy, dz, dw, dtau, dtheta, dkappa, okay)`` (psipm_v3_1_hsd.py:1160-1264)."""
        st, boxed, D = self.state, self.boxed, self.D
        upper_rhs = np.zeros_like(rhs_d)
        upper_rhs[boxed] = rhs_upper[boxed] / self.slack[boxed]
        q = rhs_d + rhs_c / st.x - upper_rhs
        dx_u, u, ok_u = self._solve(q, -np.asarray(rhs_p, dtype=np.float64))
        ok_h = ok_t = True
        if self._h is None:
            dx_h, hs, ok_h = self._solve(-self.c_direction, self.b)
            self._h = (dx_h, hs)
        if self._t is None:
            dx_t, ts, ok_t = self._solve(-self.embedding.bar_c, self.embedding.bar_b)
            self._t = (dx_t, ts)
        (dx_h, hs), (dx_t, ts) = self._h, self._t
        Dq = D * q
        gap_rhs = (rhs_g + float(self.c_gap @ Dq) + float(self.upper[boxed] @ upper_rhs[boxed])
                   + rhs_t / st.tau - float(self.g @ u))
        normal_rhs = rhs_n - float(self.embedding.bar_c @ Dq) - float(self.normal_row @ u)
        border = np.array([[self.alpha + float(self.g @ hs), self.beta - float(self.g @ ts)],
                           [self.gamma + float(self.normal_row @ hs), self.lambda_theta - float(self.normal_row @ ts)]])
        border_rhs = np.array([gap_rhs, normal_rhs])
        scale = max(float(np.linalg.norm(border, ord=np.inf)), 1.0)
        det = float(np.linalg.det(border))
        if not (np.isfinite(border).all() and np.isfinite(border_rhs).all()) or abs(det) <= 64.0 * EPS * scale ** 2:
            ok_u = False  # near-singular border: shift it (:1215-1221)
            border = border + 64.0 * EPS * scale * np.eye(2)
        try:
            dtau, dtheta = np.linalg.solve(border, border_rhs)
        except np.linalg.LinAlgError:
            dtau, dtheta = np.linalg.lstsq(border, border_rhs, rcond=None)[0]
            ok_u = False
        dy = u + hs * dtau - ts * dtheta
        dx = dx_u + dx_h * dtau - dx_t * dtheta
        dz = (rhs_c - st.z * dx) / st.x
        ds = np.zeros_like(dx)
        ds[boxed] = self.upper[boxed] * dtau - dx[boxed]
        dw = np.zeros_like(dx)
        dw[boxed] = (rhs_upper[boxed] - st.w[boxed] * ds[boxed]) / self.slack[boxed]
        dkappa = (rhs_t - st.kappa * dtau) / st.tau
        finite = bool(np.isfinite(dx).all() and np.isfinite(dy).all() and np.isfinite(dz).all()
                      and np.isfinite(dw).all() and np.isfinite([dtau, dtheta, dkappa]).all())
        return dx, dy, dz, dw, float(dtau), float(dtheta), float(dkappa), bool(ok_u and ok_h and ok_t and finite)
