"""Host arithmetic of ``psipm_b200.hsd.HSDNewtonSystem`` (no GPU).

The device Newton solve is replaced by a stand-in with the same contract
(``solve_normal``: ``dy = H^{-1}(r2 - A (r1/theta))``, ``dx = r1/theta + A' dy / theta``)
built on the oracle's HSD PCG and preconditioner, so every line of the Newton
system's own arithmetic — the border data, the folded right-hand sides, the
2 x 2 border solve and the recombined ``dx`` — runs as it does over the
device.  Bars: the same cores and factor counts as the reference fixture
hsd_newton_m1600, directions within 1e-8 of the reference's (both are PCG
solves to 1e-10 on systems with condition numbers near 700), the reference's
LinearStats counters, and the near-singular border guard.
"""

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import hsd as OH
from psipm_b200.hsd import HSDNewtonSystem, LinearStats
from test_hsd_oracle import hsd_newton_case, hsd_newton_rhs

TINY = float(np.finfo(float).tiny)
NAMES = ("dx", "dy", "dz", "dw", "dtau", "dtheta", "dkappa", "ok")


class OracleNormalSolve:
    """``GpuStableColumnPreconditioner``'s HSD contract over the oracle."""

    def __init__(self, A, **options):
        self.pre = OH.StableColumnPreconditionerOracle(A, **options)
        self.impl = self.pre.impl
        self.A = A
        self.calls = []

    def factor(self, weights, delta):
        self.theta = 1.0 / np.maximum(weights, TINY)
        self.delta = float(delta)
        return self.pre.factor(weights, delta)

    def solve_normal(self, r1, r2, rtol, max_iterations, deadline=np.inf):
        A, theta, delta = self.A, self.theta, self.delta
        w1 = r1 / theta
        rhs = r2 - A @ w1
        x, it, mv, ok, elapsed = OH.pcg(lambda v: A @ ((A.T @ v) / theta) + delta * v, rhs, self.pre, rtol,
                                        max_iterations, deadline)
        self.calls.append((np.array(r1), np.array(r2)))
        return w1 + (A.T @ x) / theta, x, it, mv, ok, elapsed

    def record_solve(self, iterations, elapsed, converged):
        self.pre.record_iterations(iterations, elapsed, converged)


def rel(a, b):
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1.0))


@pytest.fixture(scope="module")
def fixture(golden):
    g = golden("hsd_newton_m1600")
    A = sp.csc_matrix((g["A_data"], g["A_indices"], g["A_indptr"]), shape=tuple(int(v) for v in g["A_shape"]))
    return g, A


def build(g, A, pre, stats, sys_i):
    st, emb, opts, D = hsd_newton_case(g, sys_i)
    return HSDNewtonSystem(A, g["c"], g["upper"], g["b"], D, float(g["delta"]), float(g["eta"]), st, emb, pre,
                           float(g["pcg_tolerance"]), opts, np.inf, stats)


def test_directions_match_reference(fixture):
    g, A = fixture
    pre = OracleNormalSolve(A, growth_amortization=float(g["growth_amortization"]))
    stats = LinearStats()
    for sys_i in range(2):
        system = build(g, A, pre, stats, sys_i)
        assert np.array_equal(pre.impl.core, g[f"s{sys_i}_core"]) and pre.impl.n_fact == int(g[f"s{sys_i}_n_fact"])
        for d_i in range(2):
            tag = f"s{sys_i}d{d_i}"
            got = system.direction(*hsd_newton_rhs(g, tag))
            for k, name in enumerate(NAMES[:-1]):
                assert rel(got[k], g[f"{tag}_{name}"]) <= 1e-8, (tag, name, rel(got[k], g[f"{tag}_{name}"]))
            assert got[-1] == bool(g[f"{tag}_ok"])
        want = g[f"s{sys_i}_stats"].tolist()
        assert [stats.solves, stats.failures] == [want[0], want[4]]
        # iteration counts may move by one at the stopping threshold: the
        # stand-in forms A (r1/theta) where the reference forms A (D r1)
        assert abs(stats.iterations - want[1]) <= 2 * stats.solves and abs(stats.matvecs - want[3]) <= 2 * stats.solves


def test_right_hand_sides_fold_into_newton_solves(fixture):
    """The three solves of the first direction carry (q, -rhs_p), (-c_dir, b) and
    (-bar_c, bar_b); later directions reuse h' and t' (psipm_v3_1_hsd.py:1169-1176)."""
    g, A = fixture
    pre = OracleNormalSolve(A, growth_amortization=float(g["growth_amortization"]))
    system = build(g, A, pre, LinearStats(), 0)
    rhs = hsd_newton_rhs(g, "s0d0")
    system.direction(*rhs)
    assert len(pre.calls) == 3
    D, theta = system.D, pre.theta
    st = system.state
    up = np.where(system.boxed, rhs[5] / system.slack, 0.0)
    q = rhs[0] + rhs[4] / st.x - up
    (r1u, r2u), (r1h, r2h), (r1t, r2t) = pre.calls
    assert np.array_equal(r1u, q) and np.array_equal(r2u, -rhs[1])
    # the device's right-hand sides equal the reference's h and theta_row to rounding
    assert rel(r2h - A @ (r1h / theta), g["b"] + A @ (D * system.c_direction)) <= 1e-14
    assert rel(r2t - A @ (r1t / theta), system.embedding.bar_b + A @ (D * system.embedding.bar_c)) <= 1e-14
    system.direction(*hsd_newton_rhs(g, "s0d1"))
    assert len(pre.calls) == 4


def test_singular_border_is_shifted_and_reported(fixture):
    """A border matrix with determinant 0 is shifted by 64 eps ||B|| I and the
    direction is reported as not okay (psipm_v3_1_hsd.py:1210-1221)."""
    g, A = fixture
    pre = OracleNormalSolve(A, growth_amortization=float(g["growth_amortization"]))
    system = build(g, A, pre, LinearStats(), 0)
    oracle = OH.HSDNewtonSystemOracle(A, g["c"], g["upper"], g["b"], system.D, system.delta, system.eta,
                                      system.state, system.embedding, OH.StableColumnPreconditionerOracle(
                                          A, growth_amortization=float(g["growth_amortization"])),
                                      system.pcg_tolerance, system.options, np.inf,
                                      LinearStats())
    rhs = hsd_newton_rhs(g, "s0d0")
    for s in (system, oracle):
        s.direction(*rhs)  # solves h' and t'
        hs = s._h[1] if s is system else s._h_solution
        ts = s._t[1] if s is system else s._theta_solution
        # make the first border row zero: alpha = -g.h', beta = g.t'
        s.alpha = -float(s.g @ hs)
        s.beta = float(s.g @ ts)
    got, want = system.direction(*rhs), oracle.direction(*rhs)
    assert got[-1] is False and want[-1] is False
    assert abs(got[4] - want[4]) <= 1e-6 * max(1.0, abs(want[4]))
    assert rel(got[1], want[1]) <= 1e-6


def test_deadline_becomes_a_device_budget():
    """A finite deadline is passed to the device PCG as the time left (at
    least 1 ns: one iteration, as the reference when it starts past its deadline,
    psipm_v3_1_hsd.py:1054-1055) and cleared afterwards; none is set without one."""
    from types import SimpleNamespace as NS

    from psipm_b200.kkt import pcg_rows

    class Dev:
        def __init__(self):
            self.budgets = []

        def set_pcg_budget(self, seconds):
            self.budgets.append(seconds)

        def pcg(self, rhs, tol, maxit, variant):
            return NS(x=np.zeros(3), iterations=1, matvecs=2, ok=False)

    dev = Dev()
    pre = NS(impl=NS(dev=dev))
    assert pcg_rows(pre, np.ones(3), 1e-10, 50)[3] is False and dev.budgets == []
    pcg_rows(pre, np.ones(3), 1e-10, 50, deadline=0.0)
    assert dev.budgets == [1e-9, 0.0]
    import time

    pcg_rows(pre, np.ones(3), 1e-10, 50, deadline=time.perf_counter() + 100.0)
    assert 99.0 < dev.budgets[2] <= 100.0 and dev.budgets[3] == 0.0
