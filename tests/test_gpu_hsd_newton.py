"""Reduced HSD Newton system on the device (psipm_b200.hsd) against the reference.

Fixture hsd_newton_m1600: the reference's HSDNewtonSystem over its
StableColumnPreconditioner, two systems with an affine and a corrector
direction each.  Bars: the device preconditioner picks the reference's cores
and factor counts; every direction is within 1e-8 of the direction obtained
with direct solves (the reference's own are within 2e-9; the PCG tolerance is
1e-10 and the systems' condition numbers are near 700) and within 1e-8 of the
reference's; the okay flags and the LinearStats solve/failure counts match.
"""

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from oracle import hsd as OH
from test_hsd_oracle import hsd_newton_case, hsd_newton_rhs

pytestmark = pytest.mark.gpu

NAMES = ("dx", "dy", "dz", "dw", "dtau", "dtheta", "dkappa")


class _Exact(OH.HSDNewtonSystemOracle):
    """The same Newton system with direct normal-equations solves."""

    def solve_rows(self, rhs):
        H = (self.A @ sp.diags(self.D) @ self.A.T + self.delta * sp.eye(self.A.shape[0])).tocsc()
        return spla.spsolve(H, rhs), True


class _NoFactor:
    def factor(self, weights, delta):
        return 0.0


def rel(a, b):
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1.0))


def test_hsd_newton_directions(golden):
    from psipm_b200.hsd import HSDNewtonSystem, LinearStats
    from psipm_b200.kkt import GpuStableColumnPreconditioner

    g = golden("hsd_newton_m1600")
    A = sp.csc_matrix((g["A_data"], g["A_indices"], g["A_indptr"]), shape=tuple(int(v) for v in g["A_shape"]))
    pre = GpuStableColumnPreconditioner(A, growth_amortization=float(g["growth_amortization"]))
    stats = LinearStats()
    try:
        for sys_i in range(2):
            st, emb, opts, D = hsd_newton_case(g, sys_i)
            args = (A, g["c"], g["upper"], g["b"], D, float(g["delta"]), float(g["eta"]), st, emb)
            system = HSDNewtonSystem(*args, pre, float(g["pcg_tolerance"]), opts, np.inf, stats)
            assert np.array_equal(pre.impl.core, g[f"s{sys_i}_core"]), sys_i
            assert pre.impl.n_fact == int(g[f"s{sys_i}_n_fact"]), sys_i
            exact = _Exact(*args, _NoFactor(), 1e-10, opts, np.inf, LinearStats())
            for d_i in range(2):
                tag = f"s{sys_i}d{d_i}"
                rhs = hsd_newton_rhs(g, tag)
                got, want = system.direction(*rhs), exact.direction(*rhs)
                assert got[-1] and bool(g[f"{tag}_ok"]), tag
                for k, name in enumerate(NAMES):
                    assert rel(got[k], want[k]) <= 1e-8, (tag, name, rel(got[k], want[k]))
                    assert rel(got[k], g[f"{tag}_{name}"]) <= 1e-8, (tag, name)
            want_stats = g[f"s{sys_i}_stats"].tolist()
            assert [stats.solves, stats.failures] == [want_stats[0], want_stats[4]]
            assert stats.iterations > 0 and stats.preconditioner_seconds > 0.0
    finally:
        pre.impl.close()
