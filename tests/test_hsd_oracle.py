"""The oracle's V3.1 HSD surface reproduces the reference (golden fixture hsd_m1600)."""

import numpy as np
import scipy.sparse as sp

from oracle import hsd as OH


def test_hsd_factor_and_pcg_bit_exact(golden):
    g = golden("hsd_m1600")
    A = sp.csc_matrix((g["A_data"], g["A_indices"], g["A_indptr"]), shape=tuple(int(v) for v in g["A_shape"]))
    pre = OH.StableColumnPreconditionerOracle(A)
    for call in range(3):
        D, delta, rhs = g[f"c{call}_D"], float(g[f"c{call}_delta"]), g[f"c{call}_rhs"]
        pre.factor(D, delta)
        assert np.array_equal(pre.impl.core, g[f"c{call}_core"]), call
        assert pre.impl.n_fact == int(g[f"c{call}_n_fact"]), call

        def matvec(v):
            return A @ (D * (A.T @ v)) + delta * v

        x, it, mv, ok, _ = OH.pcg(matvec, rhs, pre, 1e-10, 1000)
        pre.record_iterations(it, 0.0, ok)
        assert it == int(g[f"c{call}_iterations"]) and mv == int(g[f"c{call}_matvecs"]), call
        assert bool(ok) == bool(g[f"c{call}_ok"]), call
        assert np.array_equal(x, g[f"c{call}_x"]), call


def hsd_newton_case(g, sys_i):
    """Inputs of system ``sys_i`` of the hsd_newton_m1600 fixture as plain namespaces."""
    from types import SimpleNamespace as NS

    st = NS(x=g[f"s{sys_i}_x"], z=g[f"s{sys_i}_z"], w=g[f"s{sys_i}_w"], tau=float(g[f"s{sys_i}_tau"]),
            kappa=float(g[f"s{sys_i}_kappa"]))
    emb = NS(bar_b=g[f"s{sys_i}_bar_b"], bar_c=g[f"s{sys_i}_bar_c"], bar_g=float(g[f"s{sys_i}_bar_g"]))
    opts = NS(zeta=float(g["zeta"]), pcg_max_iterations=int(g["pcg_max_iterations"]))
    return st, emb, opts, g[f"s{sys_i}_D"]


def hsd_newton_rhs(g, tag):
    return [g[f"{tag}_rhs{k}"] if g[f"{tag}_rhs{k}"].ndim else float(g[f"{tag}_rhs{k}"]) for k in range(7)]


def test_hsd_newton_system_bit_exact(golden):
    """HSDNewtonSystemOracle over the oracle preconditioner reproduces the reference's
    HSDNewtonSystem (psipm_v3_1_hsd.py:1066-1264) bit for bit: two systems, an affine
    and a corrector direction each, and the LinearStats counters."""
    from types import SimpleNamespace as NS

    g = golden("hsd_newton_m1600")
    A = sp.csc_matrix((g["A_data"], g["A_indices"], g["A_indptr"]), shape=tuple(int(v) for v in g["A_shape"]))
    pre = OH.StableColumnPreconditionerOracle(A, growth_amortization=float(g["growth_amortization"]))
    stats = NS(iterations=0, max_iterations=0, solves=0, matvecs=0, failures=0, seconds=0.0,
               preconditioner_seconds=0.0)
    names = ("dx", "dy", "dz", "dw", "dtau", "dtheta", "dkappa", "ok")
    for sys_i in range(2):
        st, emb, opts, D = hsd_newton_case(g, sys_i)
        system = OH.HSDNewtonSystemOracle(A, g["c"], g["upper"], g["b"], D, float(g["delta"]), float(g["eta"]), st,
                                          emb, pre, float(g["pcg_tolerance"]), opts, np.inf, stats)
        assert np.array_equal(pre.impl.core, g[f"s{sys_i}_core"]) and pre.impl.n_fact == int(g[f"s{sys_i}_n_fact"])
        for d_i in range(2):
            tag = f"s{sys_i}d{d_i}"
            got = system.direction(*hsd_newton_rhs(g, tag))
            for k, name in enumerate(names):
                assert np.array_equal(np.asarray(got[k]), g[f"{tag}_{name}"]), (tag, name)
        assert [stats.solves, stats.iterations, stats.max_iterations, stats.matvecs, stats.failures] == \
            g[f"s{sys_i}_stats"].tolist()
