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
