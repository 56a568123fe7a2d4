"""Device V3.1 HSD surface: stable-rule cores and the HSD PCG on the device.

Bars: the refreshed core equals the reference's (golden fixture hsd_m1600);
a converged device PCG lands within 1e-7 of the exact solution of
A D A' x + delta x = rhs; non-converged calls are reported as such.
"""

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

pytestmark = pytest.mark.gpu


def test_hsd_surface(golden):
    from psipm_b200.kkt import GpuStableColumnPreconditioner, pcg_rows

    g = golden("hsd_m1600")
    A = sp.csc_matrix((g["A_data"], g["A_indices"], g["A_indptr"]), shape=tuple(int(v) for v in g["A_shape"]))
    pre = GpuStableColumnPreconditioner(A)
    for call in range(3):
        D, delta, rhs = g[f"c{call}_D"], float(g[f"c{call}_delta"]), g[f"c{call}_rhs"]
        pre.factor(D, delta)
        assert np.array_equal(pre.impl.core, g[f"c{call}_core"]), call
        assert pre.impl.n_fact == int(g[f"c{call}_n_fact"]), call
        x, it, mv, ok, _ = pcg_rows(pre, rhs, 1e-10, 1000)
        pre.record_iterations(it, 0.0, ok)
        if bool(g[f"c{call}_ok"]):
            assert ok, (call, it)
            H = (A @ sp.diags(D) @ A.T + delta * sp.eye(A.shape[0])).tocsc()
            exact = spla.spsolve(H, rhs)
            assert np.linalg.norm(x - exact) <= 1e-7 * np.linalg.norm(exact), call
            assert abs(it - int(g[f"c{call}_iterations"])) <= 0.25 * int(g[f"c{call}_iterations"]) + 5
        else:
            # the reference's lagged factor did not reach 1e-10 in 1000 iterations
            assert it >= 1
