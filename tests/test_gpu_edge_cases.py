"""Ragged and degenerate inputs on the device, against exact host results.

* zero right-hand sides: the HSD PCG returns x = 0 after no iteration and no
  product (psipm_v3_1_hsd.py:1026-1028); the spectral Newton solve returns
  dx = dy = 0 and reports convergence;
* an LP with an empty row, empty columns and single-entry columns (the
  row's H entry is delta alone; single-entry columns are in H but never
  candidates, psipm_stable_preconditioner.py:169-172): candidates, H v
  (1e-13), P^{-1} r against a direct solve of the oracle's assembled P (1e-9)
  and a tight Newton direction against the exact one (1e-8).
"""

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from _helpers import exact_direction, normal_matrix, rel

pytestmark = pytest.mark.gpu


def test_zero_right_hand_sides():
    from psipm_b200 import _lib, synthetic
    from psipm_b200.device import NormalEquationsDevice

    lp = synthetic.random_lp(200, 600, seed=11)
    m, n = lp.A.shape
    dev = NormalEquationsDevice(lp.A)
    try:
        theta = np.exp(np.random.default_rng(2).uniform(-3.0, 3.0, n))
        dev.set_theta(theta, 1e-6)
        dev.set_core(dev.candidates[: m])
        dev.factor(1e-6, 0)
        res = dev.pcg(np.zeros(m), 1e-10, 100, _lib.PCG_HSD)
        assert res.ok and res.iterations == 0 and res.matvecs == 0
        assert np.array_equal(res.x, np.zeros(m))
        dx, res = dev.solve(np.zeros(n), np.zeros(m), 1e-10, 100)
        assert res.info == 0 and res.ok
        assert not np.any(dx) and not np.any(res.x)
    finally:
        dev.close()


def ragged_lp_matrix():
    """random_lp(200, 600) with an empty row inserted at 57, five empty columns
    and five single-entry columns appended."""
    from psipm_b200 import synthetic

    A = synthetic.random_lp(200, 600, seed=12).A.tocoo()
    rows = A.row + (A.row >= 57)
    m, n = A.shape[0] + 1, A.shape[1]
    single_rows = np.array([0, 3, 100, 150, 200])
    rows = np.concatenate([rows, single_rows])
    cols = np.concatenate([A.col, n + 5 + np.arange(5)])
    vals = np.concatenate([A.data, np.linspace(0.5, 2.5, 5)])
    return sp.csc_matrix((vals, (rows, cols)), shape=(m, n + 10))


def test_empty_rows_and_columns():
    from oracle import stable as OS
    from psipm_b200.device import NormalEquationsDevice

    A = ragged_lp_matrix()
    A.sort_indices()
    m, n = A.shape
    assert np.diff(A.tocsr().indptr)[57] == 0
    dev = NormalEquationsDevice(A)
    try:
        assert np.array_equal(dev.candidates, np.flatnonzero(np.diff(A.indptr) >= 2))
        rng = np.random.default_rng(4)
        theta = np.exp(rng.uniform(-2.0, 2.0, n))
        delta = 1e-4
        dev.set_theta(theta, delta)
        v = rng.standard_normal(m)
        assert rel(dev.matvec(v), normal_matrix(A, theta, delta) @ v) <= 1e-13
        core = dev.candidates[::2].copy()
        dev.set_core(core)
        dev.factor(delta, 0)
        orc = OS.StableOracle(A, protected=np.zeros(n, dtype=bool), matching_backbone=False,
                              full_preconditioner_row_threshold=10)
        orc._weights = 1.0 / theta
        orc.core = core
        P = orc._assemble(theta, delta)
        r = rng.standard_normal(m)
        assert rel(dev.apply(r), spla.spsolve(P, r)) <= 1e-9
        r1, r2 = rng.standard_normal(n), rng.standard_normal(m)
        dx, res = dev.solve(r1, r2, 1e-13, 1000)
        dx_e, dy_e = exact_direction(A, theta, delta, r1, r2)
        assert res.info == 0, (res.info, res.relative_residual)
        assert rel(res.x, dy_e) <= 1e-8 and rel(dx, dx_e) <= 1e-8
        # the empty row's component is r2 / delta exactly up to the PCG's tolerance
        assert abs(res.x[57] - r2[57] / delta) <= 1e-8 * abs(r2[57] / delta)
    finally:
        dev.close()


def test_hsd_deadline_stops_after_one_iteration(golden):
    """A call that starts past its deadline does one iteration and reports no
    convergence (psipm_v3_1_hsd.py:1054-1055): one product for x0 = P^{-1} rhs and
    one for the iteration; the budget is cleared afterwards."""
    from psipm_b200.kkt import GpuStableColumnPreconditioner, pcg_rows

    g = golden("hsd_m1600")
    A = sp.csc_matrix((g["A_data"], g["A_indices"], g["A_indptr"]), shape=tuple(int(v) for v in g["A_shape"]))
    pre = GpuStableColumnPreconditioner(A)
    try:
        pre.factor(g["c0_D"], float(g["c0_delta"]))
        x, it, mv, ok, _ = pcg_rows(pre, g["c0_rhs"], 1e-10, 1000, deadline=0.0)
        assert (it, mv, ok) == (1, 2, False)
        assert np.all(np.isfinite(x))
        x, it, mv, ok, _ = pcg_rows(pre, g["c0_rhs"], 1e-10, 1000)
        assert ok and it > 1
    finally:
        pre.impl.close()


def test_grid_barrier_timeout_ends_quickly_and_leaves_the_handle_usable():
    """A block that never arrives: the other blocks' first wait runs out its
    (small) poll limit, sets the timeout flag, and every later wait gives up
    within a few polls, so 200 barriers end in well under a second with
    PSIPM_ERR_TIMEOUT; the handle then computes a correct product."""
    import ctypes

    from psipm_b200 import _lib, synthetic
    from psipm_b200.device import NormalEquationsDevice

    lp = synthetic.random_lp(200, 600, seed=12)
    m, n = lp.A.shape
    dev = NormalEquationsDevice(lp.A)
    try:
        secs = ctypes.c_double()
        # no block skipped: every wait ends normally
        assert dev.lib.psipm_debug_barrier_timeout(dev.h, 50, 1 << 20, -1, ctypes.byref(secs)) == _lib.OK
        status = dev.lib.psipm_debug_barrier_timeout(dev.h, 200, 4096, 1, ctypes.byref(secs))
        assert status == _lib.ERR_TIMEOUT
        assert secs.value < 1.0, f"timed-out barriers took {secs.value:.3f} s"
        theta = np.exp(np.random.default_rng(3).uniform(-2.0, 2.0, n))
        dev.set_theta(theta, 1e-6)
        v = np.random.default_rng(4).standard_normal(m)
        assert rel(dev.matvec(v), normal_matrix(lp.A, theta, 1e-6) @ v) < 1e-13
    finally:
        dev.close()
