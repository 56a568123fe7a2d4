"""F3: dense columns left out of the factor and corrected by Woodbury.

Fixture ``dense_m1200`` (tests/golden/make_golden.py) is the reference run on
a random LP with four 1,100-entry columns, which its
``_low_rank_normal_columns`` extracts (psipm_active_pool.py:691-718).
Checked: the same columns and candidates, bit-identical scores with the
low-rank diagonal (psipm_stable_preconditioner.py:298-303), the corrected
apply equal to H^{-1} when the core holds every candidate (then
P_base + A_L W_L A_L^T = H), and a full solve at the reference's objective.
"""

import numpy as np
import pytest
import scipy.sparse.linalg as spla

from _helpers import OPTIONS, lp_from, normal_matrix, rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dense(golden):
    return golden("dense_m1200")


def test_columns_and_candidates_match_reference(dense):
    from psipm_b200.device import NormalEquationsDevice
    from psipm_b200.kkt import low_rank_normal_columns

    lp = lp_from(dense)
    cols = low_rank_normal_columns(lp.A, 8, 1024, 2.0)
    assert np.array_equal(cols, dense["low_rank_columns"])
    dev = NormalEquationsDevice(lp.A)
    try:
        dev.set_low_rank(cols)
        assert np.array_equal(dev.candidates, dense["candidates"])
    finally:
        dev.close()


def test_scores_bit_exact_with_low_rank_diagonal(dense):
    from psipm_b200.device import NormalEquationsDevice

    lp = lp_from(dense)
    dev = NormalEquationsDevice(lp.A)
    try:
        dev.set_low_rank(dense["low_rank_columns"])
        checked = 0
        for i in range(int(dense["n_factor_calls"])):
            if f"f{i}_scores" not in dense:
                continue
            dev.set_theta(dense[f"f{i}_theta"], float(dense[f"f{i}_delta"]))
            got, _ = dev.scores(0.2)
            assert np.array_equal(got, dense[f"f{i}_scores"]), i
            checked += 1
        assert checked >= 1
    finally:
        dev.close()


def test_corrected_apply_is_h_inverse(dense):
    from psipm_b200.device import NormalEquationsDevice

    lp = lp_from(dense)
    n = lp.A.shape[1]
    theta = np.exp(np.random.default_rng(4).uniform(-3, 3, n))
    delta = 1e-6
    dev = NormalEquationsDevice(lp.A)
    try:
        dev.set_low_rank(dense["low_rank_columns"])
        dev.set_theta(theta, delta)
        dev.set_core(dev.candidates)
        dev.factor(delta, 0)
        H = normal_matrix(lp.A, theta, delta)
        for seed in range(2):
            r = np.random.default_rng(seed).standard_normal(lp.A.shape[0])
            assert rel(dev.apply(r), spla.spsolve(H, r)) <= 1e-9
        # and the PCG on H converges in a couple of iterations with it
        res = dev.pcg(r, 1e-12, 50)
        assert res.relative_residual <= 1e-12 and res.iterations <= 5
    finally:
        dev.close()


def test_full_solve_matches_reference_objective(dense):
    from psipm_b200.ipm_device import psipm_solve_resident
    from psipm_b200.kkt import GpuSpectralStableColumnPreconditioner

    lp = lp_from(dense)
    solver = GpuSpectralStableColumnPreconditioner(lp.A, protected=~lp.pos, **OPTIONS)
    try:
        assert np.array_equal(solver.low_rank_columns, dense["low_rank_columns"])
        sol = psipm_solve_resident(lp, solver, tol=1e-8)
    finally:
        solver.close()
    assert sol.status == "optimal"
    ref = float(dense["obj"])
    assert abs(sol.obj - ref) <= 1e-8 * abs(ref)
