"""The CPU oracle reproduces the reference's own outputs (golden fixtures).

The fixtures were produced by the unmodified reference with the SuperLU
stand-in factor (tests/golden/make_golden.py); the oracle uses the same
stand-in, so every comparison here is exact.
"""

import numpy as np
import pytest

from _helpers import NAMES, OPTIONS, exact_direction, lp_from, rel
from oracle import ipm as OI
from oracle import stable as OS

# dense_m1200 has four dense columns: the Woodbury extraction
# (psipm_active_pool.py:691-718, 906-956) is part of every call there
PINNED = NAMES + ("dense_m1200",)


@pytest.mark.parametrize("name", PINNED)
def test_full_solve_bit_exact(name, golden):
    g = golden(name)
    lp = lp_from(g)
    solver = OS.SpectralOracle(lp.A, protected=~lp.pos, **OPTIONS)
    sol = OI.psipm_solve(lp, solver, tol=1e-8)
    assert sol.status == str(g["status"])
    assert sol.obj == float(g["obj"])
    assert np.array_equal(sol.x, g["x"])
    assert np.array_equal(sol.y, g["y"])
    assert solver.cg_iterations == [int(v) for v in g["cg_iterations"]]
    assert solver.core_sizes == [int(v) for v in g["core_sizes"]]
    assert np.array_equal(solver.candidates, g["candidates"])
    if "low_rank_columns" in g:
        assert np.array_equal(solver.low_rank_columns, g["low_rank_columns"])
    assert np.array_equal(solver.matching_columns if solver.matching_columns.size else
                          g["matching_columns"], g["matching_columns"])
    for i in range(int(g["n_cores"])):
        assert np.array_equal(solver.core_history[i], g[f"core{i}"]), f"core {i}"


@pytest.mark.parametrize("name", PINNED)
def test_scores_bit_exact(name, golden):
    g = golden(name)
    lp = lp_from(g)
    solver = OS.SpectralOracle(lp.A, protected=~lp.pos, **OPTIONS)
    checked = 0
    for i in range(int(g["n_factor_calls"])):
        key = f"f{i}_scores"
        if key not in g:
            continue
        weights = 1.0 / g[f"f{i}_theta"]
        scores = solver._scores(weights, float(g[f"f{i}_delta"]))
        assert np.array_equal(scores, g[key])
        checked += 1
    assert checked >= 1


@pytest.mark.parametrize("name", NAMES)
def test_recorded_directions(name, golden):
    """Replaying a recorded solve through the oracle meets the same tolerance
    and lands as close to the exact direction as the reference did."""
    g = golden(name)
    lp = lp_from(g)
    for i in range(min(4, int(g["n_solve_calls"]))):
        theta, delta = g[f"s{i}_theta"], float(g[f"s{i}_delta"])
        r1, r2, tol = g[f"s{i}_r1"], g[f"s{i}_r2"], float(g[f"s{i}_tolerance"])
        s = OS.SpectralOracle(lp.A, protected=~lp.pos, **OPTIONS)
        s._weights = 1.0 / theta
        s.core = g[f"s{i}_core"]
        s._initialized = True
        OS.NormalEquationsOracle.factorize(s, theta, delta)
        res = s._pcg(np.asarray(r2 - lp.A @ (r1 / theta)).ravel(), tol)
        assert res.relative_residual <= tol
        _, dy_exact = exact_direction(lp.A, theta, delta, r1, r2)
        ref_err = rel(g[f"s{i}_dy"], dy_exact)
        assert rel(res.solution, dy_exact) <= 10.0 * ref_err + 1e-9


def test_top_k_rule_matches_numpy_without_straddling_ties():
    rng = np.random.default_rng(7)
    for _ in range(50):
        s = rng.standard_normal(500)
        s[rng.integers(0, 500, 20)] = np.inf
        s[rng.integers(0, 500, 5)] = np.nan
        k = int(rng.integers(1, 600))
        assert np.array_equal(np.sort(OS.top_k(s, k)), np.sort(OS.top_k_numpy(s, k)))


def test_top_k_tie_rule_is_index_ascending():
    s = np.array([1.0, 2.0, 2.0, 2.0, 0.5, 2.0])
    assert list(OS.top_k(s, 3)) == [1, 2, 3]
    assert list(OS.top_k(s, 5)) == [1, 2, 3, 5, 0]
