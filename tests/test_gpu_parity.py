"""Device results against the reference's golden fixtures and exact solves.

Bars (FP64 mode):
* scores: bit-identical to the reference (FP64, no FMA contraction);
* refreshed cores: identical index sets;
* H v: 1e-13 relative to SciPy;
* P^{-1} r: 1e-9 relative to a sparse direct solve of the assembled P;
* Newton directions at tolerance 1e-13: 1e-8 relative to the exact direction;
  at the reference's own tolerance: the PCG contract, relative residual <=
  tolerance, checked on the host (two solves that both meet a loose tolerance
  may differ from each other by up to condition x tolerance);
* full PS-IPM solve: optimal, objective within 1e-8 relative.
"""

import numpy as np
import pytest
import scipy.sparse.linalg as spla

from _helpers import NAMES, OPTIONS, exact_direction, lp_from, normal_matrix, rel

pytestmark = pytest.mark.gpu


def device_for(lp):
    from psipm_b200.device import NormalEquationsDevice

    return NormalEquationsDevice(lp.A)


def mandatory_local(dev, g, lp):
    prot = ~lp.pos
    mandatory = np.union1d(dev.candidates[prot[dev.candidates]], g["matching_columns"])
    return np.searchsorted(dev.candidates, mandatory)


@pytest.mark.parametrize("name", NAMES)
def test_candidates_match(name, golden):
    g = golden(name)
    dev = device_for(lp_from(g))
    assert np.array_equal(dev.candidates, g["candidates"])


@pytest.mark.parametrize("name", NAMES)
def test_scores_bit_exact(name, golden):
    g = golden(name)
    dev = device_for(lp_from(g))
    checked = 0
    for i in range(int(g["n_factor_calls"])):
        if f"f{i}_scores" not in g:
            continue
        dev.set_theta(g[f"f{i}_theta"], float(g[f"f{i}_delta"]))
        scores, _ = dev.scores(0.2)
        assert np.array_equal(scores, g[f"f{i}_scores"]), f"call {i}"
        checked += 1
    assert checked


@pytest.mark.parametrize("name", NAMES)
def test_refresh_core_identical_index_set(name, golden):
    g = golden(name)
    lp = lp_from(g)
    dev = device_for(lp)
    mand = mandatory_local(dev, g, lp)
    checked = 0
    for i in range(int(g["n_factor_calls"])):
        if f"f{i}_scores" not in g:
            continue
        before = g[f"f{i}_core_before"]
        dev.set_core(before)
        dev.set_theta(g[f"f{i}_theta"], float(g[f"f{i}_delta"]))
        dev.scores(0.2, want=False)
        core, _ = dev.refresh_core(int(g[f"f{i}_core_target"]), 0.9, before.size > 0, mand)
        assert np.array_equal(core, g[f"f{i}_core"]), f"call {i}"
        checked += 1
    assert checked


@pytest.mark.parametrize("name", NAMES)
def test_matvec(name, golden):
    g = golden(name)
    lp = lp_from(g)
    dev = device_for(lp)
    theta, delta = g["s2_theta"], float(g["s2_delta"])
    dev.set_theta(theta, delta)
    v = np.random.default_rng(1).standard_normal(lp.A.shape[0])
    assert rel(dev.matvec(v), normal_matrix(lp.A, theta, delta) @ v) <= 1e-13


@pytest.mark.parametrize("name", NAMES)
def test_apply_is_inverse_of_assembled_preconditioner(name, golden):
    from oracle import stable as OS

    g = golden(name)
    lp = lp_from(g)
    dev = device_for(lp)
    for i in (0, 2, 4):
        theta, delta, core = g[f"s{i}_theta"], float(g[f"s{i}_delta"]), g[f"s{i}_core"]
        dev.set_theta(theta, delta)
        dev.set_core(core)
        shift, _ = dev.factor(delta, 0)
        assert shift == 0
        orc = OS.StableOracle(lp.A, protected=~lp.pos, matching_backbone=False, **OPTIONS)
        orc._weights = 1.0 / theta
        orc.core = core
        P = orc._assemble(theta, delta)
        r = np.random.default_rng(i).standard_normal(lp.A.shape[0])
        assert rel(dev.apply(r), spla.spsolve(P, r)) <= 1e-9, f"call {i}"


@pytest.mark.parametrize("name", NAMES)
def test_directions_tight_tolerance(name, golden):
    g = golden(name)
    lp = lp_from(g)
    dev = device_for(lp)
    for i in range(min(6, int(g["n_solve_calls"]))):
        theta, delta = g[f"s{i}_theta"], float(g[f"s{i}_delta"])
        dev.set_theta(theta, delta)
        dev.set_core(g[f"s{i}_core"])
        dev.factor(delta, 0)
        dx, res = dev.solve(g[f"s{i}_r1"], g[f"s{i}_r2"], 1e-13, 1000)
        dx_e, dy_e = exact_direction(lp.A, theta, delta, g[f"s{i}_r1"], g[f"s{i}_r2"])
        assert res.info == 0, (i, res.info, res.relative_residual)
        assert rel(res.x, dy_e) <= 1e-8, i
        assert rel(dx, dx_e) <= 1e-8, i


@pytest.mark.parametrize("name", NAMES)
def test_directions_reference_tolerance(name, golden):
    g = golden(name)
    lp = lp_from(g)
    dev = device_for(lp)
    for i in range(min(6, int(g["n_solve_calls"]))):
        theta, delta, tol = g[f"s{i}_theta"], float(g[f"s{i}_delta"]), float(g[f"s{i}_tolerance"])
        dev.set_theta(theta, delta)
        dev.set_core(g[f"s{i}_core"])
        dev.factor(delta, 0)
        dx, res = dev.solve(g[f"s{i}_r1"], g[f"s{i}_r2"], tol, 200)
        assert res.relative_residual <= tol, i
        # the residual bound is what PCG guarantees; check it independently
        H = normal_matrix(lp.A, theta, delta)
        rhs = g[f"s{i}_r2"] - lp.A @ (g[f"s{i}_r1"] / theta)
        host_rel = np.linalg.norm(rhs - H @ res.x) / max(1.0, np.linalg.norm(rhs))
        assert host_rel <= tol * (1 + 1e-6), i
        assert rel(dx, g[f"s{i}_r1"] / theta + (lp.A.T @ res.x) / theta) <= 1e-12


@pytest.mark.parametrize("name", NAMES)
def test_full_solve_matches_reference_objective(name, golden):
    from oracle import ipm as OI
    from psipm_b200.kkt import GpuSpectralStableColumnPreconditioner

    g = golden(name)
    lp = lp_from(g)
    solver = GpuSpectralStableColumnPreconditioner(lp.A, protected=~lp.pos, **OPTIONS)
    sol = OI.psipm_solve(lp, solver, tol=1e-8)
    assert sol.status == "optimal"
    ref = float(g["obj"])
    assert abs(sol.obj - ref) <= 1e-8 * abs(ref)
    assert sol.res_p < 1e-8 and sol.res_d < 1e-8
