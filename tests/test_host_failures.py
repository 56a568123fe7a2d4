"""Host-side failure handling of the drop-in solver and the IPM loop.

Failures are injected on the host (a fake device returns library status
codes or a PCG breakdown code); no GPU is involved.  The reference's
contract (psipm_active_pool.py:2033-2040, 2046-2049, 2066-2073): any
exception from ``factorize`` and a ``KKTSolveError`` from ``solve`` make
``prox_eval`` raise ``reg_extra`` and retry the iteration.
"""

import numpy as np
import pytest

from _helpers import exact_direction
from fake_device import FakeDevice
from oracle import ipm
from psipm_b200 import _lib, synthetic
from psipm_b200.kkt import GpuSpectralStableColumnPreconditioner, KKTSolveError

OPTS = dict(full_preconditioner_row_threshold=10)


def make(lp, dev, **kw):
    return GpuSpectralStableColumnPreconditioner(lp.A, protected=~lp.pos, dev=dev, **OPTS, **kw)


@pytest.fixture(scope="module")
def lp():
    return synthetic.random_lp(120, 360, seed=9)


def test_fake_device_drives_a_full_solve(lp):
    solver = make(lp, FakeDevice(lp.A))
    sol = ipm.psipm_solve(lp, solver, tol=1e-8)
    assert sol.status == "optimal"
    for name in ("cg_iterations", "core_sizes", "n_fact", "retained_fractions", "n_symbolic",
                 "condition_estimates", "lag_spectral_bounds", "residual_replacements", "krylov_breakdowns",
                 "pcg_retries", "cg_failures", "full_fallbacks", "refreshes", "t_fact", "t_solve"):
        assert hasattr(solver, name), name


def test_factor_failure_is_a_kkt_error_and_the_ipm_retries(lp):
    dev = FakeDevice(lp.A)
    solver = make(lp, dev)
    dev.fail["factor"] = [None, None, _lib.ERR_NOT_PD]  # start point, 1st IPM iteration ok, then NOT_PD
    sol = ipm.psipm_solve(lp, solver, tol=1e-8)
    assert sol.status == "optimal"
    assert solver.stats["not_pd"] > 0
    assert dev.calls["factor"] >= 4


def test_cuda_error_in_solve_becomes_kkt_error(lp):
    dev = FakeDevice(lp.A)
    solver = make(lp, dev)
    solver.factorize(np.ones(lp.A.shape[1]), 1.0)
    dev.fail["solve"] = [_lib.ERR_CUDA]
    with pytest.raises(KKTSolveError):
        solver.solve(np.zeros(lp.A.shape[1]), lp.b)
    assert solver.cg_failures == 1
    dx, dy = solver.solve(np.zeros(lp.A.shape[1]), lp.b)  # the next call works again
    assert np.isfinite(dx).all() and np.isfinite(dy).all()


def test_breakdown_triggers_retry_with_growth_then_error(lp):
    dev = FakeDevice(lp.A)
    solver = make(lp, dev, minres_fallback=False)
    solver.factorize(np.ones(lp.A.shape[1]), 1.0)
    target = solver.core_target
    dev.fail["solve_info"] = [-2, -2]  # breakdown on the first try and on the retry
    with pytest.raises(KKTSolveError):
        solver.solve(np.zeros(lp.A.shape[1]), lp.b)
    assert solver.pcg_retries == 1
    assert solver.core_target > target or solver.core_target == solver.max_core_target
    assert solver.krylov_breakdowns == 1


def test_breakdown_after_retry_falls_back_to_minres(lp):
    """PCG breaks down on the first try and on the retry: the solver answers
    with the augmented MINRES (psipm_spectral_preconditioner.py:717-737)."""
    dev = FakeDevice(lp.A)
    solver = make(lp, dev)
    solver.factorize(np.ones(lp.A.shape[1]), 1.0)
    dev.fail["solve_info"] = [-2, -2]
    r1 = np.random.default_rng(1).standard_normal(lp.A.shape[1])
    dx, dy = solver.solve(r1, lp.b)
    assert solver.minres_fallbacks == 1 and solver.full_fallbacks == 1
    assert solver.minres_iterations > 0 and solver.cg_failures == 1
    ex_dx, ex_dy = exact_direction(lp.A, solver.theta, solver.delta, r1, lp.b)
    assert np.linalg.norm(dy - ex_dy) <= 1e-4 * np.linalg.norm(ex_dy)


def test_minres_failure_is_a_kkt_error(lp):
    dev = FakeDevice(lp.A)
    solver = make(lp, dev)
    solver.factorize(np.ones(lp.A.shape[1]), 1.0)
    dev.fail["solve_info"] = [-2, -2]
    dev.fail["minres"] = [_lib.ERR_CUDA]
    with pytest.raises(KKTSolveError):
        solver.solve(np.zeros(lp.A.shape[1]), lp.b)
    assert solver.minres_fallbacks == 1


def test_device_deadline_code_is_reported(lp):
    dev = FakeDevice(lp.A)
    solver = make(lp, dev)
    solver.factorize(np.ones(lp.A.shape[1]), 1.0)
    dev.fail["solve"] = [_lib.ERR_TIMEOUT]
    with pytest.raises(KKTSolveError, match="deadline"):
        solver.solve(np.zeros(lp.A.shape[1]), lp.b)


def test_solve_before_factorize_is_an_error(lp):
    solver = make(lp, FakeDevice(lp.A))
    with pytest.raises(KKTSolveError):
        solver.solve(np.zeros(lp.A.shape[1]), lp.b)


def test_invalid_options_raise_like_the_reference(lp):
    with pytest.raises(ValueError):
        GpuSpectralStableColumnPreconditioner(lp.A, dev=FakeDevice(lp.A), core_factor=0.0)
    with pytest.raises(ValueError):
        GpuSpectralStableColumnPreconditioner(lp.A, dev=FakeDevice(lp.A), retention=1.5)
    with pytest.raises(ValueError):
        GpuSpectralStableColumnPreconditioner(lp.A, dev=FakeDevice(lp.A), cg_tol=0.5, cg_tol_max=0.1)
    with pytest.raises(ValueError):
        GpuSpectralStableColumnPreconditioner(lp.A, protected=np.ones(3, bool), dev=FakeDevice(lp.A))


def test_memory_cap_keeps_the_largest_core_that_fitted(lp):
    """A factor that does not fit lowers the core target to 0.8 of that core,
    but never below the largest core factored so far."""
    dev = FakeDevice(lp.A)
    solver = make(lp, dev)
    m = lp.A.shape[0]
    theta = np.ones(lp.A.shape[1])
    solver.factorize(theta, 1.0)
    fitted = solver.core.size
    assert fitted > 0
    solver.core = np.arange(int(1.1 * fitted) + 5, dtype=np.int64)  # a larger core
    dev.fail["factor"] = [_lib.ERR_MEMORY]
    with pytest.raises(KKTSolveError):
        solver._factor_current(theta, 1.0)
    assert solver.memory_caps == 1
    assert solver.core_target >= fitted and solver.max_core_target >= fitted
    assert solver.core_target <= int(1.1 * fitted) + 5
