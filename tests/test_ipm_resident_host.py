"""The device-resident PS-IPM driver (psipm_b200.ipm_device) on the CPU.

``FakeDevice`` answers the ``psipm_ipm_*`` calls with NumPy arithmetic that
follows the reference's prox_eval / psipm_solve (psipm_active_pool.py:
1947-2271, 2277-2788) line by line, so the resident driver must retrace the
host loop (the oracle's restatement of the reference's caller, which passes
theta, r1, r2, dx, dy across the KKT boundary) iteration for iteration.  Failures are injected
on the host, as in test_host_failures.py.
"""

import numpy as np
import pytest

from fake_device import FakeDevice
from oracle import ipm
from psipm_b200 import _lib, synthetic
from psipm_b200.ipm_device import psipm_solve_resident
from psipm_b200.kkt import GpuSpectralStableColumnPreconditioner

OPTS = dict(full_preconditioner_row_threshold=10)


def make(lp, dev):
    return GpuSpectralStableColumnPreconditioner(lp.A, protected=~lp.pos, dev=dev, **OPTS)


LPS = {
    "random": lambda: synthetic.random_lp(120, 360, seed=9),
    "grid": lambda: synthetic.grid_network(rows=6, cols=7, seed=3),
}


@pytest.mark.parametrize("name", sorted(LPS))
@pytest.mark.parametrize("pc", [1, 2, 3])
def test_resident_loop_retraces_host_loop(name, pc):
    lp = LPS[name]()
    host = ipm.psipm_solve(lp, make(lp, FakeDevice(lp.A)), tol=1e-8, pc=pc)
    solver = make(lp, FakeDevice(lp.A))
    res = psipm_solve_resident(lp, solver, tol=1e-8, pc=pc)
    assert host.status == "optimal"
    assert res.status == host.status
    assert res.outer_iter == host.outer_iter
    assert res.inner_iter == host.inner_iter
    assert abs(res.obj - host.obj) <= 1e-10 * max(1.0, abs(host.obj))
    assert res.res_p < 1e-8 and res.res_d < 1e-8
    assert np.allclose(res.x, host.x, rtol=1e-7, atol=1e-9)
    assert solver.lag_spectral_bounds and solver.n_fact == host.n_fact


def test_resident_factor_failure_retries():
    lp = LPS["grid"]()
    dev = FakeDevice(lp.A)
    solver = make(lp, dev)
    dev.fail["factor"] = [None, None, _lib.ERR_NOT_PD]
    sol = psipm_solve_resident(lp, solver, tol=1e-8)
    assert sol.status == "optimal"
    assert solver.stats["not_pd"] > 0


def test_resident_solve_failure_is_a_retry():
    lp = LPS["random"]()
    dev = FakeDevice(lp.A)
    solver = make(lp, dev)
    dev.fail["solve"] = [None, None, None, _lib.ERR_CUDA]  # start point (2), 1st predictor ok, then CUDA
    sol = psipm_solve_resident(lp, solver, tol=1e-8)
    assert sol.status == "optimal"
    assert solver.cg_failures >= 1


def test_resident_loop_needs_the_spectral_solver():
    lp = LPS["random"]()
    from psipm_b200.kkt import GpuStableActiveColumnPreconditioner

    plain = GpuStableActiveColumnPreconditioner(lp.A, protected=~lp.pos, dev=FakeDevice(lp.A), **OPTS)
    with pytest.raises(TypeError):
        psipm_solve_resident(lp, plain, tol=1e-8)


def test_warm_start_from_a_solution_converges_at_once():
    """initial=(x, y, z, w) (the reference's warm start, psipm_active_pool.py:
    2527-2550) from a converged solution: the same objective in a few outer
    iterations instead of the cold start's."""
    lp = LPS["random"]()
    cold = psipm_solve_resident(lp, make(lp, FakeDevice(lp.A)), tol=1e-8)
    assert cold.status == "optimal"
    warm = psipm_solve_resident(lp, make(lp, FakeDevice(lp.A)), tol=1e-8,
                                initial=(cold.x, cold.y, cold.z, cold.w))
    assert warm.status == "optimal"
    assert warm.outer_iter < cold.outer_iter
    assert abs(warm.obj - cold.obj) <= 1e-8 * max(1.0, abs(cold.obj))


def test_warm_start_safeguards():
    from psipm_b200.ipm_device import warm_start_point

    lp = synthetic.random_lp(20, 60, seed=4)
    rng = np.random.default_rng(0)
    n, m = lp.A.shape[1], lp.A.shape[0]
    lp.pos[:5] = False  # free columns
    lp.box[5:15] = True
    lp.u[5:15] = np.linspace(1e-17, 2.0, 10)
    lp.box[:5] = False
    x, y, z, w = rng.standard_normal(n), rng.standard_normal(m), rng.standard_normal(n), rng.standard_normal(n)
    x[5:15] = np.linspace(-1.0, 3.0, 10)
    xs, ys, zs, ws = warm_start_point(lp, (x, y, z, w))
    eps = np.finfo(float).eps
    ub = lp.u[5:15]
    x_floor = np.minimum(8 * eps, 0.25 * ub)
    s_floor = np.minimum(8 * eps * np.maximum(1.0, ub), 0.25 * ub)
    assert np.array_equal(xs[5:15], np.maximum(np.minimum(np.maximum(x[5:15], x_floor), ub - s_floor), x_floor))
    assert np.array_equal(xs[:5], x[:5]) and np.all(zs[:5] == 0.0) and np.all(ws[~lp.box] == 0.0)
    assert np.all(xs[lp.pos & ~lp.box] >= 1e-12) and np.all(zs[lp.pos] >= 1e-12) and np.all(ws[lp.box] >= 1e-12)
    assert np.array_equal(ys, y)
    with pytest.raises(ValueError):
        warm_start_point(lp, (x, y, z))
    with pytest.raises(ValueError):
        warm_start_point(lp, (x[:-1], y, z, w))
    bad = x.copy()
    bad[7] = np.nan
    with pytest.raises(ValueError):
        warm_start_point(lp, (bad, y, z, w))
