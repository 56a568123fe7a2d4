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
