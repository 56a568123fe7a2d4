"""FP32 modes against the exact direction: FP32 factor / PCG with FP64
refinement (mode 1) and FP64 PCG around an FP32 preconditioner (mode 2).

Bars: with tolerance 1e-10 the refined direction is within 1e-8 of the
exact one (the same bar as FP64 mode at 1e-13 would give 1e-8); the FP32
preconditioner apply agrees with the FP64 one to 1e-4; a full PS-IPM solve
is optimal with objective within 1e-8 of the reference.
"""

import numpy as np
import pytest

from _helpers import NAMES, OPTIONS, exact_direction, lp_from, rel

pytestmark = pytest.mark.gpu


MODES = (1, 2)  # FP32_REFINED, FP32_PRECOND


def devices(lp, mode):
    from psipm_b200 import _lib
    from psipm_b200.device import NormalEquationsDevice

    return NormalEquationsDevice(lp.A, precision=_lib.FP64), NormalEquationsDevice(lp.A, precision=mode)


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("name", NAMES)
def test_fp32_refined_directions(name, mode, golden):
    g = golden(name)
    lp = lp_from(g)
    d64, d32 = devices(lp, mode)
    for i in range(min(6, int(g["n_solve_calls"]))):
        theta, delta = g[f"s{i}_theta"], float(g[f"s{i}_delta"])
        for d in (d64, d32):
            d.set_theta(theta, delta)
            d.set_core(g[f"s{i}_core"])
            d.factor(delta, 0)
        r = np.random.default_rng(i).standard_normal(lp.A.shape[0])
        assert rel(d32.apply(r), d64.apply(r)) <= 1e-4, i
        dx, res = d32.solve(g[f"s{i}_r1"], g[f"s{i}_r2"], 1e-10, 1000)
        dx_e, dy_e = exact_direction(lp.A, theta, delta, g[f"s{i}_r1"], g[f"s{i}_r2"])
        assert res.info == 0 and res.relative_residual <= 1e-10, (i, res.info, res.relative_residual)
        assert rel(res.x, dy_e) <= 1e-8, i
        assert rel(dx, dx_e) <= 1e-8, i
        if mode == 1:
            assert res.refinements >= 1


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("name", NAMES)
def test_fp32_refined_full_solve(name, mode, golden):
    from oracle import ipm as OI
    from psipm_b200 import _lib
    from psipm_b200.kkt import GpuSpectralStableColumnPreconditioner

    g = golden(name)
    lp = lp_from(g)
    solver = GpuSpectralStableColumnPreconditioner(lp.A, protected=~lp.pos, precision=mode, **OPTIONS)
    sol = OI.psipm_solve(lp, solver, tol=1e-8)
    assert sol.status == "optimal"
    ref = float(g["obj"])
    assert abs(sol.obj - ref) <= 1e-8 * abs(ref)
