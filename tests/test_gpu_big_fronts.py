"""The multi-CTA big-front path on small problems.

Fronts with more than PSIPM_BIG_FRONT rows are factored by the blocked
multi-CTA kernels (potrf / trsm / syrk tiles, then G = [I; L21] L11^{-1} by
column blocks) and supernodes with at least PSIPM_BIG_SOLVE columns use the
split triangular solve.  The golden problems are too small to reach the
defaults (192 and 96), so these tests lower both thresholds through the
environment, which the library reads at every symbolic analysis, and put the
defaults back afterwards.  Bars as in test_gpu_parity.py: P^{-1} r within
1e-9 of a sparse direct solve, full solves optimal at the reference objective.
"""

import os

import numpy as np
import pytest
import scipy.sparse.linalg as spla

from _helpers import NAMES, OPTIONS, lp_from, rel

pytestmark = pytest.mark.gpu

DEFAULTS = {"PSIPM_BIG_FRONT": "192", "PSIPM_BIG_SOLVE": "96"}


@pytest.fixture
def big_path():
    old = {k: os.environ.get(k) for k in DEFAULTS}
    os.environ["PSIPM_BIG_FRONT"] = "8"
    os.environ["PSIPM_BIG_SOLVE"] = "4"
    yield
    for k, v in DEFAULTS.items():  # the library keeps the last values it read
        os.environ[k] = v
    from psipm_b200 import synthetic
    from psipm_b200.device import NormalEquationsDevice

    lp = synthetic.random_lp(20, 60, seed=1)
    dev = NormalEquationsDevice(lp.A)
    dev.set_theta(np.ones(60), 1.0)
    dev.set_core(dev.candidates)
    dev.factor(1.0, 0)  # one analysis with the defaults restores them
    dev.close()
    for k, v in old.items():
        if v is None:
            os.environ.pop(k, None)
        else:
            os.environ[k] = v


@pytest.mark.parametrize("name", NAMES)
def test_big_front_apply_is_inverse(name, golden, big_path):
    from oracle import stable as OS
    from psipm_b200.device import NormalEquationsDevice

    g = golden(name)
    lp = lp_from(g)
    dev = NormalEquationsDevice(lp.A)
    for i in (0, 4):
        theta, delta, core = g[f"s{i}_theta"], float(g[f"s{i}_delta"]), g[f"s{i}_core"]
        dev.set_theta(theta, delta)
        dev.set_core(core)
        shift, info = dev.factor(delta, 0)
        assert shift == 0
        assert info.max_front > 8, "the test must reach the big-front path"
        orc = OS.StableOracle(lp.A, protected=~lp.pos, matching_backbone=False, **OPTIONS)
        orc._weights = 1.0 / theta
        orc.core = core
        P = orc._assemble(theta, delta)
        r = np.random.default_rng(i).standard_normal(lp.A.shape[0])
        assert rel(dev.apply(r), spla.spsolve(P, r)) <= 1e-9, f"call {i}"
    dev.close()


@pytest.mark.parametrize("precision", [0, 2])
def test_big_front_full_solve(precision, golden, big_path):
    from psipm_b200.ipm_device import psipm_solve_resident
    from psipm_b200.kkt import GpuSpectralStableColumnPreconditioner

    g = golden("random_m300")
    lp = lp_from(g)
    solver = GpuSpectralStableColumnPreconditioner(lp.A, protected=~lp.pos, precision=precision, **OPTIONS)
    try:
        sol = psipm_solve_resident(lp, solver, tol=1e-8)
    finally:
        solver.close()
    assert sol.status == "optimal"
    ref = float(g["obj"])
    assert abs(sol.obj - ref) <= 1e-8 * abs(ref)


def test_multi_panel_fronts_apply_is_inverse():
    """A 60x80 network LP with every candidate column in the core: P equals H,
    and the top fronts have ~1,100 pivot columns, so the blocked factor runs
    many 64-column steps with their trailing updates and the column-block G
    computation many steps of its own."""
    from _helpers import normal_matrix
    from psipm_b200 import synthetic
    from psipm_b200.device import NormalEquationsDevice

    lp = synthetic.grid_network(60, 80, seed=1000)
    n = lp.A.shape[1]
    theta = np.exp(np.random.default_rng(3).uniform(-4, 4, n))
    delta = 1e-6
    dev = NormalEquationsDevice(lp.A)
    try:
        dev.set_theta(theta, delta)
        dev.set_core(dev.candidates)
        shift, info = dev.factor(delta, 0)
        assert shift == 0
        assert info.max_front > 512, "the test must reach fronts of many column blocks"
        H = normal_matrix(lp.A, theta, delta)
        for seed in range(2):
            r = np.random.default_rng(seed).standard_normal(lp.A.shape[0])
            assert rel(dev.apply(r), spla.spsolve(H, r)) <= 1e-9
    finally:
        dev.close()
