"""R2: the augmented MINRES fallback on the device (psipm_minres).

The reference answers a PCG breakdown or stagnation with preconditioned
MINRES on [diag(theta) A^T; A -delta I] [dx; q] = [r1; r2]
(psipm_spectral_preconditioner.py:583-637, 717-737).  Checked here: the
device result meets the reference's acceptance on its true residual
(recomputed on the host), and its direction agrees with the exact Newton
direction; the device-resident variant reproduces psipm_ipm_newton's
direction on the same system.
"""

import numpy as np
import pytest

from _helpers import lp_from, exact_direction, rel

pytestmark = pytest.mark.gpu


def augmented_residual(A, theta, delta, r1, r2, dx, dy):
    q = -dy
    res = np.concatenate([r1 - (theta * dx + A.T @ q), r2 - (A @ dx - delta * q)])
    return np.linalg.norm(res) / max(1.0, np.linalg.norm(np.concatenate([r1, r2])))


@pytest.mark.parametrize("call", [0, 3])
def test_minres_meets_the_reference_acceptance(call, golden):
    from psipm_b200.device import NormalEquationsDevice

    g = golden("random_m300")
    lp = lp_from(g)
    theta, delta, core = g[f"s{call}_theta"], float(g[f"s{call}_delta"]), g[f"s{call}_core"]
    r1, r2 = g[f"s{call}_r1"], g[f"s{call}_r2"]
    dev = NormalEquationsDevice(lp.A)
    try:
        dev.set_theta(theta, delta)
        dev.set_core(core)
        dev.factor(delta, 0)
        tol = 1e-8
        dx, dy, accepted, its, reported = dev.minres(r1, r2, tol, 400, 1e-6)
        assert accepted and its > 0
        host = augmented_residual(lp.A, theta, delta, r1, r2, dx, dy)
        assert host <= max(2 * tol, 1e-6)
        assert abs(host - reported) <= 1e-6 * max(host, 1e-300) + 1e-14
        ex_dx, ex_dy = exact_direction(lp.A, theta, delta, r1, r2)
        assert rel(dy, ex_dy) <= 1e-5 and rel(dx, ex_dx) <= 1e-5
    finally:
        dev.close()


def test_resident_minres_matches_newton():
    from psipm_b200 import synthetic
    from psipm_b200.device import NormalEquationsDevice

    lp = synthetic.random_lp(200, 600, seed=31)
    m, n = lp.A.shape
    rng = np.random.default_rng(2)
    pos = np.ones(n, bool)
    box = rng.uniform(size=n) < 0.3
    u = np.where(box, rng.uniform(1.0, 3.0, n), np.inf)
    x = np.where(box, 0.5 * np.where(box, u, 1.0), rng.uniform(0.1, 2.0, n))
    z, w = rng.uniform(0.1, 2.0, n), np.where(box, rng.uniform(0.1, 2.0, n), 0.0)
    y = rng.standard_normal(m)
    dev = NormalEquationsDevice(lp.A)
    try:
        dev.ipm_load(lp.c, lp.b, u, pos, box)
        dev.ipm_put(1, x, y, z, w)
        dev.ipm_copy(False)
        dev.ipm_residuals(1e-6, 1e-6)
        dev.ipm_theta(1e-6, 1e-6 / np.finfo(float).eps ** 2, 1e-6)
        dev.ipm_targets(0, 0.01)
        dev.set_core(dev.candidates)
        dev.factor(1e-6, 0)
        finite, res = dev.ipm_newton(False, 1e-12, 300)
        assert finite
        ref = dev.ipm_get(2)
        finite, accepted, its, rr = dev.ipm_minres(False, 1e-10, 400, 1e-6)
        assert finite and accepted
        got = dev.ipm_get(2)
        for a, b in zip(got, ref):
            assert rel(a, b) <= 1e-6
    finally:
        dev.close()
