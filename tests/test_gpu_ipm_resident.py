"""Device-resident PS-IPM kernels (psipm_ipm_*) against NumPy, and full solves.

Each kernel is checked against ``FakeDevice``'s NumPy model of the same call,
which restates the reference's prox_eval arithmetic
(psipm_active_pool.py:1947-2271): copies, floors, minima and maxima exactly;
sums to 1e-12 relative (the device adds block partials in no fixed order);
products that the device contracts into FMAs to a few ulps.  The full solves
run ``psipm_solve_resident`` on the golden fixtures and must reach the
reference's optimal objective.
"""

import numpy as np
import pytest

from _helpers import NAMES, OPTIONS, lp_from, normal_matrix, rel
from fake_device import FakeDevice

pytestmark = pytest.mark.gpu

EPS = float(np.finfo(float).eps)


@pytest.fixture(scope="module")
def case():
    from psipm_b200 import synthetic
    from psipm_b200.device import NormalEquationsDevice

    lp = synthetic.random_lp(200, 600, seed=31)
    rng = np.random.default_rng(7)
    n = lp.A.shape[1]
    kind = rng.integers(0, 6, n)  # 0-1 box, 2 free, 3-5 lower bound only
    box = kind <= 1
    pos = kind != 2
    u = np.where(box, rng.uniform(0.5, 3.0, n), np.inf)
    dev = NormalEquationsDevice(lp.A)
    fake = FakeDevice(lp.A)
    for d in (dev, fake):
        d.ipm_load(lp.c, lp.b, u, pos, box)
    yield lp, dev, fake, pos, box, u, rng
    dev.close()


def point(lp, rng, u, pos, box):
    m, n = lp.A.shape
    x = np.where(box, rng.uniform(0.05, 0.95, n) * np.where(box, u, 1.0), rng.uniform(0.1, 2.0, n))
    x = np.where(pos, x, rng.standard_normal(n))
    z = np.where(pos, rng.uniform(0.1, 2.0, n), 0.0)
    w = np.where(box, rng.uniform(0.1, 2.0, n), 0.0)
    return x, rng.standard_normal(m), z, w


def direction(lp, rng):
    m, n = lp.A.shape
    return rng.standard_normal(n), rng.standard_normal(m), rng.standard_normal(n), rng.standard_normal(n)


def load_state(dev, fake, lp, rng, u, pos, box):
    it, ce = point(lp, rng, u, pos, box), point(lp, rng, u, pos, box)
    for d in (dev, fake):
        d.ipm_put(1, *ce)
        d.ipm_put(0, *it)
        d.ipm_copy(False)


def test_put_get_round_trip(case):
    lp, dev, fake, pos, box, u, rng = case
    for which in range(4):
        v = direction(lp, rng)
        dev.ipm_put(which, *v)
        for a, b in zip(dev.ipm_get(which), v):
            assert np.array_equal(a, b)


def test_copy_and_box_floors_exact(case):
    lp, dev, fake, pos, box, u, rng = case
    ce = point(lp, rng, u, pos, box)
    ce[0][np.flatnonzero(box)[:5]] = 0.0  # below the floor
    for d in (dev, fake):
        d.ipm_put(1, *ce)
        d.ipm_copy(False)
    for a, b in zip(dev.ipm_get(0), fake.ipm_get(0)):
        assert np.array_equal(a, b)
    for d in (dev, fake):
        d.ipm_copy(True)
    for a, b in zip(dev.ipm_get(1), fake.ipm_get(1)):
        assert np.array_equal(a, b)


def test_residuals_match_numpy(case):
    lp, dev, fake, pos, box, u, rng = case
    load_state(dev, fake, lp, rng, u, pos, box)
    got, want = dev.ipm_residuals(1e-6, 2e-6), fake.ipm_residuals(1e-6, 2e-6)
    assert np.allclose(got, want, rtol=1e-12, atol=0.0), (got, want)


def test_metrics_match_numpy(case):
    lp, dev, fake, pos, box, u, rng = case
    load_state(dev, fake, lp, rng, u, pos, box)
    got, want = dev.ipm_metrics(), fake.ipm_metrics()
    # the maxima are exact given A x and A^T y, which the device sums in another order
    assert np.allclose(got, want, rtol=1e-12, atol=1e-300)


def test_theta_reaches_the_operator(case):
    lp, dev, fake, pos, box, u, rng = case
    load_state(dev, fake, lp, rng, u, pos, box)
    x, y, z, w = dev.ipm_get(0)
    x[np.flatnonzero(pos & ~box)[:3]] = 0.0  # z/x = inf -> the cap
    for d in (dev, fake):
        d.ipm_put(0, x, y, z, w)
    tmin, delta = 1e-6, 3e-7
    for d in (dev, fake):
        d.ipm_theta(tmin, tmin / EPS ** 2, delta)
    assert (fake.theta == tmin / EPS ** 2).sum() >= 3
    v = rng.standard_normal(lp.A.shape[0])
    H = normal_matrix(lp.A, fake.theta, delta)
    assert rel(dev.matvec(v), H @ v) <= 1e-13


def test_steps_complementarity_accept_update(case):
    lp, dev, fake, pos, box, u, rng = case
    load_state(dev, fake, lp, rng, u, pos, box)
    D, C = direction(lp, rng), direction(lp, rng)
    for d in (dev, fake):
        d.ipm_put(2, *D)
        d.ipm_put(3, *C)
    assert dev.ipm_steps() == fake.ipm_steps()
    for gamma in (1.0, 0.25):
        assert np.allclose(dev.ipm_steps(True, gamma), fake.ipm_steps(True, gamma), rtol=1e-14, atol=0.0)
        got = dev.ipm_complementarity(0.3, 0.2, True, gamma)
        want = fake.ipm_complementarity(0.3, 0.2, True, gamma)
        assert abs(got - want) <= 1e-12 * abs(want)
    assert abs(dev.ipm_complementarity(0.3, 0.2) - fake.ipm_complementarity(0.3, 0.2)) <= \
        1e-12 * abs(fake.ipm_complementarity(0.3, 0.2))
    for d in (dev, fake):
        d.ipm_accept(0.5)
    for a, b in zip(dev.ipm_get(2), fake.ipm_get(2)):
        assert np.allclose(a, b, rtol=4 * EPS, atol=4 * EPS)
    for d in (dev, fake):
        d.ipm_update(0.3, 0.2)
    for a, b in zip(dev.ipm_get(0), fake.ipm_get(0)):
        assert np.allclose(a, b, rtol=4 * EPS, atol=4 * EPS)


@pytest.mark.parametrize("kind", [0, 1, 2])
def test_newton_matches_exact_direction(case, kind):
    """Targets of each kind, then the Newton system; the PCG runs with the full
    candidate set as core, so its direction is checked against a direct solve."""
    lp, dev, fake, pos, box, u, rng = case
    load_state(dev, fake, lp, rng, u, pos, box)
    D = direction(lp, rng)
    for d in (dev, fake):
        d.ipm_put(2, *D)
        d.ipm_residuals(1e-6, 1e-6)
        d.ipm_theta(1e-6, 1e-6 / EPS ** 2, 1e-6)
    params = {0: (0.01,), 1: (0.02,), 2: (0.6, 0.7, 0.05, 1e-3, 1e3)}[kind]
    for d in (dev, fake):
        d.ipm_targets(kind, *params)
    dev.set_core(dev.candidates)
    dev.factor(1e-6, 0)
    corrector = kind != 0
    finite, res = dev.ipm_newton(corrector, 1e-10, 200)
    assert finite and res.relative_residual <= 1e-10
    x, _, z, w = fake.ipm_get(0)
    r1 = np.zeros(lp.A.shape[1]) if corrector else fake.rd.copy()
    r1[pos] += fake.rmz[pos] / x[pos]
    r1[box] -= fake.rmw[box] / fake.s[box]
    r2 = np.zeros(lp.A.shape[0]) if corrector else fake.rp
    theta = fake.theta
    H = normal_matrix(lp.A, theta, 1e-6)
    rhs = r2 - lp.A @ (r1 / theta)
    dx, dy, dz, dw = dev.ipm_get(3 if corrector else 2)
    # the reduced system holds to the PCG's residual, checked on the host ...
    assert np.linalg.norm(rhs - H @ dy) / max(1.0, np.linalg.norm(rhs)) <= 1e-10 * (1 + 1e-6)
    # ... and dx, dz, dw follow from dy by the back-substitution of newton().  For
    # dx the host's r1 stands in for the device's: both hold rd, whose A^T y is
    # summed in another order, and free columns (theta = theta_min) amplify that
    # rounding through the cancellation in (r1 + A^T dy) / theta.
    assert rel(dx, r1 / theta + (lp.A.T @ dy) / theta) <= 1e-9
    assert rel(dz, np.where(pos, (fake.rmz - z * dx) / x, 0.0)) <= 1e-12
    assert rel(dw, np.where(box, (fake.rmw + w * dx) / fake.s, 0.0)) <= 1e-12
    import scipy.sparse.linalg as spla

    assert rel(dy, spla.spsolve(H, rhs)) <= 1e-6


def test_lag_ratio_exact(case):
    lp, dev, fake, pos, box, u, rng = case
    n = lp.A.shape[1]
    t1, t2 = np.exp(rng.uniform(-5, 5, n)), np.exp(rng.uniform(-5, 5, n))
    dev.set_theta(t1, 1e-6)
    dev.lag_reference()
    dev.set_theta(t2, 1e-6)
    ratio = (1.0 / t2) / np.maximum(1.0 / t1, np.finfo(float).tiny)
    assert dev.lag_ratio() == (float(ratio.max()), float(ratio.min()))


@pytest.mark.parametrize("name", NAMES)
def test_resident_solve_reaches_reference_objective(name, golden):
    from psipm_b200.ipm_device import psipm_solve_resident
    from psipm_b200.kkt import GpuSpectralStableColumnPreconditioner

    g = golden(name)
    lp = lp_from(g)
    solver = GpuSpectralStableColumnPreconditioner(lp.A, protected=~lp.pos, **OPTIONS)
    try:
        sol = psipm_solve_resident(lp, solver, tol=1e-8)
    finally:
        solver.close()
    assert sol.status == "optimal"
    ref = float(g["obj"])
    assert abs(sol.obj - ref) <= 1e-8 * abs(ref)
    assert sol.res_p < 1e-8 and sol.res_d < 1e-8


@pytest.mark.parametrize("pc", [1, 2])
def test_resident_predictor_corrector_variants(pc, golden):
    from psipm_b200.ipm_device import psipm_solve_resident
    from psipm_b200.kkt import GpuSpectralStableColumnPreconditioner

    g = golden("grid_20x25")
    lp = lp_from(g)
    solver = GpuSpectralStableColumnPreconditioner(lp.A, protected=~lp.pos, **OPTIONS)
    try:
        sol = psipm_solve_resident(lp, solver, tol=1e-8, pc=pc)
    finally:
        solver.close()
    assert sol.status == "optimal"
    ref = float(g["obj"])
    assert abs(sol.obj - ref) <= 1e-7 * abs(ref)


@pytest.mark.parametrize("family", ["random", "grid", "cover"])
def test_device_starting_point_matches_the_oracle(family):
    """psipm_ipm_start against the oracle's arithmetic of the reference's start
    (psipm_active_pool.py:4190-4240) applied to the same two projections."""
    from oracle import ipm as OI
    from psipm_b200 import synthetic
    from psipm_b200.device import NormalEquationsDevice

    lp = {"random": lambda: synthetic.random_lp(300, 900, seed=3),
          "grid": lambda: synthetic.grid_network(12, 15, seed=4),
          "cover": lambda: synthetic.set_cover(200, 5000, seed=5)}[family]()
    m, n = lp.A.shape
    dev = NormalEquationsDevice(lp.A)
    try:
        dev.ipm_load(lp.c, lp.b, lp.u, lp.pos, lp.box)
        dev.set_theta(np.ones(n), 1.0)
        dev.set_core(dev.candidates[: min(dev.candidates.size, 2 * m)])
        dev.factor(1.0, 0)
        for which in (0, 1):
            finite, res = dev.ipm_start_solve(which, 1e-12, 500)
            assert finite and res.ok
        x0, y0, _, _ = dev.ipm_get(0)
        dev.ipm_start(True)
        x, y, z, w = dev.ipm_get(0)
        ibox = slice(None) if lp.box.all() else np.flatnonzero(lp.box)
        xr, yr, zr, wr = OI.start_from_projections(lp.A.T.tocsr(), lp.c, lp.u, lp, ibox, x0.copy(), y0.copy())
        for a, b_, name in ((x, xr, "x"), (y, yr, "y"), (z, zr, "z"), (w, wr, "w")):
            assert np.allclose(a, b_, rtol=1e-11, atol=1e-11 * max(1.0, np.abs(b_).max())), name
    finally:
        dev.close()
