"""PS-IPM with the iterate resident in device memory.

The reference's outer loop (``psipm_solve`` / ``prox_eval``,
psipm_active_pool.py:2277-2788 and :1947-2271) keeps x, y, z, w, s, the
residuals and the directions in NumPy and calls the KKT solver across the
``factorize`` / ``solve`` boundary.  This driver takes the same decisions
with the same constants, but the vectors never leave the device: every O(n)
operation is one of the ``psipm_ipm_*`` kernels of the C ABI, and the host
only sees the scalars the loop branches on (step lengths, trial mu, residual
norms, outer KKT measures).  The KKT policy object is the same
``GpuSpectralStableColumnPreconditioner``; it receives ``RESIDENT`` instead
of a theta array and solves with ``solve_resident``.

The starting point (psipm_active_pool.py:4122-4304, the default legacy
projection) runs on the device as well: the policy factors theta = 1, the two
projections go straight into the device iterate (``solve_start``) and
``psipm_ipm_start`` forms the shifted start there.

Every sum the loop branches on adds block partials in a fixed order and the
preconditioner application accumulates through fixed-order slots, so a solve
takes the same trajectory, bit for bit, on every run.
"""

from __future__ import annotations

import math
import time
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from .kkt import RESIDENT, GpuSpectralStableColumnPreconditioner, KKTSolveError

EPS = float(np.finfo(np.float64).eps)


@dataclass
class Solution:
    """Result of a solve, with the field names of the reference's ``Solution``
    (psipm_active_pool.py:1875-1941) that this driver fills in."""

    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    w: np.ndarray
    status: str = "unknown"
    obj: float = np.nan
    outer_iter: int = 0
    inner_iter: int = 0
    time: float = 0.0
    t_fact: float = 0.0
    t_solve: float = 0.0
    res_p: float = np.nan
    res_d: float = np.nan
    mu: float = np.nan
    gap: float = np.nan
    history: list = field(default_factory=list)
    pcg_iterations: int = 0
    pcg_max_iterations: int = 0
    n_fact: int = 0
    n_solve: int = 0


def warm_start_point(lp, initial):
    """The reference's safeguards on a caller's starting point
    (psipm_active_pool.py:2527-2550): finite arrays of the LP's sizes; boxed x
    kept at least the box floors inside [0, u] (floors min(8 eps, u/4) and
    min(8 eps max(1, u), u/4)), nonnegative x at least 1e-12, z and w of
    bounded entries at least 1e-12; free x as given, z zero off the
    nonnegative entries and w zero off the boxed ones."""
    if len(initial) != 4:
        raise ValueError("initial must contain (x, y, z, w)")
    x, y, z, w = (np.asarray(v, dtype=float).copy() for v in initial)
    m, n = lp.A.shape
    if x.size != n or y.size != m or z.size != n or w.size != n:
        raise ValueError("warm-start dimensions do not match the LP")
    if not all(np.isfinite(v).all() for v in (x, y, z, w)):
        raise ValueError("warm start must be finite")
    pos, box = np.asarray(lp.pos, dtype=bool), np.asarray(lp.box, dtype=bool)
    lower = np.full(n, 1e-12)
    if box.any():
        ub = np.asarray(lp.u, dtype=float)[box]
        quarter = 0.25 * ub
        x_floor = np.minimum(8.0 * EPS, quarter)
        s_floor = np.minimum(8.0 * EPS * np.maximum(1.0, ub), quarter)
        lower[box] = x_floor
        x[box] = np.minimum(np.maximum(x[box], x_floor), ub - s_floor)
    x[pos] = np.maximum(x[pos], lower[pos])
    z[pos] = np.maximum(z[pos], 1e-12)
    w[box] = np.maximum(w[box], 1e-12)
    x[~pos] = np.asarray(initial[0], dtype=float)[~pos]
    z[~pos] = 0.0
    w[~box] = 0.0
    return x, y, z, w


def starting_point_resident(dev, kkt, n: int) -> np.ndarray:
    """Device starting point: factor theta = 1, delta = 1 through the KKT
    policy (the reference's ``solver.factorize(ones, 1.0)``), the two
    projections into the device iterate, then the shifts on the device.  Any
    failure of the factorisation or a projection starts from x = y = 0, as
    the reference's legacy start does (psipm_active_pool.py:4182-4187)."""
    solved = True
    try:
        kkt.factorize(np.ones(n), 1.0)
        kkt.solve_start(0)
        kkt.solve_start(1)
    except Exception:
        solved = False
    return dev.ipm_start(solved)


class _Norms:
    """Scalars of psipm_ipm_residuals: mu numerator and the residual norms."""

    def __init__(self, out: np.ndarray):
        self.comp = float(out[0])
        self.gp = math.sqrt(max(float(out[1]), 0.0))
        self.rp = math.sqrt(max(float(out[2]), 0.0))
        self.rd = math.sqrt(max(float(out[3]), 0.0))
        self.dxk = math.sqrt(max(float(out[4]), 0.0))
        self.dyk = math.sqrt(max(float(out[5]), 0.0))

    @property
    def res_n(self) -> float:  # psipm_active_pool.py:1990-1992
        return self.gp + self.rp


def prox_eval_resident(dev, kkt, npos_box, nbox, rho, delta, tol, maxit, pc, deadline=np.inf, tau=0.995):
    """One proximal sub-problem (psipm_active_pool.py:1947-2271) on the device.

    Starts from the device's centre (xk, yk, zk, wk) and leaves the result in
    the device's iterate.
    """
    dev.ipm_copy(False)  # x, y, z, w = centre; s = 1; box floors
    sigmamin, sigmamax = 0.05, 0.95
    alpha_x = alpha_z = 0.0
    reg_extra = 0.0
    retry, max_tries = 0, 50
    stalled = 0
    res_n_best = np.inf
    iters = 0
    status = 0
    r = _Norms(dev.ipm_residuals(rho, delta))
    mu = r.comp / npos_box if npos_box else 0.0
    res_n = r.res_n

    def bump(reg):
        return min(0.5, max(max(reg, 1e-12) * 10.0, tol))

    def newton(corrector: bool) -> bool:  # :2042-2056
        try:
            return kkt.solve_resident(corrector)
        except KKTSolveError:
            return False

    while iters < maxit:
        prox_move = min(1.0, r.dxk + r.dyk)
        if res_n < 1.0e4 * tol * prox_move:
            status = 1
            break
        if time.perf_counter() > deadline:
            status = 3
            break
        iters += 1
        theta_min = rho + reg_extra
        dev.ipm_theta(theta_min, theta_min / EPS ** 2, delta + reg_extra)
        try:
            kkt.set_ipm_context_norms(r.rd, r.rp, res_n, tol)
            kkt.observe(None, None, None, None, mu)
            kkt.factorize(RESIDENT, delta + reg_extra)
        except Exception:
            if retry < max_tries:
                iters -= 1
                retry += 1
                reg_extra = bump(reg_extra)
                continue
            status = 2
            break

        def failed_retry():
            nonlocal iters, retry, reg_extra
            if retry < max_tries:
                iters -= 1
                retry += 1
                reg_extra = bump(reg_extra)
                return True
            return False

        if pc == 1:
            sigma = 0.5 if iters == 1 else max(1 - alpha_x, 1 - alpha_z) ** 5
            sigma = min(max(sigma, sigmamin), sigmamax)
            dev.ipm_targets(0, sigma * mu)
            if not newton(False):
                if failed_retry():
                    continue
                status = 2
                break
        else:
            if pc == 2:
                dev.ipm_targets(0, 0.0)
            else:
                if iters > 1 or min(alpha_x, alpha_z) > 0.5:
                    mu_target, factor = 0.1 * mu, 0.05
                else:
                    mu_target, factor = 0.7 * mu, 0.1
                dev.ipm_targets(0, factor * mu_target)
            if not newton(False):
                if failed_retry():
                    continue
                status = 2
                break
            sx, sz = dev.ipm_steps()
            alpha_x, alpha_z = tau * sx, tau * sz
            if pc == 2:
                cm = dev.ipm_complementarity(alpha_x, alpha_z)
                mu_aff = np.float64(cm) / npos_box
                mu_t = (mu_aff / mu) ** 2 * mu_aff if mu > 0 else mu_aff
                dev.ipm_targets(1, float(mu_t))
                if not newton(True):
                    if failed_retry():
                        continue
                    status = 2
                    break
                best = None
                for beta in (1.0, 0.5, 0.25, 0.125, 0.0625, 0.0):
                    sx, sz = dev.ipm_steps(True, beta)
                    axb, azb = tau * sx, tau * sz
                    if axb <= 0.0 or azb <= 0.0:
                        continue
                    mub = float(np.float64(dev.ipm_complementarity(axb, azb, True, beta)) / npos_box)
                    if not np.isfinite(mub) or mub < 0.0:
                        continue
                    merit = mub / max(min(axb, azb), 1e-8)
                    if best is None or merit < best[0]:
                        best = (merit, beta)
                if best is None:
                    if failed_retry():
                        continue
                    status = 2
                    break
                dev.ipm_accept(best[1])
            else:
                K_c, bmin, bmax, delta_a = 10, 1e-3, 1e3, 0.2
                for _ in range(K_c):
                    ta_x = min(1.0, 1.5 * alpha_x + delta_a)
                    ta_z = min(1.0, 1.5 * alpha_z + delta_a)
                    dev.ipm_targets(2, ta_x, ta_z, mu_target, bmin, bmax)
                    if not newton(True):
                        break
                    sx, sz = dev.ipm_steps(True, 1.0)
                    a_xn, a_zn = tau * sx, tau * sz
                    if a_xn < 1.01 * alpha_x and a_zn < 1.01 * alpha_z:
                        break
                    alpha_x, alpha_z = a_xn, a_zn
                    dev.ipm_accept(1.0)
        retry = 0
        if npos_box:
            sx, sz = dev.ipm_steps()
            alpha_x, alpha_z = tau * sx, tau * sz
        else:
            alpha_x = alpha_z = 1.0
        dev.ipm_update(alpha_x, alpha_z)
        if reg_extra:
            reg_extra = 0.0 if reg_extra <= 1e-12 else reg_extra * 0.1
        r = _Norms(dev.ipm_residuals(rho, delta))
        if npos_box:
            mu = r.comp / npos_box
        res_n = r.res_n
        if res_n < 0.999 * res_n_best:
            res_n_best = res_n
            stalled = 0
        elif not np.isfinite(res_n):
            stalled += 3
        else:
            stalled += 1
        if stalled >= 5:
            break
    return dict(iters=iters, status=status, stalled=stalled)


def psipm_solve_resident(lp, kkt_solver, tol=1e-6, maxit=200, inner_maxit=100, pc=3, rho=None, delta=None,
                         rf=1.0, ppm_red=0.5, compl="gap", tau=0.995, diverge_tol=1e4,
                         time_limit=np.inf, max_outer: Optional[int] = None, initial=None) -> Solution:
    """Outer proximal loop (psipm_active_pool.py:2277-2788) on device-resident vectors.

    Arguments as the reference's ``psipm_solve`` with an external KKT solver
    (``max_outer``, not in the reference, stops after that many outer
    iterations; ``initial=(x, y, z, w)`` is the reference's warm start, taken
    through :func:`warm_start_point` instead of the computed starting point);
    ``kkt_solver`` must be a :class:`GpuSpectralStableColumnPreconditioner`.
    """
    warm = None if initial is None else warm_start_point(lp, initial)
    if not isinstance(kkt_solver, GpuSpectralStableColumnPreconditioner):
        raise TypeError("the device-resident loop needs a GpuSpectralStableColumnPreconditioner")
    A = lp.A
    c, b, u = lp.c, lp.b, lp.u
    m, n = A.shape
    npos, nbox = int(lp.pos.sum()), int(lp.box.sum())
    npos_box = npos + nbox
    normA = float(abs(A).sum(axis=1).max()) if A.nnz else 1.0
    if rho is None:
        rho = rf * max(tol / max(normA, 1e-16), 1e-8)
    if delta is None:
        delta = rho
    dp = 1.0 + float(np.abs(b).max(initial=0.0))
    dd = 1.0 + float(np.abs(c).max(initial=0.0))
    solver = kkt_solver
    if solver.A.shape != A.shape:
        raise ValueError("external KKT solver dimensions do not match the LP")
    dev = solver.dev
    tic = time.perf_counter()
    deadline = tic + time_limit
    dev.ipm_load(c, b, u, lp.pos, lp.box)
    solver.resident = True
    if warm is None:
        starting_point_resident(dev, solver, n)
        solver.h2d_bytes += 8 * n  # theta = 1
    else:
        dev.ipm_put(0, *warm)
        solver.h2d_bytes += 8 * (3 * n + m)
    dev.ipm_copy(True)  # centre = iterate
    solver.h2d_bytes += 8 * (2 * n + m) + 2 * n  # c, u, b, masks
    best_mu = np.inf
    sol = Solution(x=None, y=None, z=None, w=None)
    inner_tot = 0
    it = 0
    nrpi = nrdi = mu = gap = np.nan
    for it in range(1, maxit + 1):
        met = dev.ipm_metrics()  # box floors on the iterate, then the KKT measures
        nrpi, nrdi, cx, by, wu, comp = (float(v) for v in met)
        mu = comp / npos_box if npos_box else 0.0
        gap = abs(cx - (by - wu)) / (1.0 + abs(cx + lp.obj_const))
        sol.history.append(dict(outer=it, rp=nrpi / dp, rd=nrdi / dd, mu=mu, gap=gap, inner=inner_tot,
                                t=time.perf_counter() - tic))
        ok_c = (mu < tol) if compl == "mu" else (gap < tol) if compl == "gap" else (mu < tol or gap < tol)
        if nrpi / dp < tol and nrdi / dd < tol and ok_c:
            sol.status = "optimal"
            break
        if npos_box and mu > 0.0:
            if mu < best_mu:
                best_mu = mu
            elif best_mu > 0.0 and mu > diverge_tol * best_mu:
                sol.status = "diverged"
                break
        if time.perf_counter() > deadline:
            sol.status = "time-limit"
            break
        if max_outer is not None and it > max_outer:
            sol.status = "sample-limit"
            break
        info = prox_eval_resident(dev, solver, npos_box, nbox, rho, delta, ppm_red ** it, inner_maxit, pc,
                                  deadline, tau=tau)
        inner_tot += info["iters"]
        if info["status"] == 2:
            sol.status = "ill-conditioned"
            break
        dev.ipm_copy(True)  # centre = iterate
        if info["status"] == 3:
            sol.status = "time-limit"
            break
    else:
        sol.status = "max-iterations"
    sol.x, sol.y, sol.z, sol.w = dev.ipm_get(0)
    solver.d2h_bytes += 8 * (3 * n + m)
    sol.outer_iter = it
    sol.inner_iter = inner_tot
    sol.time = time.perf_counter() - tic
    sol.t_fact, sol.t_solve = solver.t_fact, solver.t_solve
    sol.res_p, sol.res_d, sol.mu = nrpi / dp, nrdi / dd, mu
    sol.gap = gap
    sol.obj = float(c @ sol.x) + lp.obj_const
    its = getattr(solver, "cg_iterations", [])
    if its:
        sol.pcg_iterations = int(sum(its))
        sol.pcg_max_iterations = int(max(its))
    sol.n_fact = int(getattr(solver, "n_fact", 0))
    sol.n_solve = int(getattr(solver, "n_solve", 0))
    return sol


def solve_standard(lp, tol=1e-8, device=0, precision=0, solver_options=None, **kwargs):
    """Public entry point: build the device KKT solver for ``lp`` and run the
    PS-IPM on device-resident vectors (the reference's
    ``solve_standard``, psipm_spectral_preconditioner.py:755-840, with the
    spectral stable-column preconditioner).  Returns ``(Solution, solver)``;
    the caller closes the solver."""
    opts = dict(solver_options or {})
    solver = GpuSpectralStableColumnPreconditioner(lp.A, protected=~lp.pos, device=device,
                                                   precision=precision, **opts)
    try:
        return psipm_solve_resident(lp, solver, tol=tol, **kwargs), solver
    except Exception:
        solver.close()
        raise
