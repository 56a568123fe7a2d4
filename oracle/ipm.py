"""Oracle restatement of the PS-IPM outer loop — test infrastructure.

Restates the caller of the inner solve so that a KKT solver object (the
oracle's or the GPU product's) can be driven exactly as the reference drives
it: ``psipm_solve`` (psipm_active_pool.py:2277-2788) with an external
``kkt_solver``, its inner loop ``prox_eval`` (:1947-2271), the IPX-style start
``_starting_point`` (:4122-4304, legacy projection) and the helpers
(:1831-1872).  Only the external-solver path is restated; the reference's
built-in KKT back-ends and its printing are out of scope.
"""

from __future__ import annotations

import time
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from .stable import KKTSolveError

EPS = float(np.finfo(np.float64).eps)
POS_FLOOR = 8.0 * EPS


def step_to_boundary(v, dv, idx) -> float:  # psipm_active_pool.py:1831-1837
    vv, dd = v[idx], dv[idx]
    neg = dd < 0.0
    if not neg.any():
        return 1.0
    return float(min(1.0, np.min(-vv[neg] / dd[neg])))


def all_or_idx(mask):  # :1840-1842
    return slice(None) if mask.all() else np.flatnonzero(mask)


def box_floors(u, ibox):  # :1845-1857
    ub = np.asarray(u[ibox], dtype=float)
    quarter = 0.25 * ub
    return np.minimum(POS_FLOOR, quarter), np.minimum(POS_FLOOR * np.maximum(1.0, ub), quarter)


def sync_box(x, s, u, ibox, x_floor, s_floor):  # :1860-1872
    x[ibox] = np.clip(x[ibox], x_floor, u[ibox] - s_floor)
    s[ibox] = np.maximum(u[ibox] - x[ibox], s_floor)


@dataclass
class Solution:
    """Subset of the reference ``Solution`` (psipm_active_pool.py:1875-1941)."""

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


def prox_eval(lp_c, A, At, b, u, ipos, ibox, npos_box, xk, yk, zk, wk, rho, delta, tol,
              maxit, pc, kkt, deadline=np.inf, nbox=0, tau=0.995):
    """One proximal sub-problem by predictor-corrector IPM (psipm_active_pool.py:1947-2271)."""
    n = A.shape[1]
    x, y, z, w = xk.copy(), yk.copy(), zk.copy(), wk.copy()
    x_floor, s_floor = box_floors(u, ibox) if nbox else (0.0, 0.0)
    s = np.ones(n)
    if nbox:
        sync_box(x, s, u, ibox, x_floor, s_floor)
    sigmamin, sigmamax = 0.05, 0.95
    alpha_x = alpha_z = 0.0
    reg_extra = 0.0
    retry, max_tries = 0, 50
    stalled = 0
    res_n_best = np.inf
    iters = 0
    status = 0
    mu = (x[ipos] @ z[ipos] + s[ibox] @ w[ibox]) / npos_box if npos_box else 0.0
    res_muz = np.zeros(n)
    res_muw = np.zeros(n)

    def residuals(x, y, z, w, s):
        rd = -(lp_c - At @ y - z + w + rho * (x - xk))
        rp = -(A @ x - b + delta * (y - yk))
        g = lp_c - At @ y + rho * (x - xk)
        proj = np.minimum(np.maximum(x[ipos] - g[ipos], 0.0), u[ipos])
        gp = g.copy()
        gp[ipos] = x[ipos] - proj
        rn = np.linalg.norm(gp) + np.linalg.norm(A @ x - b + delta * (y - yk))
        return rd, rp, rn

    res_d, res_p, res_n = residuals(x, y, z, w, s)

    def bump(reg):
        return min(0.5, max(max(reg, 1e-12) * 10.0, tol))

    while iters < maxit:
        prox_move = min(1.0, np.linalg.norm(x - xk) + np.linalg.norm(y - yk))
        if res_n < 1.0e4 * tol * prox_move:
            status = 1
            break
        if time.perf_counter() > deadline:
            status = 3
            break
        iters += 1
        theta_min = rho + reg_extra
        theta = np.full(n, theta_min)
        theta[ipos] += z[ipos] / x[ipos]
        theta[ibox] += w[ibox] / s[ibox]
        if not np.isfinite(theta).all():
            theta = np.where(np.isfinite(theta), theta, theta_min / EPS ** 2)
        np.clip(theta, theta_min, theta_min / EPS ** 2, out=theta)
        try:
            if hasattr(kkt, "set_ipm_context"):
                kkt.set_ipm_context(res_d=res_d, res_p=res_p, res_n=res_n, tol=tol)
            if hasattr(kkt, "observe"):
                kkt.observe(x, z, w, s, mu)
            kkt.factorize(theta, delta + reg_extra)
        except Exception:
            if retry < max_tries:
                iters -= 1
                retry += 1
                reg_extra = bump(reg_extra)
                continue
            status = 2
            break

        def newton(rd, rp, rmz, rmw):
            r1 = rd.copy()
            r1[ipos] += rmz[ipos] / x[ipos]
            r1[ibox] -= rmw[ibox] / s[ibox]
            try:
                dx, dy = kkt.solve(r1, rp)
            except (KKTSolveError, np.linalg.LinAlgError, FloatingPointError):
                return None
            except RuntimeError as exc:  # KKTSolveError of another module
                if type(exc).__name__ != "KKTSolveError":
                    raise
                return None
            if not (np.isfinite(dx).all() and np.isfinite(dy).all()):
                return None
            dz = np.zeros(n)
            dw = np.zeros(n)
            dz[ipos] = (rmz[ipos] - z[ipos] * dx[ipos]) / x[ipos]
            dw[ibox] = (rmw[ibox] + w[ibox] * dx[ibox]) / s[ibox]
            return dx, dy, dz, dw

        zero_p, zero_d = np.zeros(A.shape[0]), np.zeros(n)
        if pc == 1:
            sigma = 0.5 if iters == 1 else max(1 - alpha_x, 1 - alpha_z) ** 5
            sigma = min(max(sigma, sigmamin), sigmamax)
            res_muz[ipos] = sigma * mu - x[ipos] * z[ipos]
            res_muw[ibox] = sigma * mu - s[ibox] * w[ibox]
            out = newton(res_d, res_p, res_muz, res_muw)
            if out is None:
                if retry < max_tries:
                    iters -= 1
                    retry += 1
                    reg_extra = bump(reg_extra)
                    continue
                status = 2
                break
            dx, dy, dz, dw = out
        else:
            if pc == 2:
                res_muz[ipos] = -x[ipos] * z[ipos]
                res_muw[ibox] = -s[ibox] * w[ibox]
            else:
                if iters > 1 or min(alpha_x, alpha_z) > 0.5:
                    mu_target, factor = 0.1 * mu, 0.05
                else:
                    mu_target, factor = 0.7 * mu, 0.1
                res_muz[ipos] = -x[ipos] * z[ipos] + factor * mu_target
                res_muw[ibox] = -s[ibox] * w[ibox] + factor * mu_target
            out = newton(res_d, res_p, res_muz, res_muw)
            if out is None:
                if retry < max_tries:
                    iters -= 1
                    retry += 1
                    reg_extra = bump(reg_extra)
                    continue
                status = 2
                break
            dx, dy, dz, dw = out
            ds = -dx
            alpha_x = tau * min(step_to_boundary(x, dx, ipos), step_to_boundary(s, ds, ibox))
            alpha_z = tau * min(step_to_boundary(z, dz, ipos), step_to_boundary(w, dw, ibox))
            if pc == 2:
                cm = (x[ipos] + alpha_x * dx[ipos]) @ (z[ipos] + alpha_z * dz[ipos])
                cm += (s[ibox] + alpha_x * ds[ibox]) @ (w[ibox] + alpha_z * dw[ibox])
                mu_aff = cm / npos_box
                mu_t = (mu_aff / mu) ** 2 * mu_aff if mu > 0 else mu_aff
                res_muz[ipos] = mu_t - dx[ipos] * dz[ipos]
                res_muw[ibox] = mu_t - ds[ibox] * dw[ibox]
                outc = newton(zero_d, zero_p, res_muz, res_muw)
                if outc is None:
                    if retry < max_tries:
                        iters -= 1
                        retry += 1
                        reg_extra = bump(reg_extra)
                        continue
                    status = 2
                    break

                def trial_mu(dx_, dz_, dw_, ax_, az_):
                    ds_ = -dx_
                    val = (x[ipos] + ax_ * dx_[ipos]) @ (z[ipos] + az_ * dz_[ipos])
                    val += (s[ibox] + ax_ * ds_[ibox]) @ (w[ibox] + az_ * dw_[ibox])
                    return float(val / npos_box)

                best = None
                for beta in (1.0, 0.5, 0.25, 0.125, 0.0625, 0.0):
                    dxb = dx + beta * outc[0]
                    dyb = dy + beta * outc[1]
                    dzb = dz + beta * outc[2]
                    dwb = dw + beta * outc[3]
                    axb = tau * min(step_to_boundary(x, dxb, ipos), step_to_boundary(s, -dxb, ibox))
                    azb = tau * min(step_to_boundary(z, dzb, ipos), step_to_boundary(w, dwb, ibox))
                    if axb <= 0.0 or azb <= 0.0:
                        continue
                    mub = trial_mu(dxb, dzb, dwb, axb, azb)
                    if not np.isfinite(mub) or mub < 0.0:
                        continue
                    merit = mub / max(min(axb, azb), 1e-8)
                    if best is None or merit < best[0]:
                        best = (merit, beta, dxb, dyb, dzb, dwb)
                if best is None:
                    if retry < max_tries:
                        iters -= 1
                        retry += 1
                        reg_extra = bump(reg_extra)
                        continue
                    status = 2
                    break
                _, beta, dx, dy, dz, dw = best
            else:
                K_c, bmin, bmax, delta_a = 10, 1e-3, 1e3, 0.2
                for _ in range(K_c):
                    ta_x = min(1.0, 1.5 * alpha_x + delta_a)
                    ta_z = min(1.0, 1.5 * alpha_z + delta_a)
                    xt = x + ta_x * dx
                    zt = z + ta_z * dz
                    st = s - ta_x * dx
                    wt = w + ta_z * dw
                    for (a_, b_, tgt, idx) in ((xt, zt, res_muz, ipos), (st, wt, res_muw, ibox)):
                        prod = a_[idx] * b_[idx]
                        corr = np.clip(prod, bmin * mu_target, bmax * mu_target) - prod
                        corr = np.clip(corr, -bmax * mu_target, 2 * bmax * mu_target)
                        tgt[idx] = corr
                    outc = newton(zero_d, zero_p, res_muz, res_muw)
                    if outc is None:
                        break
                    dxt = dx + outc[0]
                    dyt = dy + outc[1]
                    dzt = dz + outc[2]
                    dwt = dw + outc[3]
                    a_xn = tau * min(step_to_boundary(x, dxt, ipos), step_to_boundary(s, -dxt, ibox))
                    a_zn = tau * min(step_to_boundary(z, dzt, ipos), step_to_boundary(w, dwt, ibox))
                    if a_xn < 1.01 * alpha_x and a_zn < 1.01 * alpha_z:
                        break
                    alpha_x, alpha_z = a_xn, a_zn
                    dx, dy, dz, dw = dxt, dyt, dzt, dwt
        retry = 0
        if npos_box:
            ds = -dx
            alpha_x = tau * min(step_to_boundary(x, dx, ipos), step_to_boundary(s, ds, ibox))
            alpha_z = tau * min(step_to_boundary(z, dz, ipos), step_to_boundary(w, dw, ibox))
        else:
            alpha_x = alpha_z = 1.0
        x += alpha_x * dx
        y += alpha_z * dy
        z += alpha_z * dz
        w += alpha_z * dw
        if nbox:
            sync_box(x, s, u, ibox, x_floor, s_floor)
        if reg_extra:
            reg_extra = 0.0 if reg_extra <= 1e-12 else reg_extra * 0.1
        if npos_box:
            mu = (x[ipos] @ z[ipos] + s[ibox] @ w[ibox]) / npos_box
        res_d, res_p, res_n = residuals(x, y, z, w, s)
        if res_n < 0.999 * res_n_best:
            res_n_best = res_n
            stalled = 0
        elif not np.isfinite(res_n):
            stalled += 3
        else:
            stalled += 1
        if stalled >= 5:
            break
    return x, y, z, w, dict(iters=iters, status=status, stalled=stalled)


def starting_point(A, At, b, c, u, lp, ipos, ibox, solver):
    """IPX-style start, legacy projection, exact startup (psipm_active_pool.py:4122-4304)."""
    m, n = A.shape
    ones_n = np.ones(n)
    zeros_n = np.zeros(n)
    pos, box = lp.pos, lp.box
    lower_only = pos & ~box
    try:
        solver.factorize(ones_n, 1.0)
        x = At @ solver.solve(zeros_n, b)[1]
        y = solver.solve(zeros_n, A @ c)[1]
    except Exception:
        x = zeros_n.copy()
        y = np.zeros(m)
    return start_from_projections(At, c, u, lp, ibox, x, y)


def start_from_projections(At, c, u, lp, ibox, x, y):
    """The starting point's arithmetic after the two projections x = A' dy_b and
    y = dy_c (psipm_active_pool.py:4190-4240)."""
    n, m = x.size, y.size
    zeros_n = np.zeros(n)
    pos, box = lp.pos, lp.box
    lower_only = pos & ~box
    if not np.isfinite(x).all():
        x = zeros_n.copy()
    if not np.isfinite(y).all():
        y = np.zeros(m)
    xl = np.zeros(n)
    xu = np.zeros(n)
    if pos.any():
        xl[pos] = x[pos]
    if box.any():
        xu[box] = u[box] - x[box]
    xinfeas = 0.0
    if pos.any():
        xinfeas = max(xinfeas, -float(np.min(xl[pos], initial=0.0)))
    if box.any():
        xinfeas = max(xinfeas, -float(np.min(xu[box], initial=0.0)))
    xshift1 = 1.0 + 1.5 * xinfeas
    if pos.any():
        xl[pos] += xshift1
    if box.any():
        xu[box] += xshift1
    cnorm = float(np.linalg.norm(c))
    if cnorm > 0.0:
        r = c - At @ y
        if float(np.linalg.norm(r)) < 0.05 * cnorm:
            y *= 0.95
            r = c - At @ y
    else:
        r = zeros_n.copy()
    z = np.zeros(n)
    w = np.zeros(n)
    if cnorm == 0.0:
        z[pos] = 1.0
        w[box] = 1.0
    else:
        z[lower_only] = r[lower_only]
        if box.any():
            z[box] = 0.5 * r[box]
            w[box] = -0.5 * r[box]
        zinfeas = 0.0
        if pos.any():
            zinfeas = max(zinfeas, -float(np.min(z[pos], initial=0.0)))
        if box.any():
            zinfeas = max(zinfeas, -float(np.min(w[box], initial=0.0)))
        zshift1 = 1.0 + 1.5 * zinfeas
        z[pos] += zshift1
        w[box] += zshift1
    xsum = zsum = mu0 = 1.0
    if pos.any():
        xsum += float(np.sum(xl[pos]))
        zsum += float(np.sum(z[pos]))
        mu0 += float(xl[pos] @ z[pos])
    if box.any():
        xsum += float(np.sum(xu[box]))
        zsum += float(np.sum(w[box]))
        mu0 += float(xu[box] @ w[box])
    xshift2 = 0.5 * mu0 / zsum if zsum > 0.0 else 0.0
    zshift2 = 0.5 * mu0 / xsum if xsum > 0.0 else 0.0
    if np.isfinite(xshift2) and xshift2 > 0.0:
        xl[pos] += xshift2
        xu[box] += xshift2
    if np.isfinite(zshift2) and zshift2 > 0.0:
        z[pos] += zshift2
        w[box] += zshift2
    if lower_only.any():
        x[lower_only] = np.maximum(xl[lower_only], 1e-12)
    if box.any():
        denom = xl[box] + xu[box]
        xb = np.where(denom > 0.0, u[box] * xl[box] / denom, 0.5 * u[box])
        x_floor, s_floor = box_floors(u, ibox)
        x[box] = np.clip(xb, x_floor, u[box] - s_floor)
    return x, y, z, w


def kkt_metrics(lp, x, y, z, w, npos_box, ipos, ibox, x_floor, s_floor):
    """Unregularised KKT measures of the outer loop (psipm_active_pool.py:2561-2599)."""
    A, b, c, u = lp.A, lp.b, lp.c, lp.u
    n = A.shape[1]
    rp = b - A @ x
    rd = c - A.T @ y - z + w
    s = np.ones(n)
    if lp.box.any():
        sync_box(x, s, u, ibox, x_floor, s_floor)
    mu = (x[ipos] @ z[ipos] + s[ibox] @ w[ibox]) / npos_box if npos_box else 0.0
    dp = 1.0 + float(np.abs(b).max(initial=0.0))
    dd = 1.0 + float(np.abs(c).max(initial=0.0))
    cx = float(c @ x)
    gap = abs(cx - (float(b @ y) - float(w[ibox] @ u[ibox]))) / (1.0 + abs(cx + lp.obj_const))
    return float(np.abs(rp).max(initial=0.0)) / dp, float(np.abs(rd).max(initial=0.0)) / dd, mu, gap


def psipm_solve(lp, kkt_solver, tol=1e-6, maxit=200, inner_maxit=100, pc=3, rho=None, delta=None,
                rf=1.0, ppm_red=0.5, compl="gap", tau=0.995, diverge_tol=1e4,
                time_limit=np.inf, max_outer: Optional[int] = None) -> Solution:
    """Outer proximal loop with an external KKT solver (psipm_active_pool.py:2277-2788).

    ``max_outer`` (not in the reference) stops after that many outer
    iterations; it bounds CPU-baseline samples and is ``None`` otherwise.
    """
    A = lp.A
    At = A.T.tocsr()
    c, b, u = lp.c, lp.b, lp.u
    m, n = A.shape
    ipos = all_or_idx(lp.pos)
    ibox = all_or_idx(lp.box)
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
    if getattr(solver, "A", A).shape != A.shape:
        raise ValueError("external KKT solver dimensions do not match the LP")
    x_floor, s_floor = box_floors(u, ibox) if nbox else (0.0, 0.0)
    tic = time.perf_counter()
    deadline = tic + time_limit
    x, y, z, w = starting_point(A, At, b, c, u, lp, ipos, ibox, solver)
    xk, yk, zk, wk = x.copy(), y.copy(), z.copy(), w.copy()
    best_mu = np.inf
    sol = Solution(x=x, y=y, z=z, w=w)
    inner_tot = 0
    it = 0
    for it in range(1, maxit + 1):
        rp = b - A @ x
        rd = c - At @ y - z + w
        s = np.ones(n)
        if nbox:
            sync_box(x, s, u, ibox, x_floor, s_floor)
        mu = (x[ipos] @ z[ipos] + s[ibox] @ w[ibox]) / npos_box if npos_box else 0.0
        nrpi = float(np.abs(rp).max(initial=0.0))
        nrdi = float(np.abs(rd).max(initial=0.0))
        cx = float(c @ x)
        gap = abs(cx - (float(b @ y) - float(w[ibox] @ u[ibox]))) / (1.0 + abs(cx + lp.obj_const))
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
        x, y, z, w, info = prox_eval(c, A, At, b, u, ipos, ibox, npos_box, xk, yk, zk, wk, rho, delta,
                                     ppm_red ** it, inner_maxit, pc, solver, deadline, nbox=nbox, tau=tau)
        inner_tot += info["iters"]
        if info["status"] == 2:
            sol.status = "ill-conditioned"
            break
        if info["status"] == 3:
            sol.status = "time-limit"
            xk, yk, zk, wk = x.copy(), y.copy(), z.copy(), w.copy()
            break
        xk, yk, zk, wk = x.copy(), y.copy(), z.copy(), w.copy()
    else:
        sol.status = "max-iterations"
    sol.x, sol.y, sol.z, sol.w = x, y, z, w
    sol.outer_iter = it
    sol.inner_iter = inner_tot
    sol.time = time.perf_counter() - tic
    sol.t_fact, sol.t_solve = solver.t_fact, solver.t_solve
    sol.res_p, sol.res_d, sol.mu = nrpi / dp, nrdi / dd, mu
    sol.gap = gap
    sol.obj = float(c @ x) + lp.obj_const
    its = getattr(solver, "cg_iterations", [])
    if its:
        sol.pcg_iterations = int(sum(its))
        sol.pcg_max_iterations = int(max(its))
    sol.n_fact = int(getattr(solver, "n_fact", 0))
    sol.n_solve = int(getattr(solver, "n_solve", 0))
    return sol
