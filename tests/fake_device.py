"""A CPU stand-in for ``NormalEquationsDevice`` — test infrastructure.

It answers the same method calls with the oracle's NumPy arithmetic, so the
host-side policy of ``psipm_b200.kkt`` and the device-resident IPM driver
``psipm_b200.ipm_device`` can run without a GPU, and it can be told to fail a given
call with a library status code (host-side fault injection: no device is
involved, nothing is made to fault).
"""

from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from oracle import stable as OS
from psipm_b200 import _lib
from psipm_b200.device import DeviceError, PcgResult

EPS = float(np.finfo(float).eps)


class FakeDevice:
    def __init__(self, A):
        A = sp.csc_matrix(A)
        A.sort_indices()
        self.A = A
        self.At = A.T.tocsr()
        self.m, self.n = A.shape
        self.candidates = np.flatnonzero(np.diff(A.indptr) >= 2).astype(np.int64)
        self.A2 = sp.csc_matrix((np.square(A.data), A.indices, A.indptr), shape=A.shape)
        counts = np.diff(A.indptr)[self.candidates].astype(float)
        self.burden = 0.5 * counts * np.maximum(counts - 1.0, 0.0)
        self.core = np.empty(0, dtype=np.int64)
        self.theta = None
        self.delta = 0.0
        self._scores = None
        self._lu = None
        self.fail = {}  # method name -> list of statuses to return on successive calls
        self.calls = {}
        self.kernel_launches = 0

    # -- fault injection ---------------------------------------------------
    def _maybe_fail(self, name):
        self.calls[name] = self.calls.get(name, 0) + 1
        queue = self.fail.get(name)
        if queue:
            status = queue.pop(0)
            if status is not None:
                raise DeviceError(status, f"injected failure of {name}")

    # -- NormalEquationsDevice interface --------------------------------------
    def set_theta(self, theta, delta):
        self._maybe_fail("set_theta")
        self.theta = np.asarray(theta, dtype=float).copy()
        self.delta = float(delta)
        self.w = 1.0 / self.theta

    def scores(self, fill_weight, want=True, want_diag=False):
        self._maybe_fail("scores")
        diag = np.asarray(self.A2 @ self.w).ravel()
        inv = 1.0 / np.maximum(diag + max(self.delta, OS.TINY), OS.TINY)
        lev = self.w[self.candidates] * np.asarray(self.A2[:, self.candidates].T @ inv).ravel()
        self._scores = lev / (1.0 + fill_weight * self.burden)
        return (self._scores.copy() if want else None), (diag if want_diag else None)

    def set_core(self, core):
        self.core = np.asarray(core, dtype=np.int64).copy()

    def tie_info(self):
        return dict(straddles=0, tied=0, slots=0, selections=0)

    def set_deterministic(self, on):
        self.deterministic = bool(on)

    def get_theta(self):
        return self.theta.copy()

    def mlp_features(self, mu):
        from oracle import mlp as OM

        flags = np.isin(self.candidates, self.core).astype(float)
        return OM.features(self.A, self.candidates, self.theta, self._scores, flags, mu).astype(np.float32)

    def mlp_scores(self, weights_bf16, biases, mu, keep=0):
        from oracle import mlp as OM

        w = (np.asarray(weights_bf16, dtype=np.uint16).astype(np.uint32) << 16).view(np.float32)
        out = OM.forward(np.concatenate([w, np.asarray(biases, dtype=np.float32)]), self.mlp_features(mu))
        scores = out[:, 0].copy()
        if 0 < keep < scores.size:
            allowed = np.zeros(scores.size, dtype=bool)
            allowed[OS.top_k(self._scores, keep)] = True
            scores[~allowed] = -np.inf
        self._scores = scores
        return float(out[:, 1].mean())

    def refresh_core(self, target, retention, stable, mandatory_local):
        self._maybe_fail("refresh_core")
        scores = self._scores
        nc = self.candidates.size
        target = min(int(target), nc)
        old = self.core
        parts = [np.asarray(mandatory_local, dtype=np.int64)] if len(mandatory_local) else []
        if stable and old.size and target:
            old_local = np.searchsorted(self.candidates, old)
            keep = min(old.size, max(0, int(np.floor(retention * target))))
            if keep:
                parts.append(old_local[OS.top_k(scores[old_local], keep)])
        fixed = np.unique(np.concatenate(parts)) if parts else np.empty(0, dtype=np.int64)
        mand = np.asarray(mandatory_local, dtype=np.int64)
        if fixed.size > target:
            if mand.size >= target:
                fixed = mand[:target]
            else:
                optional = fixed[~np.isin(fixed, mand)]
                fixed = np.concatenate([mand, optional[OS.top_k(scores[optional], target - mand.size)]])
        remaining = target - fixed.size
        if remaining > 0:
            avail = scores.copy()
            avail[fixed] = -np.inf
            fixed = np.concatenate([fixed, OS.top_k(avail, remaining)])
        new = np.sort(self.candidates[np.unique(fixed)])
        retained = (np.intersect1d(old, new).size / max(1, old.size)) if old.size else 1.0
        self.core = new
        return new.copy(), float(retained)

    def factor(self, delta, start_shift=0):
        self._maybe_fail("factor")
        self.delta = float(delta)
        Ac = self.A[:, self.core]
        P = OS.column_weighted_normal(sp.csc_matrix(Ac), self.w[self.core])
        diag_full = np.asarray(self.A2 @ self.w).ravel()
        diag_core = np.asarray(self.A2[:, self.core] @ self.w[self.core]).ravel()
        P = (P + sp.diags(np.maximum(diag_full - diag_core, 0.0) + delta)).tocsc()
        self._lu = spla.splu(P)

        class Info:
            symbolic_analyses = 1
            nnz_factor = int(self._lu.L.nnz)
            factor_seconds = 0.0

        return int(start_shift), Info()

    def _H(self, v):
        return self.A @ (self.w * (self.At @ v)) + self.delta * v

    def apply(self, r):
        return self._lu.solve(np.asarray(r, dtype=float))

    def matvec(self, v):
        return self._H(np.asarray(v, dtype=float))

    def set_pcg_budget(self, seconds):
        self.pcg_budget = float(seconds)

    def solve(self, r1, r2, tol, maxit, variant=_lib.PCG_SPECTRAL, replacement=100, gap_tolerance=0.1,
              want_residual=False):
        self._maybe_fail("solve")
        w1 = r1 / self.theta
        rhs = r2 - self.A @ w1
        scale = max(1.0, np.linalg.norm(rhs))
        x = self.apply(rhs)
        r = rhs - self._H(x)
        z = self.apply(r)
        p = z.copy()
        rz = r @ z
        alphas, betas, history = [], [], [np.linalg.norm(r) / scale]
        it = 0
        info = 0 if history[0] <= tol else maxit
        while info > 0 and it < maxit:
            q = self._H(p)
            alpha = rz / (p @ q)
            x += alpha * p
            r -= alpha * q
            it += 1
            alphas.append(alpha)
            if np.linalg.norm(r) / scale <= tol:
                info = 0
                break
            z = self.apply(r)
            rz_new = r @ z
            betas.append(rz_new / rz)
            p = z + betas[-1] * p
            rz = rz_new
        rel = np.linalg.norm(rhs - self._H(x)) / scale
        history.append(rel)
        dx = w1 + (self.At @ x) / self.theta
        res = PcgResult(x=x, info=info, iterations=it, matvecs=it + 2, replacements=0, residual_checks=1,
                        relative_residual=float(rel), ok=info == 0, alphas=np.array(alphas),
                        betas=np.array(betas), history=np.array(history), residual=None, seconds=0.0)
        forced = self.fail.get("solve_info")
        if forced:
            res.info = forced.pop(0)
            res.relative_residual = 1.0
        return dx, res

    # -- MINRES fallback (psipm_minres): the reference's _minres with SciPy ----
    def minres(self, r1, r2, tol, maxit, fail_tol):
        self._maybe_fail("minres")
        n, m = self.n, self.m

        def matvec(v):
            return np.concatenate([self.theta * v[:n] + self.At @ v[n:], self.A @ v[:n] - self.delta * v[n:]])

        def precondition(v):
            return np.concatenate([v[:n] / self.theta, self.apply(v[n:])])

        K = spla.LinearOperator((n + m, n + m), matvec=matvec, dtype=float)
        M = spla.LinearOperator((n + m, n + m), matvec=precondition, dtype=float)
        rhs = np.concatenate([r1, r2])
        scale = max(1.0, float(np.linalg.norm(rhs)))
        target = max(2.0 * tol, fail_tol)
        x = np.zeros(n + m)
        its = [0]
        for _ in range(3):
            cr = rhs - matvec(x)
            if np.linalg.norm(cr) / scale <= target:
                break
            corr, info = spla.minres(K, cr, M=M, rtol=max(EPS, min(tol, 1e-8)), maxiter=maxit,
                                     callback=lambda _: its.__setitem__(0, its[0] + 1))
            x += corr
            if info < 0:
                break
        rel = float(np.linalg.norm(rhs - matvec(x)) / scale)
        return x[:n].copy(), -x[n:], bool(np.isfinite(rel) and rel <= target), its[0], rel

    def ipm_minres(self, corrector, tol, maxit, fail_tol):
        x, _, z, w = self.sets[0]
        r1 = np.zeros(self.n) if corrector else self.rd.copy()
        r1[self.pos] += self.rmz[self.pos] / x[self.pos]
        r1[self.box] -= self.rmw[self.box] / self.s[self.box]
        r2 = np.zeros(self.m) if corrector else self.rp
        dx, dy, accepted, its, rel = self.minres(r1, r2, tol, maxit, fail_tol)
        dz = np.where(self.pos, (self.rmz - z * dx) / x, 0.0)
        dw = np.where(self.box, (self.rmw + w * dx) / self.s, 0.0)
        self.sets[3 if corrector else 2] = [dx, dy, dz, dw]
        return all(np.isfinite(v).all() for v in (dx, dy, dz, dw)), accepted, its, rel

    # -- device-resident IPM vectors (psipm_ipm_*), in NumPy -----------------
    def ipm_load(self, c, b, u, pos, box):
        self.c, self.b, self.u = (np.array(v, dtype=float) for v in (c, b, u))
        self.pos = np.asarray(pos, dtype=bool).copy()
        self.box = np.asarray(box, dtype=bool).copy()
        n, m = self.n, self.m
        self.sets = [[np.zeros(n), np.zeros(m), np.zeros(n), np.zeros(n)] for _ in range(4)]
        self.s = np.ones(n)
        self.rd, self.rp = np.zeros(n), np.zeros(m)
        self.rmz, self.rmw = np.zeros(n), np.zeros(n)
        self.wref = None

    def ipm_start_solve(self, which, tol, maxit, variant=_lib.PCG_SPECTRAL, replacement=100, gap_tolerance=0.1):
        r2 = self.b if which == 0 else self.A @ self.c
        dx, res = self.solve(np.zeros(self.n), r2, tol, maxit, variant, replacement, gap_tolerance)
        if which == 0:
            self.sets[0][0] = self.At @ res.x
        else:
            self.sets[0][1] = res.x.copy()
        return bool(np.isfinite(dx).all() and np.isfinite(res.x).all()), res

    def ipm_start(self, solved):
        from oracle import ipm as OI

        class _LP:
            pos, box = self.pos, self.box

        x, y = self.sets[0][0], self.sets[0][1]
        if not solved:
            x, y = np.zeros(self.n), np.zeros(self.m)
        ibox = slice(None) if self.box.all() else np.flatnonzero(self.box)
        self.sets[0] = list(OI.start_from_projections(self.At, self.c, self.u, _LP, ibox, x.copy(), y.copy()))
        return np.zeros(5)

    def ipm_put(self, which, x, y, z, w):
        self.sets[which] = [np.array(v, dtype=float) for v in (x, y, z, w)]

    def ipm_get(self, which=0):
        return tuple(v.copy() for v in self.sets[which])

    def _floors(self, x):
        s = np.ones(self.n)
        ub = self.u[self.box]
        q = 0.25 * ub
        xf = np.minimum(8.0 * EPS, q)
        sf = np.minimum(8.0 * EPS * np.maximum(1.0, ub), q)
        x[self.box] = np.clip(x[self.box], xf, ub - sf)
        s[self.box] = np.maximum(ub - x[self.box], sf)
        return s

    def ipm_copy(self, to_centre):
        if to_centre:
            self.sets[1] = [v.copy() for v in self.sets[0]]
        else:
            self.sets[0] = [v.copy() for v in self.sets[1]]
            self.s = self._floors(self.sets[0][0])

    def _comp(self, x, z, w, s):
        return float(x[self.pos] @ z[self.pos] + s[self.box] @ w[self.box])

    def ipm_residuals(self, rho, delta):
        x, y, z, w = self.sets[0]
        xk, yk = self.sets[1][0], self.sets[1][1]
        aty = self.At @ y
        self.rd = -(self.c - aty - z + w + rho * (x - xk))
        self.rp = -(self.A @ x - self.b + delta * (y - yk))
        g = self.c - aty + rho * (x - xk)
        gp = g.copy()
        gp[self.pos] = x[self.pos] - np.clip(x[self.pos] - g[self.pos], 0.0, self.u[self.pos])
        return np.array([self._comp(x, z, w, self.s), gp @ gp, self.rp @ self.rp, self.rd @ self.rd,
                         (x - xk) @ (x - xk), (y - yk) @ (y - yk)])

    def ipm_theta(self, theta_min, theta_cap, delta):
        x, _, z, w = self.sets[0]
        t = np.full(self.n, theta_min)
        t[self.pos] += z[self.pos] / x[self.pos]
        t[self.box] += w[self.box] / self.s[self.box]
        t = np.where(np.isfinite(t), t, theta_cap)
        self.set_theta(np.clip(t, theta_min, theta_cap), delta)

    def ipm_targets(self, kind, *p):
        x, _, z, w = self.sets[0]
        dx, _, dz, dw = self.sets[2]
        s, pos, box = self.s, self.pos, self.box
        if kind == 0:
            self.rmz = np.where(pos, -x * z + p[0], 0.0)
            self.rmw = np.where(box, -s * w + p[0], 0.0)
        elif kind == 1:
            self.rmz = np.where(pos, p[0] - dx * dz, 0.0)
            self.rmw = np.where(box, p[0] + dx * dw, 0.0)
        else:
            ta_x, ta_z, mu_t, bmin, bmax = p
            for prod, tgt, mask in (((x + ta_x * dx) * (z + ta_z * dz), self.rmz, pos),
                                    ((s - ta_x * dx) * (w + ta_z * dw), self.rmw, box)):
                corr = np.clip(prod, bmin * mu_t, bmax * mu_t) - prod
                tgt[mask] = np.clip(corr, -bmax * mu_t, 2 * bmax * mu_t)[mask]

    def ipm_newton(self, corrector, tol, maxit, variant=_lib.PCG_SPECTRAL, replacement=100, gap_tolerance=0.1):
        x, _, z, w = self.sets[0]
        r1 = (np.zeros(self.n) if corrector else self.rd.copy())
        r1[self.pos] += self.rmz[self.pos] / x[self.pos]
        r1[self.box] -= self.rmw[self.box] / self.s[self.box]
        r2 = np.zeros(self.m) if corrector else self.rp
        dx, res = self.solve(r1, r2, tol, maxit, variant, replacement, gap_tolerance)
        dy = res.x
        dz = np.where(self.pos, (self.rmz - z * dx) / x, 0.0)
        dw = np.where(self.box, (self.rmw + w * dx) / self.s, 0.0)
        self.sets[3 if corrector else 2] = [dx, dy, dz, dw]
        finite = all(np.isfinite(v).all() for v in (dx, dy, dz, dw))
        return bool(finite), res

    @staticmethod
    def _step(v, d, mask):
        neg = mask & (d < 0.0)
        return 1.0 if not neg.any() else float(min(1.0, np.min(-v[neg] / d[neg])))

    def _combined(self, with_corrector, gamma):
        d = self.sets[2]
        if not with_corrector:
            return d
        return [a + gamma * b for a, b in zip(d, self.sets[3])]

    def ipm_steps(self, with_corrector=False, gamma=0.0):
        x, _, z, w = self.sets[0]
        dx, _, dz, dw = self._combined(with_corrector, gamma)
        return (min(self._step(x, dx, self.pos), self._step(self.s, -dx, self.box)),
                min(self._step(z, dz, self.pos), self._step(w, dw, self.box)))

    def ipm_complementarity(self, alpha_x, alpha_z, with_corrector=False, gamma=0.0):
        x, _, z, w = self.sets[0]
        dx, _, dz, dw = self._combined(with_corrector, gamma)
        return self._comp(x + alpha_x * dx, z + alpha_z * dz, w + alpha_z * dw, self.s - alpha_x * dx)

    def ipm_accept(self, gamma):
        self.sets[2] = self._combined(True, gamma)

    def ipm_update(self, alpha_x, alpha_z):
        x, y, z, w = self.sets[0]
        dx, dy, dz, dw = self.sets[2]
        x = x + alpha_x * dx
        self.sets[0] = [x, y + alpha_z * dy, z + alpha_z * dz, w + alpha_z * dw]
        s = self._floors(x)
        self.s[self.box] = s[self.box]

    def ipm_metrics(self):
        x, y, z, w = self.sets[0]
        self.s = self._floors(x)
        rp = self.b - self.A @ x
        rd = self.c - self.At @ y - z + w
        return np.array([np.abs(rp).max(initial=0.0), np.abs(rd).max(initial=0.0), self.c @ x, self.b @ y,
                         w[self.box] @ self.u[self.box], self._comp(x, z, w, self.s)])

    def lag_reference(self):
        self.wref = self.w.copy()

    def lag_ratio(self):
        ratio = self.w / np.maximum(self.wref, OS.TINY)
        if not (np.isfinite(ratio) & (ratio > 0.0)).all():
            return np.inf, 0.0
        return float(ratio.max()), float(ratio.min())

    def close(self):
        pass
