"""A CPU stand-in for ``NormalEquationsDevice`` — test infrastructure.

It answers the same method calls with the oracle's NumPy arithmetic, so the
host-side policy of ``psipm_b200.kkt`` and the IPM loop of
``psipm_b200.ipm`` can run without a GPU, and it can be told to fail a given
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

    def close(self):
        pass
