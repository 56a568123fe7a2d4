"""One LP's device state: a thin Python owner of a ``psipm_handle``.

Every method is one C-ABI call (include/psipm_b200.h); arrays cross the
boundary as contiguous NumPy buffers.  A nonzero status raises
:class:`DeviceError`, whose ``status`` is the library's code; the KKT
wrappers translate it into the reference's ``KKTSolveError``.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Optional, Tuple

import numpy as np
import scipy.sparse as sp

from . import _lib
from ._lib import f64, i64, ptr


class DeviceError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{_lib.STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


@dataclass
class PcgResult:
    x: np.ndarray
    info: int
    iterations: int
    matvecs: int
    replacements: int
    residual_checks: int
    relative_residual: float
    ok: bool
    alphas: np.ndarray
    betas: np.ndarray
    history: np.ndarray
    residual: Optional[np.ndarray]
    seconds: float
    refinements: int = 0
    phase_seconds: tuple = (0.0, 0.0, 0.0, 0.0)


class NormalEquationsDevice:
    """Device-resident ``A``, weights, active core, factor and PCG workspace."""

    def __init__(self, A: sp.csc_matrix, device: int = 0, precision: int = _lib.FP64):
        self.lib = _lib.load()
        A = sp.csc_matrix(A)
        A.sum_duplicates()
        A.sort_indices()
        self.A = A
        self.m, self.n = A.shape
        self._colptr = i64(A.indptr)
        self._rowidx = np.ascontiguousarray(A.indices, dtype=np.int32)
        self._values = f64(A.data)
        handle = ctypes.c_void_p()
        status = self.lib.psipm_create(self.m, self.n, A.nnz, ptr(self._colptr), ptr(self._rowidx),
                                       ptr(self._values), int(device), int(precision),
                                       ctypes.byref(handle))
        if status != _lib.OK:
            message = self.lib.psipm_last_error(handle).decode() if handle.value else ""
            if handle.value:
                self.lib.psipm_destroy(handle)
            if status == _lib.ERR_CUDA:
                raise _lib.GpuUnavailable(f"CUDA initialisation failed: {message}")
            raise DeviceError(status, message)
        self.h = handle
        ncand = self.lib.psipm_num_candidates(self.h)
        self.candidates = np.empty(ncand, dtype=np.int64)
        self._check(self.lib.psipm_get_candidates(self.h, ptr(self.candidates)))
        self.precision = precision

    # -- plumbing -------------------------------------------------------------
    def _check(self, status: int) -> None:
        if status != _lib.OK:
            raise DeviceError(status, self.lib.psipm_last_error(self.h).decode())

    def close(self) -> None:
        if getattr(self, "h", None) is not None and self.h.value:
            self.lib.psipm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def kernel_launches(self) -> int:
        return int(self.lib.psipm_kernel_launches(self.h))

    def timer_start(self) -> None:
        self._check(self.lib.psipm_timer_start(self.h))

    def timer_stop(self) -> float:
        out = ctypes.c_double()
        self._check(self.lib.psipm_timer_stop(self.h, ctypes.byref(out)))
        return float(out.value)

    # -- operations -----------------------------------------------------------
    def set_low_rank(self, columns: np.ndarray) -> None:
        """Extracted dense columns (psipm_set_low_rank); the candidates change."""
        cols = i64(np.sort(np.asarray(columns)))
        self._check(self.lib.psipm_set_low_rank(self.h, ptr(cols), cols.size))
        ncand = self.lib.psipm_num_candidates(self.h)
        self.candidates = np.empty(ncand, dtype=np.int64)
        self._check(self.lib.psipm_get_candidates(self.h, ptr(self.candidates)))

    def set_theta(self, theta: np.ndarray, delta: float) -> None:
        theta = f64(theta)
        if theta.shape != (self.n,):
            raise ValueError("theta has the wrong dimension")
        self._check(self.lib.psipm_set_theta(self.h, ptr(theta), float(delta)))

    def scores(self, fill_weight: float, want: bool = True, want_diag: bool = False):
        out = np.empty(self.candidates.size) if want else None
        diag = np.empty(self.m) if want_diag else None
        self._check(self.lib.psipm_scores(self.h, float(fill_weight), ptr(out), ptr(diag)))
        return out, diag

    def refresh_core(self, target: int, retention: float, stable: bool,
                     mandatory_local: np.ndarray) -> Tuple[np.ndarray, float]:
        mandatory_local = i64(mandatory_local)
        core = np.empty(max(1, self.candidates.size), dtype=np.int64)
        ncore = ctypes.c_int64()
        retained = ctypes.c_double()
        self._check(self.lib.psipm_refresh_core(
            self.h, int(target), float(retention), int(bool(stable)), ptr(mandatory_local),
            mandatory_local.size, ptr(core), ctypes.byref(ncore), ctypes.byref(retained)))
        return core[: ncore.value].copy(), float(retained.value)

    def set_tree(self, parent, depth, tree_child) -> None:
        """Switch to the network tree-plus-diagonal preconditioner (psipm_set_tree)."""
        i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)  # noqa: E731
        parent, depth, tree_child = i32(parent), i32(depth), i32(tree_child)
        if parent.shape != (self.m,) or depth.shape != (self.m,) or tree_child.shape != (self.n,):
            raise ValueError("forest arrays have the wrong dimensions")
        self._check(self.lib.psipm_set_tree(self.h, ptr(parent), ptr(depth), ptr(tree_child)))

    def tree_factor(self, weights, delta: float) -> None:
        w = f64(weights)
        if w.shape != (self.n,):
            raise ValueError("weights have the wrong dimension")
        self._check(self.lib.psipm_tree_factor(self.h, ptr(w), float(delta)))

    def tree_get(self):
        pivot, mult = np.empty(self.m), np.empty(self.m)
        self._check(self.lib.psipm_tree_get(self.h, ptr(pivot), ptr(mult)))
        return pivot, mult

    def price_load(self, c: np.ndarray) -> None:
        c = f64(c)
        if c.shape != (self.n,):
            raise ValueError("c has the wrong dimension")
        self._check(self.lib.psipm_price_load(self.h, ptr(c)))

    def price(self, y, tau: float, active: np.ndarray, threshold: float, batch: int):
        """HSD pricing round (psipm_price): returns (violation, candidates)."""
        y = f64(y)
        act = np.ascontiguousarray(active, dtype=np.uint8)
        if y.shape != (self.m,) or act.shape != (self.n,):
            raise ValueError("y or the active mask has the wrong dimension")
        violation = np.empty(self.n)
        cand = np.empty(max(1, min(self.n, int(batch))), dtype=np.int64)
        count = ctypes.c_int64()
        self._check(self.lib.psipm_price(self.h, ptr(y), float(tau), ptr(act), float(threshold), int(batch),
                                         ptr(violation), ptr(cand), ctypes.byref(count)))
        return violation, cand[: count.value].copy()

    def get_theta(self) -> np.ndarray:
        out = np.empty(self.n)
        self._check(self.lib.psipm_get_theta(self.h, ptr(out)))
        return out

    def mlp_features(self, mu: float) -> np.ndarray:
        """The learned selector's six inputs per candidate (psipm_mlp_features)."""
        out = np.empty((self.candidates.size, _lib.MLP_INPUTS), dtype=np.float32)
        self._check(self.lib.psipm_mlp_features(self.h, float(mu), ptr(out)))
        return out

    def mlp_scores(self, weights_bf16: np.ndarray, biases: np.ndarray, mu: float, keep: int = 0) -> float:
        """Replace the handle's scores by the network's (only the rule's `keep`
        best candidates stay eligible when keep > 0); returns the shift vote."""
        w = np.ascontiguousarray(weights_bf16, dtype=np.uint16)
        b = np.ascontiguousarray(biases, dtype=np.float32)
        if w.size != _lib.MLP_WEIGHTS or b.size != _lib.MLP_BIASES:
            raise ValueError("selector parameters have the wrong size")
        vote = ctypes.c_double()
        self._check(self.lib.psipm_mlp_scores(self.h, ptr(w), ptr(b), float(mu), int(keep), ctypes.byref(vote)))
        return float(vote.value)

    def set_deterministic(self, on: bool) -> None:
        """Fixed-order accumulation in the preconditioner apply (psipm_set_deterministic)."""
        self._check(self.lib.psipm_set_deterministic(self.h, int(bool(on))))

    def set_factor_tc(self, passes: int) -> None:
        """FP32 big fronts on the tensor cores: 3 (3xTF32, default), 1 (TF32) or
        0 (CUDA cores) (psipm_set_factor_tc)."""
        self._check(self.lib.psipm_set_factor_tc(self.h, int(passes)))

    def set_grid(self, blocks: int) -> None:
        """Blocks of this handle's persistent kernels (0: the full co-resident grid)."""
        self._check(self.lib.psipm_set_grid(self.h, int(blocks)))

    def tie_info(self) -> dict:
        """Straddling ties of the top-k selections so far (psipm_tie_info)."""
        out = np.zeros(4, dtype=np.int64)
        self._check(self.lib.psipm_tie_info(self.h, ptr(out)))
        return dict(straddles=int(out[0]), tied=int(out[1]), slots=int(out[2]), selections=int(out[3]))

    def set_core(self, core: np.ndarray) -> None:
        core = i64(core)
        self._check(self.lib.psipm_set_core(self.h, ptr(core), core.size))

    def top_k(self, scores: np.ndarray, count: int, mask: Optional[np.ndarray] = None) -> np.ndarray:
        scores = f64(scores)
        m = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint8)
        out = np.empty(max(1, int(count)), dtype=np.int64)
        nout = ctypes.c_int64()
        self._check(self.lib.psipm_top_k(self.h, ptr(scores), scores.size, ptr(m), int(count),
                                         ptr(out), ctypes.byref(nout)))
        return out[: nout.value].copy()

    def factor(self, delta: float, start_shift: int = 0):
        shift = ctypes.c_int32(-1)
        info = _lib.FactorInfo()
        status = self.lib.psipm_factor(self.h, float(delta), int(start_shift), ctypes.byref(shift),
                                       ctypes.byref(info))
        if status != _lib.OK:
            raise DeviceError(status, self.lib.psipm_last_error(self.h).decode())
        return int(shift.value), info

    def apply(self, r: np.ndarray) -> np.ndarray:
        r = f64(r)
        z = np.empty(self.m)
        self._check(self.lib.psipm_apply(self.h, ptr(r), ptr(z)))
        return z

    def matvec(self, v: np.ndarray) -> np.ndarray:
        v = f64(v)
        y = np.empty(self.m)
        self._check(self.lib.psipm_matvec(self.h, ptr(v), ptr(y)))
        return y

    def pcg(self, rhs, tol, maxit, variant=_lib.PCG_SPECTRAL, replacement=100, gap_tolerance=0.1,
            want_residual=False) -> PcgResult:
        rhs = f64(rhs)
        x = np.empty(self.m)
        res = np.empty(self.m) if want_residual else None
        alphas = np.empty(max(1, maxit))
        betas = np.empty(max(1, maxit))
        history = np.empty(maxit + 2)
        info = _lib.PcgInfo()
        self._check(self.lib.psipm_pcg(self.h, ptr(rhs), float(tol), int(maxit), int(variant),
                                       int(replacement), float(gap_tolerance), ptr(x), ptr(res),
                                       ptr(alphas), ptr(betas), ptr(history), ctypes.byref(info)))
        return self._result(x, info, alphas, betas, history, res)

    def set_pcg_budget(self, seconds: float) -> None:
        """Wall-clock budget of every later PCG launch (0: none), psipm_set_pcg_budget."""
        self._check(self.lib.psipm_set_pcg_budget(self.h, float(seconds)))

    def solve(self, r1, r2, tol, maxit, variant=_lib.PCG_SPECTRAL, replacement=100, gap_tolerance=0.1,
              want_residual=False):
        r1 = f64(r1)
        r2 = f64(r2)
        dx = np.empty(self.n)
        dy = np.empty(self.m)
        res = np.empty(self.m) if want_residual else None
        alphas = np.empty(max(1, maxit))
        betas = np.empty(max(1, maxit))
        history = np.empty(maxit + 2)
        info = _lib.PcgInfo()
        self._check(self.lib.psipm_solve(self.h, ptr(r1), ptr(r2), float(tol), int(maxit), int(variant),
                                         int(replacement), float(gap_tolerance), ptr(dx), ptr(dy),
                                         ptr(res), ptr(alphas), ptr(betas), ptr(history),
                                         ctypes.byref(info)))
        return dx, self._result(dy, info, alphas, betas, history, res)

    # -- device-resident IPM vectors (include/psipm_b200.h, psipm_ipm_*) -------
    def ipm_load(self, c, b, u, pos, box) -> None:
        self._ipm_data = (f64(c), f64(b), f64(u), np.ascontiguousarray(pos, dtype=np.uint8),
                          np.ascontiguousarray(box, dtype=np.uint8))
        c, b, u, pos, box = self._ipm_data
        if c.shape != (self.n,) or b.shape != (self.m,) or u.shape != (self.n,) or pos.shape != (self.n,) \
                or box.shape != (self.n,):
            raise ValueError("LP data has the wrong dimensions")
        self._check(self.lib.psipm_ipm_load(self.h, ptr(c), ptr(b), ptr(u), ptr(pos), ptr(box)))
        self._scal = np.zeros(8)

    # vector sets of psipm_ipm_put / psipm_ipm_get
    ITERATE, CENTRE, DIRECTION, CORRECTOR = 0, 1, 2, 3

    def ipm_put(self, which: int, x, y, z, w) -> None:
        x, y, z, w = f64(x), f64(y), f64(z), f64(w)
        if x.shape != (self.n,) or y.shape != (self.m,) or z.shape != (self.n,) or w.shape != (self.n,):
            raise ValueError("vector set has the wrong dimensions")
        self._check(self.lib.psipm_ipm_put(self.h, int(which), ptr(x), ptr(y), ptr(z), ptr(w)))

    def ipm_get(self, which: int = 0):
        x, z, w = np.empty(self.n), np.empty(self.n), np.empty(self.n)
        y = np.empty(self.m)
        self._check(self.lib.psipm_ipm_get(self.h, int(which), ptr(x), ptr(y), ptr(z), ptr(w)))
        return x, y, z, w

    def ipm_copy(self, to_centre: bool) -> None:
        self._check(self.lib.psipm_ipm_copy(self.h, int(to_centre)))

    def ipm_residuals(self, rho: float, delta: float) -> np.ndarray:
        out = np.empty(6)
        self._check(self.lib.psipm_ipm_residuals(self.h, float(rho), float(delta), ptr(out)))
        return out

    def ipm_theta(self, theta_min: float, theta_cap: float, delta: float) -> None:
        self._check(self.lib.psipm_ipm_theta(self.h, float(theta_min), float(theta_cap), float(delta)))

    def ipm_targets(self, kind: int, *params: float) -> None:
        p = np.zeros(5)
        p[: len(params)] = params
        self._check(self.lib.psipm_ipm_targets(self.h, int(kind), ptr(p)))

    def ipm_newton(self, corrector: bool, tol, maxit, variant=_lib.PCG_SPECTRAL, replacement=100,
                   gap_tolerance=0.1):
        alphas = np.empty(max(1, maxit))
        betas = np.empty(max(1, maxit))
        history = np.empty(maxit + 2)
        finite = ctypes.c_int32()
        info = _lib.PcgInfo()
        self._check(self.lib.psipm_ipm_newton(self.h, int(corrector), float(tol), int(maxit), int(variant),
                                              int(replacement), float(gap_tolerance), ptr(alphas), ptr(betas),
                                              ptr(history), ctypes.byref(finite), ctypes.byref(info)))
        return bool(finite.value), self._result(None, info, alphas, betas, history, None)

    def ipm_start_solve(self, which: int, tol, maxit, variant=_lib.PCG_SPECTRAL, replacement=100,
                        gap_tolerance=0.1):
        """One projection of the starting point (which 0: x = A^T dy for r2 = b;
        1: y = dy for r2 = A c) into the iterate; returns (finite, result)."""
        alphas = np.empty(max(1, maxit))
        betas = np.empty(max(1, maxit))
        history = np.empty(maxit + 2)
        finite = ctypes.c_int32()
        info = _lib.PcgInfo()
        self._check(self.lib.psipm_ipm_start_solve(self.h, int(which), float(tol), int(maxit), int(variant),
                                                   int(replacement), float(gap_tolerance), ptr(alphas),
                                                   ptr(betas), ptr(history), ctypes.byref(finite),
                                                   ctypes.byref(info)))
        return bool(finite.value), self._result(None, info, alphas, betas, history, None)

    def ipm_start(self, solved: bool) -> np.ndarray:
        """The rest of the starting point on the device (psipm_ipm_start)."""
        out = np.zeros(5)
        self._check(self.lib.psipm_ipm_start(self.h, int(bool(solved)), ptr(out)))
        return out

    def ipm_steps(self, with_corrector: bool = False, gamma: float = 0.0) -> Tuple[float, float]:
        out = np.empty(2)
        self._check(self.lib.psipm_ipm_steps(self.h, int(with_corrector), float(gamma), ptr(out)))
        return float(out[0]), float(out[1])

    def ipm_complementarity(self, alpha_x, alpha_z, with_corrector: bool = False, gamma: float = 0.0) -> float:
        out = ctypes.c_double()
        self._check(self.lib.psipm_ipm_complementarity(self.h, int(with_corrector), float(gamma), float(alpha_x),
                                                       float(alpha_z), ctypes.byref(out)))
        return float(out.value)

    def ipm_accept(self, gamma: float) -> None:
        self._check(self.lib.psipm_ipm_accept(self.h, float(gamma)))

    def ipm_update(self, alpha_x: float, alpha_z: float) -> None:
        self._check(self.lib.psipm_ipm_update(self.h, float(alpha_x), float(alpha_z)))

    def ipm_metrics(self) -> np.ndarray:
        out = np.empty(6)
        self._check(self.lib.psipm_ipm_metrics(self.h, ptr(out)))
        return out

    def lag_reference(self) -> None:
        self._check(self.lib.psipm_lag_reference(self.h))

    def lag_ratio(self) -> Tuple[float, float]:
        out = np.empty(2)
        self._check(self.lib.psipm_lag_ratio(self.h, ptr(out)))
        return float(out[0]), float(out[1])

    # -- R2 MINRES fallback (psipm_minres / psipm_ipm_minres) ------------------
    def minres(self, r1, r2, tol, maxit, fail_tol):
        """(dx, dy, accepted, iterations, relative residual) of the augmented MINRES."""
        r1, r2 = f64(r1), f64(r2)
        dx, dy = np.empty(self.n), np.empty(self.m)
        info = _lib.PcgInfo()
        self._check(self.lib.psipm_minres(self.h, ptr(r1), ptr(r2), float(tol), int(maxit), float(fail_tol),
                                          ptr(dx), ptr(dy), ctypes.byref(info)))
        return dx, dy, bool(info.ok), int(info.iterations), float(info.relative_residual)

    def ipm_minres(self, corrector: bool, tol, maxit, fail_tol):
        """(finite, accepted, iterations, relative residual); the directions stay on the device."""
        finite = ctypes.c_int32()
        info = _lib.PcgInfo()
        self._check(self.lib.psipm_ipm_minres(self.h, int(corrector), float(tol), int(maxit), float(fail_tol),
                                              ctypes.byref(finite), ctypes.byref(info)))
        return bool(finite.value), bool(info.ok), int(info.iterations), float(info.relative_residual)

    @staticmethod
    def _result(x, info, alphas, betas, history, res) -> PcgResult:
        return PcgResult(
            x=x, info=int(info.info), iterations=int(info.iterations), matvecs=int(info.matvecs),
            replacements=int(info.replacements), residual_checks=int(info.residual_checks),
            relative_residual=float(info.relative_residual), ok=bool(info.ok),
            alphas=alphas[: info.n_alpha].copy(), betas=betas[: info.n_beta].copy(),
            history=history[: info.n_history].copy(), residual=res, seconds=float(info.seconds),
            refinements=int(info.refinements), phase_seconds=tuple(float(v) for v in info.phase_seconds),
        )
