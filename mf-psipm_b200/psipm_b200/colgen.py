"""Column generation over device solves.

The reference's column-generation drivers (``retrospective_solve`` and
``warm_sparse_solve``, psipm_active_pool.py:2950-4083) solve a sequence of
restricted master LPs on a working set of columns with ``psipm_solve`` and
price the remaining columns with the duals after each converged master.
This module is the device counterpart of that loop in its basic form (no
retrospective elimination, no l1 budgets):

* the first working set is the covering crash support when asked for and
  the LP is a covering LP (:func:`covering_crash`), else the free columns and
  the cheapest others;
* the master is the LP restricted to the working columns plus one
  artificial column ``+e_i`` and one ``-e_i`` per row at a large cost, so
  every master is feasible (the reference's ``cg_artificial_cost``);
* each master is solved to ``tol`` by the device-resident PS-IPM
  (``ipm_device.solve_standard``), from its own starting point or, when
  asked for, from the previous master's solution mapped onto its columns;
* pricing runs on the device over all columns (``pricing.DevicePricing``:
  ``A' y - c`` and the ``pricing_batch`` most violated columns not yet
  working), the same kernels as the HSD pricing round;
* the loop stops when no column prices out with the artificials at zero
  (then the master's solution, extended by zeros, is optimal for the full
  LP), raises the artificial cost when they are not, and gives up after
  ``max_rounds``.
"""

from __future__ import annotations

import time
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np
import scipy.sparse as sp

from .pricing import DevicePricing
from .synthetic import StandardLP


@dataclass
class ColumnGenerationResult:
    status: str
    obj: float
    x: np.ndarray
    y: np.ndarray
    rounds: int
    working: int
    columns_added: int
    artificial: float  # largest artificial value of the last master
    seconds: float
    history: List[dict] = field(default_factory=list)


_EPS = float(np.finfo(float).eps)
_POS_FLOOR = 8.0 * _EPS


def covering_crash(lp) -> Optional[np.ndarray]:
    """A feasible starting support for a covering LP, or None.

    The reference's crash (``_covering_crash_mask``, psipm_active_pool.py:
    3436-3533) applies to an LP whose rows have positive demand b_i, whose
    structural columns are nonnegative and whose every row has a zero-cost,
    unbounded, negative singleton surplus column.  An unbounded structural
    column of nonnegative cost never needs to exceed max_i b_i / a_ij over its
    rows, so that value caps it; each row then takes the structural column
    that can cover it alone at its cap with the least cap cost per unit of
    covered demand (the first such column in index order on ties), and the
    surplus columns absorb the overcoverage.  The selected columns plus all
    surplus columns are a feasible restricted master.  This is the same
    decision rule, computed over the CSR arrays at once instead of row by row.
    """
    A = lp.A.tocsc(copy=True)
    A.eliminate_zeros()
    m, n = A.shape
    b, c, u = np.asarray(lp.b, float), np.asarray(lp.c, float), np.asarray(lp.u, float)
    if m == 0 or np.any(b <= 0.0) or not np.all(lp.pos):
        return None
    nnz_col = np.diff(A.indptr)
    scale = 1.0 + float(np.abs(c).max(initial=0.0))
    single = np.flatnonzero((nnz_col == 1) & (np.abs(c) <= 100.0 * _EPS * scale) & ~np.isfinite(u))
    srow = A.indices[A.indptr[single]]
    sval = A.data[A.indptr[single]]
    neg = sval < 0.0
    single, srow, sval = single[neg], srow[neg], sval[neg]
    # per row the surplus of largest |value|, the lowest column index among equals
    order = np.lexsort((single, sval, srow))  # by row, then most negative value, then index
    first = np.ones(order.size, dtype=bool)
    first[1:] = srow[order][1:] != srow[order][:-1]
    pick = order[first]
    surplus = np.full(m, -1, dtype=np.int64)
    surplus_value = np.zeros(m)
    surplus[srow[pick]] = single[pick]
    surplus_value[srow[pick]] = sval[pick]
    if np.any(surplus < 0):
        return None
    structural = np.ones(n, dtype=bool)
    structural[surplus] = False
    cols = np.repeat(np.arange(n), nnz_col)
    if np.any((A.data < -100.0 * _EPS) & structural[cols]):
        return None
    cap = u.copy()
    ratio_max = np.full(n, np.inf)
    nonempty = nnz_col > 0
    if nonempty.any():
        ratio_max[nonempty] = np.maximum.reduceat(b[A.indices] / A.data, A.indptr[:-1][nonempty])
    implied = structural & ~np.isfinite(cap) & (c >= -100.0 * _EPS * scale)
    cap[implied] = ratio_max[implied]
    usable_col = structural & np.isfinite(cap) & (cap > 0.0)
    R = A.tocsr()
    rows = np.repeat(np.arange(m), np.diff(R.indptr))
    jj, aa = R.indices, R.data
    tol = 100.0 * _EPS * (1.0 + np.abs(b))
    ok = usable_col[jj] & (aa > 0.0)
    contribution = np.where(ok, aa * np.where(ok, cap[jj], 0.0), 0.0)
    ok &= contribution + tol[rows] >= b[rows]
    if not np.all(np.bincount(rows[ok], minlength=m) > 0):
        return None
    score = np.full(jj.size, np.inf)
    cj = np.where(ok, cap[jj], 0.0)
    score[ok] = np.maximum(c[jj[ok]] * cj[ok], 0.0) / np.maximum(np.minimum(contribution[ok], b[rows[ok]]),
                                                                   _POS_FLOOR)
    # per row the first entry (CSR order) of least score among the valid ones
    pos = np.arange(jj.size)
    best_order = np.lexsort((pos, score, rows))
    head = np.ones(best_order.size, dtype=bool)
    head[1:] = rows[best_order][1:] != rows[best_order][:-1]
    best = jj[best_order[head]]
    selected = np.unique(best)
    coverage = np.asarray(A[:, selected] @ cap[selected]).ravel()
    over = coverage - b
    if np.any(over < -tol):
        return None
    with np.errstate(divide="ignore", invalid="ignore"):
        surplus_x = over / (-surplus_value)
    if np.any(~np.isfinite(surplus_x)) or np.any(surplus_x < 0.0):
        return None
    working = np.zeros(n, dtype=bool)
    working[selected] = True
    working[surplus] = True
    return working


def mapped_master_start(lp, old_cols: np.ndarray, old_sol, new_cols: np.ndarray):
    """A starting point for the next master from the last one's solution, as
    the reference's ``_mapped_rmp_start`` (psipm_active_pool.py:3536-3599)
    maps a restricted master across a change of support: columns kept from
    the old master keep their x, z, w; the artificial columns (here 2m of
    them, +e_i and -e_i, after the structural ones) keep theirs; y is kept; a
    new column starts central at mu = max(old mu, 1e-10): x = max(sqrt(min(mu,
    1)), 1e-8) (a boxed one inside [floor, u/2], floor = max(1e-12, 8 eps (1 +
    |u|))), z = mu / x and, if boxed, w = mu / (u - x).  Returns (x, y, z, w)
    for the new master, or None without an old solution."""
    if old_sol is None or old_cols is None:
        return None
    m = lp.A.shape[0]
    k_old, k_new = old_cols.size, new_cols.size
    x = np.zeros(k_new + 2 * m)
    z = np.zeros_like(x)
    w = np.zeros_like(x)
    loc = np.searchsorted(old_cols, new_cols)
    common = (loc < k_old) & (old_cols[np.minimum(loc, max(0, k_old - 1))] == new_cols)
    src = loc[common]
    x[:k_new][common] = old_sol.x[src]
    z[:k_new][common] = old_sol.z[src]
    w[:k_new][common] = old_sol.w[src]
    x[k_new:] = old_sol.x[k_old:]
    z[k_new:] = old_sol.z[k_old:]
    w[k_new:] = old_sol.w[k_old:]
    fresh = np.flatnonzero(~common)
    if fresh.size:
        mu = max(float(old_sol.mu) if np.isfinite(old_sol.mu) else 0.0, 1e-10)
        jj = new_cols[fresh]
        xn = np.full(fresh.size, max(np.sqrt(min(mu, 1.0)), 1e-8))
        boxed = np.asarray(lp.box, dtype=bool)[jj]
        if boxed.any():
            ub = lp.u[jj[boxed]]
            floor = np.maximum(1e-12, _POS_FLOOR * (1.0 + np.abs(ub)))
            xn[boxed] = np.minimum(np.maximum(xn[boxed], floor), 0.5 * ub)
        x[fresh] = xn
        z[fresh] = mu / np.maximum(xn, 1e-12)
        if boxed.any():
            w[fresh[boxed]] = mu / np.maximum(lp.u[jj[boxed]] - xn[boxed], 1e-12)
    return x, np.array(old_sol.y, dtype=float), z, w


def initial_working(lp, count: int) -> np.ndarray:
    """Free columns (never priced out) and the `count` cheapest others."""
    n = lp.A.shape[1]
    working = ~np.asarray(lp.pos, dtype=bool)
    need = max(0, min(n, int(count)) - int(working.sum()))
    rest = np.flatnonzero(~working)
    if need and rest.size:
        pick = rest[np.argsort(lp.c[rest], kind="stable")[:need]]
        working[pick] = True
    return working


def _master(lp, cols: np.ndarray, big: float) -> StandardLP:
    m = lp.A.shape[0]
    eye = sp.identity(m, format="csc")
    A = sp.hstack([lp.A[:, cols], eye, -eye], format="csc")
    c = np.concatenate([lp.c[cols], np.full(2 * m, big)])
    u = np.concatenate([lp.u[cols], np.full(2 * m, np.inf)])
    pos = np.concatenate([lp.pos[cols], np.ones(2 * m, dtype=bool)])
    box = pos & np.isfinite(u)
    return StandardLP(c=c, A=A, b=lp.b, u=u, pos=pos, box=box, obj_const=lp.obj_const, name=f"{lp.name}-master")


def column_generation_solve(lp, tol: float = 1e-8, initial: Optional[int] = None,
                            pricing_batch: Optional[int] = None, pricing_tol: Optional[float] = None,
                            max_rounds: int = 30, artificial_cost: Optional[float] = None,
                            device: int = 0, solver_options: Optional[dict] = None,
                            crash: bool = False, warm: bool = False) -> ColumnGenerationResult:
    """``crash=True`` starts a covering LP from :func:`covering_crash`'s
    feasible support (the reference's ``sparse_cover_crash``, on by default
    there, psipm_active_pool.py:3746-3749), else from the cheapest columns.
    ``warm=True`` starts every master after the first from the previous
    master's solution (:func:`mapped_master_start`)."""
    from .ipm_device import solve_standard

    started = time.perf_counter()
    m, n = lp.A.shape
    start = covering_crash(lp) if crash else None
    working = start.copy() if start is not None else initial_working(lp, max(256, m) if initial is None else initial)
    batch = max(1000, min(n, max(1, m // 2))) if pricing_batch is None else int(pricing_batch)
    ptol = max(tol, 1e-9) if pricing_tol is None else float(pricing_tol)
    big = (1e3 * (1.0 + float(np.abs(lp.c).max(initial=0.0)))) if artificial_cost is None else float(artificial_cost)
    pricer = DevicePricing(lp.A, lp.c, device=device)
    history: List[dict] = []
    added = 0
    status, sol, cols = "round-limit", None, np.flatnonzero(working)
    try:
        prev_cols, prev_sol = None, None
        for rnd in range(1, max_rounds + 1):
            cols = np.flatnonzero(working)
            master = _master(lp, cols, big)
            start = mapped_master_start(lp, prev_cols, prev_sol, cols) if warm else None
            sol, solver = solve_standard(master, tol=tol, device=device, solver_options=solver_options,
                                         initial=start)
            solver.close()
            prev_cols, prev_sol = cols, sol
            if sol.status != "optimal":
                status = f"master-{sol.status}"
                break
            art = float(np.abs(sol.x[cols.size:]).max(initial=0.0))
            _, cand = pricer.price(sol.y, 1.0, working, ptol, batch)
            history.append(dict(round=rnd, working=int(cols.size), candidates=int(cand.size), artificial=art,
                                obj=float(sol.obj)))
            if cand.size == 0:
                if art <= tol * (1.0 + float(np.abs(lp.b).max(initial=0.0))):
                    status = "optimal"
                    break
                big *= 10.0  # artificials still carry flow: make them dearer
                continue
            working[cand] = True
            added += int(cand.size)
    finally:
        pricer.close()
    x = np.zeros(n)
    if sol is not None:
        x[cols] = sol.x[:cols.size]
    y = sol.y if sol is not None else np.zeros(m)
    art = float(np.abs(sol.x[cols.size:]).max(initial=0.0)) if sol is not None else np.inf
    return ColumnGenerationResult(status, float(lp.c @ x) + lp.obj_const, x, y, len(history), int(cols.size), added,
                                  art, time.perf_counter() - started, history)
