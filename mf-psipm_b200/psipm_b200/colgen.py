"""Column generation over device solves.

The reference's column-generation drivers (``retrospective_solve`` and
``warm_sparse_solve``, psipm_active_pool.py:2950-4083) solve a sequence of
restricted master LPs on a working set of columns with ``psipm_solve`` and
price the remaining columns with the duals after each converged master.
This module is the device counterpart of that loop in its basic form (no
retrospective elimination, no warm start mapping):

* the master is the LP restricted to the working columns plus one
  artificial column ``+e_i`` and one ``-e_i`` per row at a large cost, so
  every master is feasible (the reference's ``cg_artificial_cost``);
* each master is solved to ``tol`` by the device-resident PS-IPM
  (``ipm_device.solve_standard``);
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
                            device: int = 0, solver_options: Optional[dict] = None) -> ColumnGenerationResult:
    from .ipm_device import solve_standard

    started = time.perf_counter()
    m, n = lp.A.shape
    working = initial_working(lp, max(256, m) if initial is None else initial)
    batch = max(1000, min(n, max(1, m // 2))) if pricing_batch is None else int(pricing_batch)
    ptol = max(tol, 1e-9) if pricing_tol is None else float(pricing_tol)
    big = (1e3 * (1.0 + float(np.abs(lp.c).max(initial=0.0)))) if artificial_cost is None else float(artificial_cost)
    pricer = DevicePricing(lp.A, lp.c, device=device)
    history: List[dict] = []
    added = 0
    status, sol, cols = "round-limit", None, np.flatnonzero(working)
    try:
        for rnd in range(1, max_rounds + 1):
            cols = np.flatnonzero(working)
            master = _master(lp, cols, big)
            sol, solver = solve_standard(master, tol=tol, device=device, solver_options=solver_options)
            solver.close()
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
