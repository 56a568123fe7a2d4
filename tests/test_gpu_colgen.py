"""Column generation over device solves (psipm_b200.colgen): restricted
masters on a working set plus artificial columns, device pricing of every
column after each converged master (the loop of the reference's
column-generation drivers, psipm_active_pool.py:2950-4083, in its basic
form).  On a random LP with ten columns per row it must reach the full
solve's objective (1e-6 relative) in more than one round, with a primal
solution of the full LP and no column left that prices out."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_column_generation_reaches_the_full_solve():
    from psipm_b200 import synthetic
    from psipm_b200.colgen import column_generation_solve
    from psipm_b200.ipm_device import solve_standard

    lp = synthetic.random_lp(300, 3000, seed=21)
    full, solver = solve_standard(lp, tol=1e-8)
    solver.close()
    res = column_generation_solve(lp, tol=1e-8, initial=400, pricing_batch=200)
    print(f"full {full.obj!r}; column generation {res.obj!r}, {res.status}, rounds {res.rounds}, "
          f"working {res.working} of {lp.A.shape[1]}, history {res.history}")
    assert full.status == "optimal" and res.status == "optimal"
    assert res.rounds >= 2
    assert abs(res.obj - full.obj) <= 1e-6 * max(1.0, abs(full.obj))
    rp = np.abs(lp.b - lp.A @ res.x).max() / (1.0 + np.abs(lp.b).max())
    assert rp <= 1e-6 and res.x.min() >= -1e-9
    reduced = lp.c - lp.A.T @ res.y
    assert reduced.min() >= -1e-6 * (1.0 + np.abs(lp.c).max())
