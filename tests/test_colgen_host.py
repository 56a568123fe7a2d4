"""Column-generation host logic without a GPU: the covering crash support.

``colgen.covering_crash`` must return the same support as the reference's
``_covering_crash_mask`` (psipm_active_pool.py:3436-3533) — the fixture
``golden/crash_masks.npz`` holds the reference's masks for covering LPs with
explicit and with implied upper bounds, and an LP it declines — and the
support must make the restricted master feasible.
"""

import os
import sys

import numpy as np
import pytest

from psipm_b200 import synthetic
from psipm_b200.colgen import covering_crash

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from make_golden import CRASH_CASES, crash_lp  # noqa: E402

FIX = np.load(os.path.join(HERE, "golden", "crash_masks.npz"))


@pytest.mark.parametrize("name", sorted(CRASH_CASES))
def test_crash_support_matches_the_reference(name):
    family, kwargs = CRASH_CASES[name]
    assert FIX[f"{name}_kwargs"] == repr(kwargs)
    lp = crash_lp(synthetic, name, family, kwargs)
    mask = covering_crash(lp)
    if bool(FIX[f"{name}_none"]):
        assert mask is None
        return
    assert mask is not None
    assert np.array_equal(mask, FIX[f"{name}_mask"])


@pytest.mark.parametrize("name", ["cover_a", "cover_unbounded"])
def test_crash_support_is_feasible(name):
    """Selected columns at their caps cover every row; the surplus columns
    take the overcoverage with nonnegative values."""
    family, kwargs = CRASH_CASES[name]
    lp = crash_lp(synthetic, name, family, kwargs)
    mask = covering_crash(lp)
    A = lp.A.tocsc()
    cols = np.flatnonzero(mask)
    single = np.diff(A.indptr)[cols] == 1
    surplus = cols[single & (A.data[A.indptr[cols]] < 0)]
    structural = np.setdiff1d(cols, surplus)
    cap = np.where(np.isfinite(lp.u), lp.u, 0.0)
    if not np.isfinite(lp.u).all():
        ratios = np.maximum.reduceat(lp.b[A.indices] / A.data, A.indptr[:-1])
        cap = np.where(np.isfinite(lp.u), lp.u, ratios)
    x = np.zeros(A.shape[1])
    x[structural] = cap[structural]
    r = lp.b - A @ x  # <= 0: overcoverage, taken by the surplus columns
    assert np.all(r <= 1e-12 * (1 + np.abs(lp.b)))
    rows = A.indices[A.indptr[surplus]]
    assert np.unique(rows).size == lp.A.shape[0]


def test_mapped_master_start():
    """Kept columns and the artificials keep their values, new columns start
    central (boxed ones inside their box), y is kept."""
    from types import SimpleNamespace

    from psipm_b200.colgen import mapped_master_start

    lp = synthetic.set_cover(30, 400, seed=7)
    m = lp.A.shape[0]
    rng = np.random.default_rng(1)
    old_cols = np.array([2, 5, 9, 40, 41, 77], dtype=np.int64)
    new_cols = np.array([2, 3, 9, 41, 77, 100, 350], dtype=np.int64)
    k = old_cols.size + 2 * m
    old = SimpleNamespace(x=rng.uniform(0.1, 0.9, k), z=rng.uniform(0.1, 2, k), w=rng.uniform(0.1, 2, k),
                          y=rng.standard_normal(m), mu=0.04)
    x, y, z, w = mapped_master_start(lp, old_cols, old, new_cols)
    assert x.size == new_cols.size + 2 * m and np.array_equal(y, old.y)
    for a, j in enumerate(new_cols):
        hit = np.flatnonzero(old_cols == j)
        if hit.size:
            assert (x[a], z[a], w[a]) == (old.x[hit[0]], old.z[hit[0]], old.w[hit[0]])
        else:
            assert x[a] == pytest.approx(0.2) and z[a] == pytest.approx(0.04 / 0.2)
            assert (w[a] > 0) == bool(lp.box[j])
    assert np.array_equal(x[new_cols.size:], old.x[old_cols.size:])
    assert mapped_master_start(lp, None, None, new_cols) is None
