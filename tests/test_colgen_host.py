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
