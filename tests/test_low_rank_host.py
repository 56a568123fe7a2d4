"""F3 host side: the dense-column selection against the reference fixture.

``dense_m1200`` is the reference run on an LP with four 1,100-entry columns;
its ``_low_rank_normal_columns`` (psipm_active_pool.py:691-718) extracted
them, and its candidate set (psipm_stable_preconditioner.py:169-172) leaves
them out.
"""

import numpy as np

from _helpers import lp_from
from psipm_b200.kkt import low_rank_normal_columns


def test_dense_columns_and_candidates(golden):
    g = golden("dense_m1200")
    lp = lp_from(g)
    cols = low_rank_normal_columns(lp.A, 8, 1024, 2.0)
    assert np.array_equal(cols, g["low_rank_columns"])
    counts = np.diff(lp.A.indptr)
    keep = np.ones(lp.A.shape[1], bool)
    keep[cols] = False
    assert np.array_equal(np.flatnonzero(keep & (counts >= 2)), g["candidates"])


def test_other_fixtures_have_no_dense_columns(golden):
    for name in ("random_m300", "grid_20x25", "cover_m200"):
        lp = lp_from(golden(name))
        assert low_rank_normal_columns(lp.A, 8, 1024, 2.0).size == 0
