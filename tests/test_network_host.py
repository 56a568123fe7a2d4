"""The network tree-plus-diagonal preconditioner on the host (no GPU).

The fixture ``tree_grid_20x25`` holds the unmodified reference's spanning
forest (NetworkTopology.from_incidence, psipm_v3_1_hsd.py:495-610) of an
ungrounded grid network and its TreePreconditioner's pivots, multipliers and
solves (:715-785).  The product's forest (psipm_b200.network.spanning_forest)
must equal it; the oracle's factor and solve must reproduce it bit for bit.
"""

import numpy as np
import scipy.sparse as sp

from oracle.network import TreeOracle
from psipm_b200 import synthetic
from psipm_b200.network import spanning_forest


def _A(g):
    return sp.csc_matrix((g["A_data"], g["A_indices"], g["A_indptr"]), shape=tuple(int(v) for v in g["A_shape"]))


def test_forest_matches_the_reference(golden):
    g = golden("tree_grid_20x25")
    A = _A(g)
    assert np.array_equal(A.toarray(), synthetic.grid_network(20, 25, seed=1001, ground=False).A.toarray())
    f = spanning_forest(A)
    for key in ("parent", "depth", "tree_child", "protected"):
        assert np.array_equal(getattr(f, key), g[key]), key
    assert f.root == int(g["root"]) and f.components == int(g["components"])


def test_oracle_factor_and_solve_pin_the_reference(golden):
    g = golden("tree_grid_20x25")
    A = _A(g)
    active = g["active"]
    orc = TreeOracle(A[:, active], g["parent"], g["depth"], g["tree_child"][active])
    for c in range(3):
        orc.factor(g[f"c{c}_D"], float(g[f"c{c}_delta"]))
        assert np.array_equal(orc.pivot, g[f"c{c}_pivot"])
        assert np.array_equal(orc.mult, g[f"c{c}_multiplier"])
        for k in range(2):
            assert np.array_equal(orc.solve(g[f"c{c}_rhs{k}"]), g[f"c{c}_sol{k}"])
