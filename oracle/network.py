"""Oracle restatement of the V3.1 tree-plus-diagonal preconditioner — test infrastructure.

Follows ``TreePreconditioner.factor`` / ``solve`` (psipm_v3_1_hsd.py:732-776)
in the reference's operation order: level by level from the deepest, the
children scatter into their parents with ``np.add.at`` in ascending node
order.  Pinned bit for bit to the reference's own outputs in
``tests/golden/tree_grid_20x25.npz`` (tests/test_network_host.py).
"""

from __future__ import annotations

import numpy as np

TINY = float(np.finfo(np.float64).tiny)


class TreeOracle:
    def __init__(self, A, parent, depth, tree_child):
        A = A.tocsc()
        lo = A.indptr[:-1]
        self.first = A.indices[lo]
        self.second = A.indices[lo + 1]
        self.child = np.asarray(tree_child)
        self.parent = np.asarray(parent)
        self.m = A.shape[0]
        depth = np.asarray(depth)
        self.max_depth = int(depth.max(initial=0))
        self.order = np.argsort(depth, kind="stable")
        self.start = np.concatenate(([0], np.cumsum(np.bincount(depth, minlength=self.max_depth + 1))))

    def _level(self, level):
        return self.order[self.start[level]:self.start[level + 1]]

    def factor(self, weights, delta):  # :732-760
        m = self.m
        diagonal = delta + np.bincount(self.first, weights=weights, minlength=m) + np.bincount(
            self.second, weights=weights, minlength=m)
        tree = self.child >= 0
        edge_w = np.bincount(self.child[tree], weights=weights[tree], minlength=m)
        pivot = diagonal
        mult = np.zeros(m)
        for level in range(self.max_depth, 0, -1):
            nodes = self._level(level)
            piv = np.maximum(pivot[nodes], TINY)
            edge = edge_w[nodes]
            mult[nodes] = -edge / piv
            np.add.at(pivot, self.parent[nodes], -(edge * edge) / piv)
        np.maximum(pivot, max(delta * 1.0e-8, TINY), out=pivot)
        self.pivot, self.mult = pivot, mult

    def solve(self, rhs):  # :762-776
        v = np.array(rhs, dtype=np.float64)
        for level in range(self.max_depth, 0, -1):
            nodes = self._level(level)
            np.add.at(v, self.parent[nodes], -self.mult[nodes] * v[nodes])
        v /= self.pivot
        for level in range(1, self.max_depth + 1):
            nodes = self._level(level)
            v[nodes] -= self.mult[nodes] * v[self.parent[nodes]]
        return v
