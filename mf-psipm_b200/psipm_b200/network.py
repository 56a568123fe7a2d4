"""Network LPs: the spanning forest and the device tree-plus-diagonal preconditioner.

The reference engages a special preconditioner when the constraint matrix is
a node-arc incidence matrix (every column one +1 and one -1) that is not
grounded (psipm_v3_1_hsd.py:2005-2032): ``NetworkTopology.from_incidence``
(:495-610) builds a BFS spanning forest from the highest-degree node of each
component, and ``TreePreconditioner`` (:715-785) factors the tree arcs plus
the full diagonal of ``A D A' + delta I`` exactly, level by level.

:func:`spanning_forest` computes the same forest (the same breadth-first
search, so the same parents).  :class:`GpuTreePreconditioner` keeps the
restricted incidence matrix, the forest and the factor on the device
(``psipm_set_tree`` / ``psipm_tree_factor``); its ``solve`` and the HSD
Newton solves (``solve_normal``, the HSD PCG with the tree as preconditioner)
run there.  The factor and a solve are bit-identical to the reference's.
"""

from __future__ import annotations

import time
from dataclasses import dataclass

import numpy as np
import scipy.sparse as sp
from scipy.sparse import csgraph

from . import _lib
from .device import NormalEquationsDevice

TINY = float(np.finfo(np.float64).tiny)


@dataclass
class Forest:
    rows: int
    first: np.ndarray       # row of each column's first entry
    second: np.ndarray      # row of its second entry
    tail: np.ndarray        # row of its +1
    head: np.ndarray        # row of its -1
    parent: np.ndarray      # BFS parent of each node, -1 at the roots
    depth: np.ndarray       # BFS depth
    tree_child: np.ndarray  # per column: the child end of a forest arc, or -1
    protected: np.ndarray   # one forest arc per tree relation (the lowest column index)
    root: int
    components: int


def spanning_forest(A) -> Forest:
    """BFS spanning forest of an incidence matrix (NetworkTopology.from_incidence)."""
    A = sp.csc_matrix(A)
    m, n = A.shape
    if n and not np.all(np.diff(A.indptr) == 2):
        raise ValueError("an incidence matrix has exactly two entries per column")
    lo = A.indptr[:-1]
    first = A.indices[lo].astype(np.int32)
    second = A.indices[lo + 1].astype(np.int32)
    v1, v2 = A.data[lo], A.data[lo + 1]
    if not (np.allclose(np.abs(v1), 1.0) and np.allclose(v1 + v2, 0.0)):
        raise ValueError("every column needs one +1 and one -1")
    tail = np.where(v1 > 0, first, second).astype(np.int32)
    head = np.where(v1 > 0, second, first).astype(np.int32)
    degree = np.bincount(first, minlength=m) + np.bincount(second, minlength=m)
    root = int(np.argmax(degree))
    graph = sp.csr_matrix((np.ones(2 * n, dtype=np.int8),
                           (np.concatenate((first, second)), np.concatenate((second, first)))), shape=(m, m))
    ncomp, labels = csgraph.connected_components(graph, directed=False, return_labels=True)
    if ncomp == 1:
        dist, pred = csgraph.shortest_path(graph, directed=False, indices=root, unweighted=True,
                                           return_predecessors=True)
    else:
        # a virtual node joined to the lowest-index node of highest degree in each
        # component; one search from it gives a shallow forest
        best = np.zeros(ncomp, dtype=degree.dtype)
        np.maximum.at(best, labels, degree)
        roots = np.full(ncomp, m, dtype=np.int64)
        cand = np.flatnonzero(degree == best[labels])
        np.minimum.at(roots, labels[cand], cand)
        link = sp.csr_matrix((np.ones(ncomp, dtype=np.int8), (np.zeros(ncomp, dtype=np.int32), roots)), shape=(1, m))
        aug = sp.vstack((sp.hstack((graph, link.T), format="csr"),
                         sp.hstack((link, sp.csr_matrix((1, 1))), format="csr")), format="csr")
        dist_a, pred_a = csgraph.shortest_path(aug, directed=False, indices=m, unweighted=True,
                                               return_predecessors=True)
        dist = dist_a[:m] - 1.0
        pred = pred_a[:m]
        pred[pred == m] = -1
        root = int(roots[0])
    if not np.all(np.isfinite(dist)):
        raise ValueError("the incidence graph is disconnected")
    parent = pred.astype(np.int32)
    parent[root] = -1
    depth = dist.astype(np.int32)
    tree_child = np.full(n, -1, dtype=np.int32)
    fc = parent[first] == second
    sc = parent[second] == first
    tree_child[fc] = first[fc]
    tree_child[sc] = second[sc]
    lowest = np.full(m, n, dtype=np.int64)
    arcs = np.flatnonzero(tree_child >= 0)
    np.minimum.at(lowest, tree_child[arcs], arcs)
    protected = np.zeros(n, dtype=bool)
    chosen = lowest[lowest < n]
    protected[chosen] = True
    if chosen.size != m - ncomp:
        raise RuntimeError("the forest does not span every component")
    return Forest(m, first, second, tail, head, parent, depth, tree_child, protected, root, int(ncomp))


class GpuTreePreconditioner:
    """HSD preconditioner protocol (``factor``, ``solve``, ``backend``,
    ``record_iterations``) with the tree-plus-diagonal factor on the device,
    for the active columns ``columns`` of an incidence matrix."""

    def __init__(self, forest: Forest, A, columns, device: int = 0, stats=None):
        columns = np.asarray(columns, dtype=np.int64)
        self.forest = forest
        self.columns = columns
        self.stats = stats
        self.A = sp.csc_matrix(A)[:, columns]
        self.dev = NormalEquationsDevice(self.A, device=device, precision=_lib.FP64)
        self.dev.set_tree(forest.parent, forest.depth, forest.tree_child[columns])
        self.impl = self  # hsd.HSDNewtonSystem reads impl.A / impl.dev
        self.factorizations = 0

    @property
    def backend(self) -> str:
        return "tree-laplacian-b200"

    def close(self) -> None:
        self.dev.close()

    def factor(self, weights, delta) -> float:
        started = time.perf_counter()
        w = np.asarray(weights, dtype=np.float64)
        self.dev.tree_factor(w, float(delta))
        # the PCG's operator A diag(w) A' + delta I
        self.dev.set_theta(1.0 / np.maximum(w, TINY), float(delta))
        self.factorizations += 1
        if self.stats is not None:
            self.stats.factorizations += 1
            self.stats.observe_core(self.columns.size)
        return time.perf_counter() - started

    def solve(self, rhs):
        return self.dev.apply(np.asarray(rhs, dtype=np.float64))

    def record_iterations(self, iterations, elapsed=0.0, converged=True) -> None:
        del iterations, elapsed, converged

    def record_solve(self, iterations, elapsed, converged) -> None:
        del iterations, elapsed, converged

    def solve_normal(self, r1, r2, rtol, max_iterations, deadline=np.inf):
        """``dy = H^{-1} (r2 - A D r1)`` by the HSD PCG with the tree as
        preconditioner and ``dx = D (r1 + A' dy)``, on the device.  Returns
        ``(dx, dy, iterations, matvecs, okay, elapsed)``."""
        from .kkt import _under_deadline

        started = time.perf_counter()
        dx, res = _under_deadline(self.dev, deadline,
                                  lambda: self.dev.solve(r1, r2, rtol, int(max_iterations), _lib.PCG_HSD))
        return dx, res.x, res.iterations, res.matvecs, bool(res.ok), time.perf_counter() - started
