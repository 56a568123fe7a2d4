"""Seeded synthetic LPs in the solver's canonical form.

Every instance is returned as a :class:`StandardLP` with the field meaning of
the reference's container (psipm_active_pool.py:111-148):

    min  c'v + obj_const   s.t.  A v = b,  0 <= v_j (j in pos),  v_j <= u_j (j in box)

Families (sizes are the defaults; every generator takes its sizes as
arguments so tests can run scaled-down copies):

* ``random_lp``      random standard-form LP, m=2,000, n=6,000, 5 nonzeros per
                     column at uniformly random distinct rows, values N(0,1);
                     feasible and bounded by construction (b = A x0, c = A'y0 + s0).
* ``grid_network``   min-cost flow on a directed 2-D grid (both arc orientations)
                     plus 10% random long-range arcs; integer costs U{1..100},
                     capacities U{10..1000} as upper bounds, b = A f for a random
                     feasible flow; one row per connected component grounded
                     (highest degree, lowest index).
* ``set_cover``      covering LP relaxation A x >= 1, 0 <= x <= 1 with 0/1
                     columns of U{2..10} distinct rows drawn by Zipf(1.2)
                     popularity, costs U{1,2,3}; brought to equality form with
                     one surplus column per row (the canonicalisation of
                     psipm_active_pool.py:340-447 for this row/column type).
* ``random_lp_batch``  uneven batch of ``random_lp`` instances, m ~ U{500..5000}, n = 3m.

Generators use ``numpy.random.default_rng(seed)`` only, so an instance is a
pure function of its arguments.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import List

import numpy as np
import scipy.sparse as sp


@dataclass
class StandardLP:
    """Canonical LP: ``min c'v + obj_const, A v = b, 0 <= v[pos], v[box] <= u[box]``."""

    c: np.ndarray
    A: sp.csc_matrix
    b: np.ndarray
    u: np.ndarray
    pos: np.ndarray
    box: np.ndarray
    obj_const: float = 0.0
    name: str = ""
    meta: dict = field(default_factory=dict)

    @property
    def shape(self):
        return self.A.shape


def _finish(A, b, c, u, name, meta) -> StandardLP:
    A = sp.csc_matrix(A)
    A.sum_duplicates()
    A.sort_indices()
    u = np.asarray(u, dtype=np.float64)
    pos = np.ones(A.shape[1], dtype=bool)
    return StandardLP(
        c=np.ascontiguousarray(c, dtype=np.float64),
        A=A,
        b=np.ascontiguousarray(b, dtype=np.float64),
        u=u,
        pos=pos,
        box=pos & np.isfinite(u),
        obj_const=0.0,
        name=name,
        meta=meta,
    )


def random_lp(m: int = 2000, n: int = 6000, per_column: int = 5, seed: int = 0) -> StandardLP:
    """Random feasible, bounded standard-form LP (all ``x >= 0``, no upper bounds)."""
    rng = np.random.default_rng(seed)
    per_column = min(per_column, m)
    # distinct rows per column: argsort of uniform keys, first ``per_column``
    rows = np.argsort(rng.random((n, m)), axis=1)[:, :per_column] if m * n <= 5e7 else None
    if rows is None:
        rows = np.empty((n, per_column), dtype=np.int64)
        for j in range(n):
            rows[j] = rng.choice(m, per_column, replace=False)
    values = rng.standard_normal((n, per_column))
    indptr = np.arange(0, n * per_column + 1, per_column, dtype=np.int64)
    A = sp.csc_matrix((values.ravel(), rows.ravel(), indptr), shape=(m, n))
    x0 = rng.uniform(0.5, 1.5, n)
    b = A @ x0
    y0 = rng.standard_normal(m)
    s0 = rng.uniform(0.1, 1.0, n)
    c = A.T @ y0 + s0
    return _finish(A, b, c, np.full(n, np.inf), f"random_lp_m{m}_n{n}_s{seed}",
                   dict(family="random_lp", m=m, n=n, seed=seed))


def random_lp_dense(m: int = 1200, n: int = 3600, dense: int = 4, dense_nnz: int = 1100, per_column: int = 5,
                    seed: int = 0) -> StandardLP:
    """``random_lp`` whose first ``dense`` columns hold ``dense_nnz`` entries each.

    Such columns (>= 1,024 entries, large potential clique in A A^T) are the
    ones the reference leaves out of the factor and corrects for by Woodbury
    (psipm_active_pool.py:691-718, 906-956); the other families have none.
    """
    rng = np.random.default_rng(seed)
    base = random_lp(m, n, per_column, seed)
    A = base.A.tolil()
    for j in range(min(dense, n)):
        rows = rng.choice(m, min(dense_nnz, m), replace=False)
        A[:, j] = 0.0
        A[rows, j] = rng.standard_normal(rows.size)[:, None]
    A = sp.csc_matrix(A)
    x0 = rng.uniform(0.5, 1.5, n)
    b = A @ x0
    y0 = rng.standard_normal(m)
    s0 = rng.uniform(0.1, 1.0, n)
    c = A.T @ y0 + s0
    return _finish(A, b, c, np.full(n, np.inf), f"random_lp_dense_m{m}_n{n}_d{dense}_s{seed}",
                   dict(family="random_lp_dense", m=m, n=n, dense=dense, dense_nnz=dense_nnz, seed=seed))


def _ground(A: sp.csc_matrix) -> np.ndarray:
    """Rows to keep after removing one row per connected component.

    The removed row of a component is its highest-degree node, lowest index
    among ties, which is the grounding rule of batch_test_vlsi_spectral.py:242-287.
    """
    m = A.shape[0]
    import scipy.sparse.csgraph as csgraph

    Ab =sp.csc_matrix((np.ones(A.nnz), A.indices, A.indptr), shape=A.shape)
    adjacency = (Ab @ Ab.T).tocsr()
    ncomp, labels = csgraph.connected_components(adjacency, directed=False)
    degree = np.diff(A.tocsr().indptr)
    removed = np.empty(ncomp, dtype=np.int64)
    order = np.lexsort((np.arange(m), -degree, labels))
    first = np.searchsorted(labels[order], np.arange(ncomp))
    removed[:] = order[first]
    keep = np.ones(m, dtype=bool)
    keep[removed] = False
    return np.flatnonzero(keep)


def grid_network(rows: int = 200, cols: int = 250, long_range: float = 0.10, seed: int = 1000,
                 ground: bool = True) -> StandardLP:
    """Grounded min-cost flow LP on a directed grid plus random long-range arcs
    (``ground=False`` keeps every node row: a pure incidence matrix, the case
    of the reference's network preconditioner)."""
    rng = np.random.default_rng(seed)
    nodes = rows * cols
    idx = np.arange(nodes).reshape(rows, cols)
    right = np.stack([idx[:, :-1].ravel(), idx[:, 1:].ravel()], axis=1)
    down = np.stack([idx[:-1, :].ravel(), idx[1:, :].ravel()], axis=1)
    grid = np.concatenate([right, down])
    arcs = np.concatenate([grid, grid[:, ::-1]])
    extra = int(round(long_range * arcs.shape[0]))
    tail = rng.integers(0, nodes, extra)
    head = rng.integers(0, nodes - 1, extra)
    head = head + (head >= tail)  # no self loops
    arcs = np.concatenate([arcs, np.stack([tail, head], axis=1)])
    narcs = arcs.shape[0]
    data = np.concatenate([np.ones(narcs), -np.ones(narcs)])
    r = np.concatenate([arcs[:, 0], arcs[:, 1]])
    cidx = np.concatenate([np.arange(narcs), np.arange(narcs)])
    A_full = sp.csc_matrix((data, (r, cidx)), shape=(nodes, narcs))
    cost = rng.integers(1, 101, narcs).astype(np.float64)
    cap = rng.integers(10, 1001, narcs).astype(np.float64)
    flow = np.floor(rng.random(narcs) * (cap + 1.0))
    b_full = A_full @ flow
    keep = _ground(A_full) if ground else np.arange(nodes)
    A = A_full[keep, :]
    b = b_full[keep]
    return _finish(A, b, cost, cap, f"grid_network_{rows}x{cols}_s{seed}",
                   dict(family="grid_network", rows=rows, cols=cols, arcs=narcs,
                        nodes=nodes, seed=seed, grounded=int(nodes - keep.size)))


def set_cover(m: int = 4000, n: int = 1_000_000, kmin: int = 2, kmax: int = 10,
              zipf: float = 1.2, seed: int = 2000) -> StandardLP:
    """Covering LP ``A x >= 1, 0 <= x <= 1`` in equality form with surplus columns."""
    rng = np.random.default_rng(seed)
    permutation = rng.permutation(m)
    weights = np.arange(1, m + 1, dtype=np.float64) ** (-zipf)
    cdf = np.cumsum(weights)
    cdf /= cdf[-1]
    k = rng.integers(kmin, kmax + 1, n)
    draws = 4 * kmax
    sample = np.searchsorted(cdf, rng.random((n, draws)), side="right")
    sample = np.minimum(sample, m - 1)
    rows_list: List[np.ndarray] = []
    counts = np.empty(n, dtype=np.int64)
    # first k distinct draws per column (in draw order)
    order = np.argsort(sample, axis=1, kind="stable")
    sorted_sample = np.take_along_axis(sample, order, axis=1)
    first = np.ones_like(sorted_sample, dtype=bool)
    first[:, 1:] = sorted_sample[:, 1:] != sorted_sample[:, :-1]
    is_first = np.zeros_like(first)
    np.put_along_axis(is_first, order, first, axis=1)
    rank_in_draw = np.cumsum(is_first, axis=1)
    take = is_first & (rank_in_draw <= k[:, None])
    counts[:] = take.sum(axis=1)
    short = np.flatnonzero(counts < k)
    rows_flat = sample[take]
    col_flat = np.repeat(np.arange(n), counts)
    if short.size:
        extra_rows = []
        extra_cols = []
        for j in short:
            have = set(sample[j][take[j]].tolist())
            while len(have) < k[j]:
                have.add(int(min(np.searchsorted(cdf, rng.random(), side="right"), m - 1)))
            new = sorted(have - set(sample[j][take[j]].tolist()))
            extra_rows.extend(new)
            extra_cols.extend([j] * len(new))
        rows_flat = np.concatenate([rows_flat, np.asarray(extra_rows, dtype=np.int64)])
        col_flat = np.concatenate([col_flat, np.asarray(extra_cols, dtype=np.int64)])
    rows_flat = permutation[rows_flat]
    A_cover = sp.csc_matrix((np.ones(rows_flat.size), (rows_flat, col_flat)), shape=(m, n))
    cost = rng.integers(1, 4, n).astype(np.float64)
    # a'x - t = 0, t in [1, inf)  ->  t = 1 + v, v >= 0:  [A, -I][x; v] = 1
    surplus = -sp.eye(m, format="csc")
    A = sp.hstack([A_cover, surplus], format="csc")
    c = np.concatenate([cost, np.zeros(m)])
    u = np.concatenate([np.ones(n), np.full(m, np.inf)])
    b = np.ones(m)
    return _finish(A, b, c, u, f"set_cover_m{m}_n{n}_s{seed}",
                   dict(family="set_cover", m=m, n=n, seed=seed))


def random_lp_batch(count: int = 256, mmin: int = 500, mmax: int = 5000, seed: int = 4000) -> List[StandardLP]:
    """Uneven batch of ``random_lp`` instances with ``m ~ U{mmin..mmax}``, ``n = 3m``."""
    rng = np.random.default_rng(seed)
    sizes = rng.integers(mmin, mmax + 1, count)
    return [random_lp(int(mm), 3 * int(mm), seed=seed + 1 + i) for i, mm in enumerate(sizes)]


CONFIGS = {
    "C0": dict(family="random_lp", kwargs=dict(m=2000, n=6000, seed=0)),
    "C1": dict(family="grid_network", kwargs=dict(rows=200, cols=250, seed=1000)),
    "C2": dict(family="set_cover", kwargs=dict(m=4000, n=1_000_000, seed=2000)),
    "C3": dict(family="grid_network", kwargs=dict(rows=1000, cols=1000, seed=3000)),
}


def make(config: str, **overrides) -> StandardLP:
    """Instance of a named configuration, optionally with overridden sizes."""
    spec = CONFIGS[config]
    kwargs = dict(spec["kwargs"])
    kwargs.update(overrides)
    return globals()[spec["family"]](**kwargs)
