"""Shared test helpers: fixtures -> LPs, exact reference solutions."""

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from psipm_b200.synthetic import StandardLP

NAMES = ("random_m300", "grid_20x25", "cover_m200")
OPTIONS = dict(full_preconditioner_row_threshold=10)


def lp_from(g) -> StandardLP:
    A = sp.csc_matrix((g["A_data"], g["A_indices"], g["A_indptr"]), shape=tuple(int(v) for v in g["A_shape"]))
    return StandardLP(c=g["c"], A=A, b=g["b"], u=g["u"], pos=g["pos"].astype(bool), box=g["box"].astype(bool))


def normal_matrix(A, theta, delta):
    """H = A diag(1/theta) A' + delta I (FP64, SciPy)."""
    w = 1.0 / theta
    return (A @ sp.diags(w) @ A.T + delta * sp.eye(A.shape[0])).tocsc()


def exact_direction(A, theta, delta, r1, r2):
    """Exact Newton direction of the reduced system by a sparse direct solve."""
    H = normal_matrix(A, theta, delta)
    w = r1 / theta
    rhs = r2 - A @ w
    dy = spla.spsolve(H, rhs)
    dx = w + (A.T @ dy) / theta
    return dx, dy


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
