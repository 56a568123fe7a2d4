"""Algorithmic byte counts of the inner-solve kernels (the roofline numerator).

For one CSR SpMV ``y = M x`` with R rows, C columns, Z stored entries,
values of ``bv`` bytes and 4-byte indices, reading x once and writing y once:

    B_spmv = Z (bv + 4) + 4 (R + 1) + bv C + bv R

One operator product ``H p = A (w o (A' p)) + delta p`` as the fused pair:

    B_Hp = B_spmv(A': R=n, C=m) + bv n   (w, read in the epilogue)
         + B_spmv(A:  R=m, C=n) + bv m   (p, for delta p)

One preconditioner application (two triangular sweeps over L's stored
entries, the permutation and the Jacobi scaling):

    B_prec = 2 (nnz(L) (bv + 4) + 4 (m + 1)) + 2 bv m

and the PCG vector updates of one iteration, about ``10 bv m``.
"""

from __future__ import annotations


def spmv_bytes(rows: int, cols: int, nnz: int, bv: int) -> float:
    return nnz * (bv + 4) + 4 * (rows + 1) + bv * cols + bv * rows


def hp_bytes(m: int, n: int, nnz: int, bv: int = 8) -> float:
    return spmv_bytes(n, m, nnz, bv) + bv * n + spmv_bytes(m, n, nnz, bv) + bv * m


def prec_bytes(m: int, nnz_l: int, bv: int = 8) -> float:
    return 2 * (nnz_l * (bv + 4) + 4 * (m + 1)) + 2 * bv * m


def pcg_launch_bytes(m: int, n: int, nnz: int, nnz_l: int, iterations: int, matvecs: int,
                     applies: int, bv: int = 8) -> float:
    """Algorithmic bytes of one persistent PCG launch."""
    return (matvecs * hp_bytes(m, n, nnz, bv) + applies * prec_bytes(m, nnz_l, bv)
            + iterations * 10 * bv * m)
