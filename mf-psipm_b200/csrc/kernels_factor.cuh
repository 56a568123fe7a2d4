// Numeric factorisation of the active-core normal matrix on the device.
//
// F1  (assembly, psipm_stable_preconditioner.py:373-395 + psipm_active_pool.py:999-1006)
//     P_e = sum_{contributions} (a_ik a_jk) w_k over the fixed symbolic pattern,
//     diagonal fixed to  core_ii + (max(diag_full_i - core_ii, 0) + delta),
//     then Jacobi scaling to unit diagonal (psipm_active_pool.py:850-853).
// F2  (multifrontal Cholesky, one launch per level of the supernodal tree):
//     each block owns one front: it scatters the scaled entries (+ the
//     diagonal shift), extend-adds the children's update matrices, runs the
//     partial Cholesky of the pivot columns, writes its own update matrix and
//     the solve panel G = [L11^-1 ; L21 L11^-1] (row-major r x c) used by the
//     triangular solves.  A non-positive or non-finite pivot sets `fail`.
#pragma once

#include "common.cuh"

namespace psipm {

constexpr int kFactorThreads = 256;

template <typename T>
struct FactorArgs {
    // symbolic
    const int* sn_first = nullptr;
    const long long* sn_rowptr = nullptr;
    const long long* panel_off = nullptr;
    const long long* update_off = nullptr;
    const long long* uvec_off = nullptr;
    const int* child_ptr = nullptr;
    const int* child_list = nullptr;
    const int* relind = nullptr;
    const long long* sn_entptr = nullptr;
    const int* ent_col = nullptr;     // local column
    const int* ent_rowpos = nullptr;  // row position in the supernode
    // numeric inputs
    const T* ms = nullptr;  // scaled entries
    double eta = 0.0;       // diagonal shift
    // outputs / work
    T* G = nullptr;
    T* GT = nullptr;  // transposed panels (c x r row-major), same offsets as G
    T* update = nullptr;
    T* front = nullptr;                  // level workspace
    const long long* front_off = nullptr;  // per supernode, within the level workspace
    int* fail = nullptr;
};

// ---- F1 -----------------------------------------------------------------
// P_e for every entry; core_ii for diagonal entries (sequential per entry in
// core-column order, the order of the reference's CSC matvec).
__global__ void k_assemble_entries(long long nent, const long long* __restrict__ ent_ptr,
                                   const int* __restrict__ contrib_col,
                                   const double* __restrict__ contrib_val,
                                   const long long* __restrict__ core, const double* __restrict__ w,
                                   double* __restrict__ pval) {
    long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (e >= nent) return;
    double acc = 0.0;
    for (long long c = ent_ptr[e]; c < ent_ptr[e + 1]; ++c)
        acc = __dadd_rn(acc, __dmul_rn(contrib_val[c], w[core[contrib_col[c]]]));
    pval[e] = acc;
}

// Diagonal: P_ii = core_ii + (drop_i + delta), drop_i = max(diag_full_i - core_ii, 0);
// dscp[k] = 1/sqrt(P_kk) (1 where P_kk <= 0), permuted order.
__global__ void k_diag_fix(int m, const long long* __restrict__ diag_entry, const int* __restrict__ perm,
                           const double* __restrict__ diag_full, double delta, double* __restrict__ pval,
                           double* __restrict__ dscp) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m) return;
    const long long e = diag_entry[k];
    const double core_ii = pval[e];
    const double drop = fmax(__dadd_rn(diag_full[perm[k]], -core_ii), 0.0);
    const double v = __dadd_rn(core_ii, __dadd_rn(drop, delta));
    pval[e] = v;
    dscp[k] = v > 0.0 ? 1.0 / sqrt(v) : 1.0;
}

template <typename T>
__global__ void k_scale_entries(long long nent, const int* __restrict__ ent_row,
                                const int* __restrict__ ent_colg, const double* __restrict__ pval,
                                const double* __restrict__ dscp, T* __restrict__ ms) {
    long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (e >= nent) return;
    ms[e] = (T)(pval[e] * (dscp[ent_row[e]] * dscp[ent_colg[e]]));
}

template <typename T>
__global__ void k_cast(long long n, const double* __restrict__ in, T* __restrict__ out) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) out[i] = (T)in[i];
}

// ---- F2: one block per supernode of a level ---------------------------------
template <typename T>
__global__ void __launch_bounds__(kFactorThreads) k_factor_level(FactorArgs<T> a, const int* level_sn) {
    const int s = level_sn[blockIdx.x];
    const int tid = threadIdx.x, bs = blockDim.x;
    const int first = a.sn_first[s];
    const int c = a.sn_first[s + 1] - first;
    const int r = (int)(a.sn_rowptr[s + 1] - a.sn_rowptr[s]);
    T* F = a.front + a.front_off[s];  // column-major r x r, lower triangle used
    __shared__ T piv;
    __shared__ int bad;
    if (tid == 0) bad = 0;
    // zero the lower triangle
    const long long rr = (long long)r * r;
    for (long long q = tid; q < rr; q += bs) F[q] = (T)0;
    __syncthreads();
    // scatter this supernode's entries (+ shift on the diagonal)
    for (long long e = a.sn_entptr[s] + tid; e < a.sn_entptr[s + 1]; e += bs) {
        const int col = a.ent_col[e], row = a.ent_rowpos[e];
        T v = a.ms[e];
        if (row == col) v += (T)a.eta;
        F[(long long)col * r + row] = v;
    }
    __syncthreads();
    // extend-add the children's update matrices (fixed child order)
    for (int ci = a.child_ptr[s]; ci < a.child_ptr[s + 1]; ++ci) {
        const int ch = a.child_list[ci];
        const int rc = (int)(a.uvec_off[ch + 1] - a.uvec_off[ch]);
        const T* U = a.update + a.update_off[ch];
        const int* ri = a.relind + a.uvec_off[ch];
        const long long n2 = (long long)rc * rc;
        for (long long q = tid; q < n2; q += bs) {
            const int ia = (int)(q % rc), ib = (int)(q / rc);
            if (ia >= ib) F[(long long)ri[ib] * r + ri[ia]] += U[q];
        }
        __syncthreads();
    }
    // partial right-looking Cholesky of the first c columns
    for (int k = 0; k < c; ++k) {
        if (tid == 0) {
            T d = F[(long long)k * r + k];
            if (!(d > (T)0) || !isfinite((double)d)) {
                bad = 1;
                d = (T)1;
            }
            d = sqrt(d);
            F[(long long)k * r + k] = d;
            piv = d;
        }
        __syncthreads();
        const T inv = (T)1 / piv;
        T* colk = F + (long long)k * r;
        for (int i = k + 1 + tid; i < r; i += bs) colk[i] *= inv;
        __syncthreads();
        const int rem = r - k - 1;
        const long long n2 = (long long)rem * rem;
        for (long long q = tid; q < n2; q += bs) {
            const int ii = (int)(q % rem), jj = (int)(q / rem);
            if (ii >= jj) {
                const int i = k + 1 + ii, j = k + 1 + jj;
                F[(long long)j * r + i] -= colk[i] * colk[j];
            }
        }
        __syncthreads();
    }
    if (tid == 0 && bad) atomicExch(a.fail, 1);
    // update matrix: F[c:r, c:r] (column-major rc x rc)
    const int rc = r - c;
    if (rc > 0) {
        T* U = a.update + a.update_off[s];
        const long long n2 = (long long)rc * rc;
        for (long long q = tid; q < n2; q += bs) {
            const int ia = (int)(q % rc), ib = (int)(q / rc);
            U[q] = ia >= ib ? F[(long long)(c + ib) * r + (c + ia)] : (T)0;
        }
    }
    // G_top = L11^{-1} (row-major c x c, lower), row by row
    T* G = a.G + a.panel_off[s];
    for (int i = 0; i < c; ++i) {
        const T lii = F[(long long)i * r + i];
        for (int j = tid; j < c; j += bs) {
            T v;
            if (j > i) {
                v = (T)0;
            } else if (j == i) {
                v = (T)1 / lii;
            } else {
                T sum = 0;
                for (int k = j; k < i; ++k) sum += F[(long long)k * r + i] * G[(long long)k * c + j];
                v = -sum / lii;
            }
            G[(long long)i * c + j] = v;
        }
        __syncthreads();
    }
    // G_bot = L21 L11^{-1}: row i (c <= i < r), column j: sum_{k>=j} L[i,k] Linv[k,j]
    const long long nb = (long long)rc * c;
    for (long long q = tid; q < nb; q += bs) {
        const int i = c + (int)(q / c), j = (int)(q % c);
        T sum = 0;
        for (int k = j; k < c; ++k) sum += F[(long long)k * r + i] * G[(long long)k * c + j];
        G[(long long)i * c + j] = sum;
    }
    __syncthreads();
    // GT = G^T (c x r, row-major)
    T* GT = a.GT + a.panel_off[s];
    const long long nrc = (long long)r * c;
    for (long long q = tid; q < nrc; q += bs) {
        const int j = (int)(q / r), i = (int)(q % r);
        GT[q] = G[(long long)i * c + j];
    }
}

}  // namespace psipm

namespace psipm {

// ===========================================================================
// Large fronts: the front is processed by many CTAs, one kernel per step of
// a blocked right-looking Cholesky (block width kNB), then the solve panel
// G = [I; L21] L11^{-1} by a row-parallel blocked triangular solve.
// The front F is column-major r x r (lower triangle used).
constexpr int kNB = 64;

// scatter this supernode's scaled entries (+ shift on the diagonal)
template <typename T>
__global__ void k_front_scatter(T* __restrict__ F, int r, long long e0, long long e1,
                                const int* __restrict__ ent_col, const int* __restrict__ ent_rowpos,
                                const T* __restrict__ ms, double eta) {
    for (long long e = e0 + blockIdx.x * (long long)blockDim.x + threadIdx.x; e < e1;
         e += (long long)gridDim.x * blockDim.x) {
        const int col = ent_col[e], row = ent_rowpos[e];
        T v = ms[e];
        if (row == col) v += (T)eta;
        F[(long long)col * r + row] = v;
    }
}

// F += child's update matrix (lower part) at its relative indices
template <typename T>
__global__ void k_front_extend_add(T* __restrict__ F, int r, const T* __restrict__ U, int rc,
                                   const int* __restrict__ ri) {
    const long long n2 = (long long)rc * rc;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n2;
         q += (long long)gridDim.x * blockDim.x) {
        const int ia = (int)(q % rc), ib = (int)(q / rc);
        if (ia >= ib) F[(long long)ri[ib] * r + ri[ia]] += U[q];
    }
}

// Cholesky of the diagonal block F[k0:k0+kb, k0:k0+kb] in shared memory (1 CTA)
template <typename T>
__global__ void __launch_bounds__(256) k_potrf_diag(T* __restrict__ F, int r, int k0, int kb, int* fail) {
    __shared__ T D[kNB][kNB + 1];
    __shared__ int bad;
    const int tid = threadIdx.x;
    if (tid == 0) bad = 0;
    for (int q = tid; q < kb * kb; q += blockDim.x) {
        const int i = q % kb, j = q / kb;
        D[i][j] = i >= j ? F[(long long)(k0 + j) * r + (k0 + i)] : (T)0;
    }
    __syncthreads();
    for (int k = 0; k < kb; ++k) {
        if (tid == 0) {
            T d = D[k][k];
            if (!(d > (T)0) || !isfinite((double)d)) {
                bad = 1;
                d = (T)1;
            }
            D[k][k] = sqrt(d);
        }
        __syncthreads();
        const T inv = (T)1 / D[k][k];
        for (int i = k + 1 + tid; i < kb; i += blockDim.x) D[i][k] *= inv;
        __syncthreads();
        const int rem = kb - k - 1;
        for (int q = tid; q < rem * rem; q += blockDim.x) {
            const int i = k + 1 + q % rem, j = k + 1 + q / rem;
            if (i >= j) D[i][j] -= D[i][k] * D[j][k];
        }
        __syncthreads();
    }
    for (int q = tid; q < kb * kb; q += blockDim.x) {
        const int i = q % kb, j = q / kb;
        if (i >= j) F[(long long)(k0 + j) * r + (k0 + i)] = D[i][j];
    }
    if (tid == 0 && bad) atomicExch(fail, 1);
}

// panel: F[i, k0:k0+kb] <- F[i, k0:k0+kb] L_kk^{-T} for rows i >= k0+kb
// (one thread per row, 64 rows per CTA; dynamic shared memory 2 x 64 x 65 T)
constexpr int kTrsmRows = 64;
template <typename T>
__global__ void __launch_bounds__(kTrsmRows) k_trsm_panel(T* __restrict__ F, int r, int k0, int kb) {
    extern __shared__ __align__(16) unsigned char smem_f[];
    T* Lk = reinterpret_cast<T*>(smem_f);  // [64][65]
    T* X = Lk + kNB * (kNB + 1);           // [64][65]
    const int tid = threadIdx.x;
    const int row0 = k0 + kb + blockIdx.x * kTrsmRows;
    for (int q = tid; q < kb * kb; q += blockDim.x) {
        const int i = q % kb, j = q / kb;
        Lk[i * (kNB + 1) + j] = F[(long long)(k0 + j) * r + (k0 + i)];
    }
    const int i = row0 + tid;
    for (int j = 0; j < kb; ++j) X[tid * (kNB + 1) + j] = i < r ? F[(long long)(k0 + j) * r + i] : (T)0;
    __syncthreads();
    if (i < r) {
        T* x = X + tid * (kNB + 1);
        for (int j = 0; j < kb; ++j) {
            T s = x[j];
            const T* lj = Lk + j * (kNB + 1);
            for (int l = 0; l < j; ++l) s -= x[l] * lj[l];
            x[j] = s / lj[j];
        }
        for (int j = 0; j < kb; ++j) F[(long long)(k0 + j) * r + i] = x[j];
    }
}

// trailing update of the lower triangle: F[I, J] -= P[I] P[J]^T for the
// rows/cols >= k0+kb, P = F[:, k0:k0+kb]; 64x64 output tiles, 4x4 per thread
template <typename T>
__global__ void __launch_bounds__(256) k_syrk_update(T* __restrict__ F, int r, int k0, int kb, int ntile) {
    extern __shared__ __align__(16) unsigned char smem_f[];
    T(*Pi)[kNB + 1] = reinterpret_cast<T(*)[kNB + 1]>(smem_f);  // [row in tile][k]
    T(*Pj)[kNB + 1] = Pi + kNB;
    const int base = k0 + kb;
    // lower-triangular tile index -> (ti, tj), ti >= tj
    const int t = blockIdx.x;
    int ti = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
    while ((ti + 1) * (ti + 2) / 2 <= t) ++ti;
    while (ti * (ti + 1) / 2 > t) --ti;
    const int tj = t - ti * (ti + 1) / 2;
    if (ti >= ntile) return;
    const int i0 = base + ti * 64, j0 = base + tj * 64;
    const int tid = threadIdx.x;
    for (int q = tid; q < 64 * kb; q += blockDim.x) {
        const int a = q % 64, k = q / 64;
        const int ii = i0 + a, jj = j0 + a;
        Pi[a][k] = ii < r ? F[(long long)(k0 + k) * r + ii] : (T)0;
        Pj[a][k] = jj < r ? F[(long long)(k0 + k) * r + jj] : (T)0;
    }
    __syncthreads();
    // thread (tx, ty): rows i0 + tx + 16*a, cols j0 + ty + 16*b
    const int tx = tid % 16, ty = tid / 16;
    T acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = 0;
    for (int k = 0; k < kb; ++k) {
        T pi[4], pj[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) pi[a] = Pi[tx + 16 * a][k];
#pragma unroll
        for (int b = 0; b < 4; ++b) pj[b] = Pj[ty + 16 * b][k];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) acc[a][b] += pi[a] * pj[b];
    }
#pragma unroll
    for (int b = 0; b < 4; ++b) {
        const int j = j0 + ty + 16 * b;
        if (j >= r) continue;
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const int i = i0 + tx + 16 * a;
            if (i < r && i >= j) F[(long long)j * r + i] -= acc[a][b];
        }
    }
}

// update matrix U = F[c:r, c:r] (column-major rc x rc, lower part)
template <typename T>
__global__ void k_extract_update(const T* __restrict__ F, int r, int c, T* __restrict__ U) {
    const int rc = r - c;
    const long long n2 = (long long)rc * rc;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n2;
         q += (long long)gridDim.x * blockDim.x) {
        const int ia = (int)(q % rc), ib = (int)(q / rc);
        U[q] = ia >= ib ? F[(long long)(c + ib) * r + (c + ia)] : (T)0;
    }
}

// G (row-major r x c) solves X L11 = [I_c ; L21] row-block by row-block:
// 32 rows per CTA, column blocks of 32 from right to left.
template <typename T>
__global__ void __launch_bounds__(256) k_g_trsm(const T* __restrict__ F, int r, int c, T* __restrict__ G) {
    __shared__ T Xs[32][33];
    __shared__ T Ls[32][33];
    __shared__ T Acc[32][33];
    __shared__ T Ld[32][33];
    const int tid = threadIdx.x;
    const int row0 = blockIdx.x * 32;
    const int nrows = min(32, r - row0);
    const int nblk = (c + 31) / 32;
    const int maxrow = row0 + nrows - 1;
    // rows < c are rows of L11^{-1}: zero right of the diagonal
    const int last_blk = maxrow < c ? maxrow / 32 : nblk - 1;
    // zero the blocks entirely right of the diagonal for top rows
    for (int jb = last_blk + 1; jb < nblk; ++jb)
        for (int q = tid; q < 32 * 32; q += blockDim.x) {
            const int a = q / 32, j = jb * 32 + q % 32;
            if (a < nrows && j < c) G[(long long)(row0 + a) * c + j] = (T)0;
        }
    const int tr = tid / 8, tc = (tid % 8) * 4;  // this thread: row tr, cols tc..tc+3
    for (int jb = last_blk; jb >= 0; --jb) {
        const int jc0 = jb * 32;
        const int jn = min(32, c - jc0);
        // acc = B[rows, J]
        T acc[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int i = row0 + tr, j = jc0 + tc + u;
            T b = 0;
            if (tr < nrows && j < c) b = i < c ? (T)(i == j ? 1 : 0) : F[(long long)j * r + i];
            acc[u] = b;
        }
        // acc -= X[rows, k] L11[k, J] over k >= jc0 + 32 (already solved)
        for (int k0 = jc0 + 32; k0 < c; k0 += 32) {
            __syncthreads();
            for (int q = tid; q < 32 * 32; q += blockDim.x) {
                const int a = q / 32, kk = q % 32;
                const int i = row0 + a, k = k0 + kk;
                Xs[a][kk] = (a < nrows && k < c) ? G[(long long)i * c + k] : (T)0;
                const int j = jc0 + a;  // here a indexes the column j of the block
                Ls[kk][a] = (j < c && k < c) ? F[(long long)j * r + k] : (T)0;  // L11[k, j]
            }
            __syncthreads();
#pragma unroll 8
            for (int kk = 0; kk < 32; ++kk) {
                const T xv = Xs[tr][kk];
#pragma unroll
                for (int u = 0; u < 4; ++u) acc[u] -= xv * Ls[kk][tc + u];
            }
        }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < 4; ++u) Acc[tr][tc + u] = acc[u];
        for (int q = tid; q < 32 * 32; q += blockDim.x) {
            const int a = q / 32, b = q % 32;  // L11[jc0+a, jc0+b]
            Ld[a][b] = (a < jn && b < jn && a >= b) ? F[(long long)(jc0 + b) * r + (jc0 + a)] : (T)0;
        }
        __syncthreads();
        // in-block back substitution, one row per thread: x_j = (acc_j - sum_{l>j} x_l L[l,j]) / L[j,j]
        if (tid < nrows) {
            for (int j = jn - 1; j >= 0; --j) {
                T s = Acc[tid][j];
                for (int l = j + 1; l < jn; ++l) s -= Acc[tid][l] * Ld[l][j];
                Acc[tid][j] = s / Ld[j][j];
            }
        }
        __syncthreads();
        for (int q = tid; q < 32 * 32; q += blockDim.x) {
            const int a = q / 32, b = q % 32;
            if (a < nrows && b < jn) G[(long long)(row0 + a) * c + jc0 + b] = Acc[a][b];
        }
    }
}


// transposed copy of a big supernode's panel: GT (c x r, row-major) = G^T
template <typename T>
__global__ void k_transpose_panel(const T* __restrict__ G, int r, int c, T* __restrict__ GT) {
    __shared__ T tile[32][33];
    const int bi = blockIdx.y * 32, bj = blockIdx.x * 32;  // rows of G, cols of G
    for (int y = threadIdx.y; y < 32; y += blockDim.y) {
        const int i = bi + y, j = bj + threadIdx.x;
        tile[y][threadIdx.x] = (i < r && j < c) ? G[(long long)i * c + j] : (T)0;
    }
    __syncthreads();
    for (int y = threadIdx.y; y < 32; y += blockDim.y) {
        const int j = bj + y, i = bi + threadIdx.x;
        if (j < c && i < r) GT[(long long)j * r + i] = tile[threadIdx.x][y];
    }
}

}  // namespace psipm
