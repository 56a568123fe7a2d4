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
    T* dinv = nullptr;                   // D_J^T blocks of the big front being factored
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
    if (tid == 0 && bad) atomicOr(a.fail, 1);
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

// Cholesky of the diagonal block F[k0:k0+kb, k0:k0+kb] in shared memory (1 CTA).
// Right-looking with the columns left unscaled until the end, so each step
// is one update and one barrier: step k subtracts D[i][k] D[j][k] / d_k from
// the trailing triangle (d_k = D[k][k], final after step k - 1; every thread
// reads it and takes the same branch), then L[i][k] = D[i][k] / sqrt(d_k).
// A non-positive or non-finite pivot sets `fail` and is replaced by 1.
template <typename T>
__global__ void __launch_bounds__(256) k_potrf_diag(T* __restrict__ F, int r, int k0, int kb, int* fail) {
    __shared__ T D[kNB][kNB + 1];
    __shared__ T piv[kNB];
    const int tid = threadIdx.x;
    for (int q = tid; q < kb * kb; q += blockDim.x) {
        const int i = q % kb, j = q / kb;
        D[i][j] = i >= j ? F[(long long)(k0 + j) * r + (k0 + i)] : (T)0;
    }
    __syncthreads();
    bool bad = false;
    for (int k = 0; k < kb; ++k) {
        T d = D[k][k];
        if (!(d > (T)0) || !isfinite((double)d)) {
            bad = true;
            d = (T)1;
        }
        if (tid == 0) piv[k] = d;
        const T invd = (T)1 / d;
        const int rem = kb - k - 1;
        for (int q = tid; q < rem * rem; q += blockDim.x) {
            const int i = k + 1 + q % rem, j = k + 1 + q / rem;
            if (i >= j) D[i][j] -= D[i][k] * invd * D[j][k];
        }
        __syncthreads();
    }
    for (int q = tid; q < kb * kb; q += blockDim.x) {
        const int i = q % kb, j = q / kb;
        if (i >= j) {
            const T sj = sqrt(piv[j]);
            F[(long long)(k0 + j) * r + (k0 + i)] = i == j ? sj : D[i][j] / sj;
        }
    }
    if (tid == 0 && bad) atomicOr(fail, 1);
}

// panel: F[i, k0:k0+kb] <- F[i, k0:k0+kb] L_kk^{-T} for rows i >= k0+kb
// (one thread per row, 64 rows per CTA; dynamic shared memory 64 x 65 T).
// Each thread keeps its row in registers and eliminates column by column
// (x_j = b_j / L_jj, then b_l -= x_j L_lj for every l > j): 64 dependent
// steps whose 63, 62, ... updates are independent.  Past kb the block is the
// identity, so the fully unrolled loop serves every kb <= 64.
constexpr int kTrsmRows = 64;
template <typename T>
__global__ void __launch_bounds__(kTrsmRows) k_trsm_panel(T* __restrict__ F, int r, int k0, int kb) {
    extern __shared__ __align__(16) unsigned char smem_f[];
    T* Lk = reinterpret_cast<T*>(smem_f);  // Lk[l * 65 + j] = L[l][j]
    __shared__ T rdiag[kNB];
    const int tid = threadIdx.x;
    const int row0 = k0 + kb + blockIdx.x * kTrsmRows;
    for (int q = tid; q < kNB * kNB; q += blockDim.x) {
        const int l = q % kNB, j = q / kNB;
        T v;
        if (l < kb && j < kb)
            v = l >= j ? F[(long long)(k0 + j) * r + (k0 + l)] : (T)0;
        else
            v = l == j ? (T)1 : (T)0;
        Lk[l * (kNB + 1) + j] = v;
    }
    const int i = row0 + tid;
    T x[kNB];
#pragma unroll
    for (int j = 0; j < kNB; ++j) x[j] = (i < r && j < kb) ? F[(long long)(k0 + j) * r + i] : (T)0;
    __syncthreads();
    if (tid < kNB) rdiag[tid] = (T)1 / Lk[tid * (kNB + 1) + tid];
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kNB; ++j) {
        x[j] *= rdiag[j];
#pragma unroll
        for (int l = j + 1; l < kNB; ++l) x[l] -= x[j] * Lk[l * (kNB + 1) + j];
    }
    if (i < r) {
#pragma unroll
        for (int j = 0; j < kNB; ++j)
            if (j < kb) F[(long long)(k0 + j) * r + i] = x[j];
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

// G = [I_c ; L21] L11^{-1} (row-major r x c) for a big front, solving
// X L11 = B = [I_c ; L21] by column blocks of kGB from the right:
//   X[:, J] = B[:, J] D_J  with D_J = L11[J, J]^{-1},
//   B[:, K] -= X[:, J] L11[J, K]  for every block K < J.
// Rows are independent, so each step is one launch over (row tile, column
// block) tiles of the trailing part; the tiles of block J-1 finish the step
// by multiplying with D_{J-1}.  X[J, J] = D_J is written up front (the
// identity rows of B only ever meet their own diagonal block), and the rows
// of X above the diagonal block of J are zero, so step J touches rows >= 64 J.
constexpr int kGB = 64;

// D_J^T for every diagonal block J (row n holds column n of D_J).
// One CTA of kGB threads per block; past c the block is the identity.
template <typename T>
__global__ void __launch_bounds__(kGB) k_diag_block_inv(const T* __restrict__ F, int r, int c, T* __restrict__ DT) {
    extern __shared__ __align__(16) unsigned char smem_d[];  // kGB * (kGB + 1) scalars
    T(*L)[kGB + 1] = reinterpret_cast<T(*)[kGB + 1]>(smem_d);
    __shared__ T rdiag[kGB];
    const int jc0 = blockIdx.x * kGB, jn = min(kGB, c - jc0);
    const int tid = threadIdx.x;
    for (int q = tid; q < kGB * kGB; q += blockDim.x) {
        const int i = q % kGB, j = q / kGB;
        L[i][j] = (i < jn && j < jn) ? (i >= j ? F[(long long)(jc0 + j) * r + jc0 + i] : (T)0) : (T)(i == j);
    }
    __syncthreads();
    rdiag[tid] = (T)1 / L[tid][tid];
    __syncthreads();
    // thread n: column n of D = L^{-1} by forward elimination of e_n in
    // registers (x_k = x_k / L_kk, then x_i -= L_ik x_k for i > k)
    T x[kGB];
#pragma unroll
    for (int k = 0; k < kGB; ++k) x[k] = (T)(k == tid);
#pragma unroll
    for (int k = 0; k < kGB; ++k) {
        x[k] *= rdiag[k];
#pragma unroll
        for (int i = k + 1; i < kGB; ++i) x[i] -= L[i][k] * x[k];
    }
    T* out = DT + (long long)blockIdx.x * kGB * kGB + (long long)tid * kGB;  // out[n][k] = D[k][n]
#pragma unroll
    for (int k = 0; k < kGB; ++k) out[k] = x[k];
}

// B into G: rows < c hold D_J on their diagonal block and zeros elsewhere,
// rows >= c hold L21 (read from the column-major front through a tile).
template <typename T>
__global__ void k_g_init(const T* __restrict__ F, int r, int c, const T* __restrict__ DT, T* __restrict__ G) {
    __shared__ T tile[32][33];
    const int bi = blockIdx.y * 32, bj = blockIdx.x * 32;  // rows, cols of G
    for (int y = threadIdx.y; y < 32; y += blockDim.y) {
        const int j = bj + y, i = bi + threadIdx.x;  // coalesced over rows of F's column j
        tile[y][threadIdx.x] = (i >= c && i < r && j < c) ? F[(long long)j * r + i] : (T)0;
    }
    __syncthreads();
    for (int y = threadIdx.y; y < 32; y += blockDim.y) {
        const int i = bi + y, j = bj + threadIdx.x;
        if (i >= r || j >= c) continue;
        T v = tile[threadIdx.x][y];
        if (i < c) {
            const int bI = i / kGB, bJ = j / kGB;
            v = (bI == bJ && i >= j) ? DT[(long long)bJ * kGB * kGB + (j % kGB) * kGB + (i % kGB)] : (T)0;
        }
        G[(long long)i * c + j] = v;
    }
}

// acc[a][u] += sum_k As[ty*4 + a][k] Bs[tx + 16 u][k]
template <typename T>
__device__ __forceinline__ void g_tile_product(const T (*As)[kGB + 1], const T (*Bs)[kGB + 1], int tx, int ty,
                                               T (&acc)[4][4]) {
#pragma unroll 4
    for (int k = 0; k < kGB; ++k) {
        T av[4], bv[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) av[a] = As[ty * 4 + a][k];
#pragma unroll
        for (int u = 0; u < 4; ++u) bv[u] = Bs[tx + 16 * u][k];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int u = 0; u < 4; ++u) acc[a][u] += av[a] * bv[u];
    }
}

// X[i0:i0+64, J] = acc D_J for the tile whose C values are in acc (rows >= r
// are ignored); As and Bs are free on entry.
template <typename T>
__device__ __forceinline__ void g_tile_convert(T (*As)[kGB + 1], T (*Bs)[kGB + 1], const T* __restrict__ DTj,
                                               int tx, int ty, T (&acc)[4][4], int i0, int r, int c, int jc0, int jn,
                                               T* __restrict__ G) {
    const int tid = threadIdx.x;
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int u = 0; u < 4; ++u) As[ty * 4 + a][tx + 16 * u] = acc[a][u];
    for (int q = tid; q < kGB * kGB; q += blockDim.x) Bs[q / kGB][q % kGB] = DTj[q];
    __syncthreads();
    T x[4][4] = {};
    g_tile_product(As, Bs, tx, ty, x);
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const int i = i0 + ty * 4 + a;
        if (i >= r) continue;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int n = tx + 16 * u;
            if (n < jn) G[(long long)i * c + jc0 + n] = x[a][u];
        }
    }
}

// last column block J (of width jn): rows i0 = c.. of X[:, J] = B[:, J] D_J
template <typename T>
__global__ void __launch_bounds__(256) k_g_convert(int r, int c, const T* __restrict__ DT, int jb,
                                                  T* __restrict__ G) {
    extern __shared__ __align__(16) unsigned char smem_g[];
    T(*As)[kGB + 1] = reinterpret_cast<T(*)[kGB + 1]>(smem_g);
    T(*Bs)[kGB + 1] = As + kGB;
    const int jc0 = jb * kGB, jn = min(kGB, c - jc0);
    const int i0 = c + blockIdx.x * kGB;
    const int tid = threadIdx.x, tx = tid % 16, ty = tid / 16;
    T acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const int i = i0 + ty * 4 + a;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int n = tx + 16 * u;
            acc[a][u] = (i < r && n < jn) ? G[(long long)i * c + jc0 + n] : (T)0;
        }
    }
    g_tile_convert(As, Bs, DT + (long long)jb * kGB * kGB, tx, ty, acc, i0, r, c, jc0, jn, G);
}

// step J = jb: B[rows >= 64 jb, K] -= X[., J] L11[J, K] for the column block
// K = blockIdx.y < jb; the tiles of K = jb - 1 then convert it to X.
template <typename T>
__global__ void __launch_bounds__(256) k_g_update(const T* __restrict__ F, int r, int c, const T* __restrict__ DT,
                                                 int jb, T* __restrict__ G) {
    extern __shared__ __align__(16) unsigned char smem_g[];
    T(*As)[kGB + 1] = reinterpret_cast<T(*)[kGB + 1]>(smem_g);  // As[row][k] = X[i0 + row, J]
    T(*Bs)[kGB + 1] = As + kGB;                                  // Bs[n][k] = L11[J + k, K + n]
    const int jc0 = jb * kGB, jn = min(kGB, c - jc0);
    const int kc0 = blockIdx.y * kGB;
    const int i0 = jc0 + blockIdx.x * kGB;
    const int tid = threadIdx.x, tx = tid % 16, ty = tid / 16;
    for (int q = tid; q < kGB * kGB; q += blockDim.x) {
        const int a = q / kGB, k = q % kGB;
        As[a][k] = (i0 + a < r && k < jn) ? G[(long long)(i0 + a) * c + jc0 + k] : (T)0;
        Bs[a][k] = k < jn ? F[(long long)(kc0 + a) * r + jc0 + k] : (T)0;
    }
    __syncthreads();
    T acc[4][4] = {};
    g_tile_product(As, Bs, tx, ty, acc);
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const int i = i0 + ty * 4 + a;
#pragma unroll
        for (int u = 0; u < 4; ++u) acc[a][u] = i < r ? G[(long long)i * c + kc0 + tx + 16 * u] - acc[a][u] : (T)0;
    }
    if ((int)blockIdx.y != jb - 1) {
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const int i = i0 + ty * 4 + a;
            if (i >= r) continue;
#pragma unroll
            for (int u = 0; u < 4; ++u) G[(long long)i * c + kc0 + tx + 16 * u] = acc[a][u];
        }
        return;
    }
    __syncthreads();  // As, Bs are reused by the conversion
    g_tile_convert(As, Bs, DT + (long long)blockIdx.y * kGB * kGB, tx, ty, acc, i0, r, c, kc0, kGB, G);
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
