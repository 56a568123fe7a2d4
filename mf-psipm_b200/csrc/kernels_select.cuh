// Leverage scores (S3) and radix top-k selection (S4) on the device.
//
// Scores follow psipm_stable_preconditioner.py:293-309 operation by
// operation so the FP64 results are bit-identical: every product and sum is
// rounded separately (no FMA contraction: __dmul_rn / __dadd_rn), sums run
// sequentially in the order of SciPy's CSC/CSR matvec, divisions are IEEE.
//
// Top-k (psipm_stable_preconditioner.py:97-110) selects the `count` largest
// finite scores among the eligible candidates by an 8-pass MSB radix select
// on order-preserving 64-bit keys; the tie rule at the threshold value is
// "lower candidate index first", the order the reference sorts its result in.
#pragma once

#include "common.cuh"

namespace psipm {

constexpr int kSelectThreads = 256;

// weights: w = 1/theta (psipm_stable_preconditioner.py:399)
__global__ void k_weights(long long n, const double* __restrict__ theta, double* __restrict__ w) {
    long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j < n) w[j] = __ddiv_rn(1.0, theta[j]);
}

// diag_full_i = sum_j (a_ij^2) w_j over row i in column order (A2_factor @ w);
// columns with skip[j] != 0 (extracted dense columns) are left out
__global__ void k_diag_full(int m, const int* __restrict__ a_ptr, const int* __restrict__ a_idx,
                            const double* __restrict__ a_val, const double* __restrict__ w,
                            const unsigned char* __restrict__ skip, double* __restrict__ diag) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    // the sum stays sequential in column order (bit-identical to the sparse
    // product); the loads of eight terms are issued before their additions
    double acc = 0.0;
    const int e0 = a_ptr[i], e1 = a_ptr[i + 1];
    int k = e0;
    for (; k + 8 <= e1; k += 8) {
        double t[8];
        bool use[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int j = a_idx[k + u];
            const double a = a_val[k + u];
            use[u] = !(skip && skip[j]);
            t[u] = __dmul_rn(__dmul_rn(a, a), w[j]);
        }
#pragma unroll
        for (int u = 0; u < 8; ++u)
            if (use[u]) acc = __dadd_rn(acc, t[u]);
    }
    for (; k < e1; ++k) {
        const int j = a_idx[k];
        if (skip && skip[j]) continue;
        const double a = a_val[k];
        acc = __dadd_rn(acc, __dmul_rn(__dmul_rn(a, a), w[j]));
    }
    diag[i] = acc;
}

// d_i += a_ij^2 w_j over one extracted column j (A2_low_rank @ w_L, one launch
// per column in ascending column order, as the sparse product sums them)
__global__ void k_diag_lr_column(int nnz, const int* __restrict__ rows, const double* __restrict__ vals,
                                 const double* __restrict__ w, long long j, double* __restrict__ d) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nnz) return;
    const double a = vals[e];
    d[rows[e]] = __dadd_rn(d[rows[e]], __dmul_rn(__dmul_rn(a, a), w[j]));
}

__global__ void k_add_rn(int m, const double* __restrict__ a, const double* __restrict__ b,
                         double* __restrict__ out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) out[i] = __dadd_rn(a[i], b[i]);
}

// inv_i = 1 / max(diag_i + max(delta, tiny), tiny)
__global__ void k_inv_diag(int m, const double* __restrict__ diag, double dplus,
                           double* __restrict__ inv) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const double tiny = 2.2250738585072014e-308;
    const double d = __dadd_rn(diag[i], dplus);
    inv[i] = __ddiv_rn(1.0, fmax(d, tiny));
}

// score_c = (w_j * sum_i a_ij^2 inv_i) / (1 + fill_weight * q(q-1)/2)
__global__ void k_scores(long long ncand, const long long* __restrict__ cand,
                         const int* __restrict__ at_ptr, const int* __restrict__ at_idx,
                         const double* __restrict__ at_val, const double* __restrict__ w,
                         const double* __restrict__ inv, double fill_weight,
                         double* __restrict__ score) {
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= ncand) return;
    const long long j = cand[c];
    double acc = 0.0;
    const int b = at_ptr[j], e = at_ptr[j + 1];
    for (int k = b; k < e; ++k) {
        const double a = at_val[k];
        acc = __dadd_rn(acc, __dmul_rn(__dmul_rn(a, a), inv[at_idx[k]]));
    }
    const double lev = __dmul_rn(w[j], acc);
    const double q = (double)(e - b);
    const double burden = __dmul_rn(__dmul_rn(0.5, q), fmax(__dadd_rn(q, -1.0), 0.0));
    score[c] = __ddiv_rn(lev, __dadd_rn(1.0, __dmul_rn(fill_weight, burden)));
}

// ---- radix select ------------------------------------------------------------
// Order-preserving key: larger score -> larger key.
__device__ __forceinline__ unsigned long long score_key(double s) {
    unsigned long long b = (unsigned long long)__double_as_longlong(s);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

__device__ __forceinline__ bool eligible(const double* score, const unsigned char* mask, long long i) {
    return (mask == nullptr || mask[i]) && isfinite(score[i]);
}

__global__ void k_count_eligible(long long n, const double* __restrict__ score,
                                 const unsigned char* __restrict__ mask,
                                 unsigned long long* __restrict__ out) {
    __shared__ unsigned long long s;
    if (threadIdx.x == 0) s = 0;
    __syncthreads();
    unsigned long long local = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        local += eligible(score, mask, i);
    atomicAdd(&s, local);
    __syncthreads();
    if (threadIdx.x == 0) atomicAdd(out, s);
}

// histogram of the 8-bit digit at `shift` among eligible keys whose higher
// digits equal `prefix` (under `pmask`)
__global__ void k_radix_hist(long long n, const double* __restrict__ score,
                             const unsigned char* __restrict__ mask, int shift,
                             unsigned long long prefix, unsigned long long pmask,
                             unsigned int* __restrict__ hist) {
    __shared__ unsigned int h[256];
    for (int b = threadIdx.x; b < 256; b += blockDim.x) h[b] = 0;
    __syncthreads();
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        if (!eligible(score, mask, i)) continue;
        const unsigned long long k = score_key(score[i]);
        if ((k & pmask) != prefix) continue;
        atomicAdd(&h[(k >> shift) & 0xffu], 1u);
    }
    __syncthreads();
    for (int b = threadIdx.x; b < 256; b += blockDim.x)
        if (h[b]) atomicAdd(&hist[b], h[b]);
}

// flag[i] = 1 for eligible keys above the threshold; eq[i] = 1 for keys equal to it
__global__ void k_mark_threshold(long long n, const double* __restrict__ score,
                                 const unsigned char* __restrict__ mask, unsigned long long thr,
                                 int select_all, unsigned char* __restrict__ flag,
                                 int* __restrict__ eq) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    int e = 0;
    if (eligible(score, mask, i)) {
        const unsigned long long k = score_key(score[i]);
        if (select_all || k > thr)
            flag[i] = 1;
        else if (k == thr)
            e = 1;
    }
    eq[i] = e;
}

// among the keys equal to the threshold take the first `need` by index
// (eqscan = exclusive prefix sum of eq)
__global__ void k_mark_ties(long long n, const int* __restrict__ eq, const int* __restrict__ eqscan,
                            long long need, unsigned char* __restrict__ flag) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (eq[i] && eqscan[i] < need) flag[i] = 1;
}

__global__ void k_set_flags(long long cnt, const long long* __restrict__ idx, unsigned char v,
                            unsigned char* __restrict__ flag) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < cnt) flag[idx[i]] = v;
}

// out = a & ~b  (or a | b)
__global__ void k_flag_op(long long n, const unsigned char* __restrict__ a,
                          const unsigned char* __restrict__ b, int op, unsigned char* __restrict__ out) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = op == 0 ? (unsigned char)(a[i] && !b[i]) : (unsigned char)(a[i] || b[i]);
}

// ---- HSD pricing (psipm_v3_1_hsd.py:2101-2158) ---------------------------------
// violation_j = (A^T y)_j - c_j tau, with the products and sums in index order
// and no contraction (bit-identical to SciPy's CSR product); eligible_j = 1 for
// inactive columns with violation_j > threshold
__global__ void k_price(long long n, const int* __restrict__ at_ptr, const int* __restrict__ at_idx,
                        const double* __restrict__ at_val, const double* __restrict__ y,
                        const double* __restrict__ c, double tau, const unsigned char* __restrict__ active,
                        double threshold, double* __restrict__ violation, unsigned char* __restrict__ eligible) {
    const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j >= n) return;
    double s = 0.0;
    for (int k = at_ptr[j]; k < at_ptr[j + 1]; ++k) s = __dadd_rn(s, __dmul_rn(at_val[k], y[at_idx[k]]));
    const double v = __dsub_rn(s, __dmul_rn(c[j], tau));
    violation[j] = v;
    eligible[j] = (unsigned char)(!active[j] && v > threshold);
}

}  // namespace psipm
