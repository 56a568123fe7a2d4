// Persistent PCG on H = A diag(w) A^T + delta I with the supernodal
// active-core preconditioner, in ONE cooperative launch.
//
// Every phase of an iteration runs over the whole grid; phases are separated
// by cooperative-groups grid barriers.  All blocks evaluate the scalar
// recurrences (alpha, beta, norms) redundantly from the same per-block
// partial sums in the same order, so every thread takes the same branches and
// every block executes the same number of barriers; the loop is bounded by
// `maxit`, so the kernel always terminates.
//
// Phases of one iteration (spectral variant, psipm_spectral_preconditioner.py:489-556):
//   A   t = w o (A^T p')                    p' = z + beta p (deferred update)
//   B   p = p'; q = A t + delta p; partial p.q, p.p, q.q
//   B2  (only if A has long rows) finish the long rows from chunk partials
//   U   x += alpha p; r -= alpha q; partial r.r
//   [verify: A/B on x -> true residual, partial |tr|^2, |tr - r|^2]
//   P   z = P^{-1} r: forward levels, backward levels, then z with partial r.z
#pragma once

#include <cooperative_groups.h>

#include "common.cuh"

namespace psipm {

namespace cgx = cooperative_groups;

constexpr int kPcgThreads = 256;
constexpr int kPcgWarps = kPcgThreads / 32;
constexpr int kStageChunk = 512;  // f_top staging per warp (elements)
constexpr int kLongRow = 4096;    // rows with more nonzeros are split into chunks

struct SpmvLayout {
    int m = 0, n = 0;
    const int* at_ptr = nullptr;  // A^T in CSR: n rows
    const int* at_idx = nullptr;
    const int* a_ptr = nullptr;   // A in CSR: m rows
    const int* a_idx = nullptr;
    int vw = 32;                  // lanes per short row (power of two)
    const int* short_rows = nullptr;
    int n_short = 0;
    const int* long_rows = nullptr;
    int n_long = 0;
    const int* long_chunk_ptr = nullptr;  // n_long + 1
    const int* chunk_beg = nullptr;
    const int* chunk_end = nullptr;
    int n_chunks = 0;
};

template <typename T>
struct PrecLayout {
    int m = 0;
    const int* perm = nullptr;
    const int* iperm = nullptr;
    const T* dscp = nullptr;  // Jacobi scale in permuted order
    const T* G = nullptr;     // supernode panels [L11^-1 ; L21 L11^-1], row-major r x c
    const long long* panel_off = nullptr;
    const int* sn_first = nullptr;
    const long long* sn_rowptr = nullptr;
    const int* sn_rows = nullptr;
    const long long* uvec_off = nullptr;
    const long long* fg_ptr = nullptr;
    const long long* fg_idx = nullptr;
    int nlevels = 0;
    const int* fwd_ptr = nullptr;
    const int4* fwd_tasks = nullptr;  // {sn, row0, row1, 0}
    const int* bwd_ptr = nullptr;
    const int4* bwd_tasks = nullptr;  // {sn, col0, col1, kind}
    // big supernodes: pre-phase tasks per level that assemble the front
    // vector (forward) / the gathered right-hand side (backward) in global memory
    const int* fpre_ptr = nullptr;
    const int4* fpre_tasks = nullptr;  // {sn, p0, p1, 0}
    const int* bpre_ptr = nullptr;
    const int4* bpre_tasks = nullptr;
    T* fvec = nullptr;                 // indexed like sn_rows
    T* bvec = nullptr;
    const T* GT = nullptr;             // transposed panels of big supernodes (c x r row-major)
    const long long* gt_off = nullptr;
    long long* trace = nullptr;  // optional: %globaltimer after every barrier of an apply
    int trace_cap = 0;
    T* xp = nullptr;
    T* yp = nullptr;
    T* uvec = nullptr;
};

template <typename T, typename P = T>
struct PcgArgs {
    SpmvLayout sp;
    const T* at_val = nullptr;
    const T* a_val = nullptr;
    const T* w = nullptr;
    T delta = 0;
    PrecLayout<P> pc;
    const T* rhs = nullptr;
    T* x = nullptr;
    T* r = nullptr;
    T* z = nullptr;
    T* p = nullptr;
    T* q = nullptr;
    T* t = nullptr;
    T* tr = nullptr;
    T* chunk_part = nullptr;
    double* part = nullptr;  // gridDim.x * 4
    int* ctrl = nullptr;     // [0] deadline flag
    int variant = 0;
    int maxit = 0;
    int replacement = 0;
    double tol = 0.0;
    double gap_tol = 0.1;
    long long budget_ns = 0;
    double* alphas = nullptr;
    double* betas = nullptr;
    double* history = nullptr;
    int* iout = nullptr;     // info, it, matvecs, repl, checks, nalpha, nbeta, nhist, ok
    double* dout = nullptr;  // relative residual, last |r|
};

__device__ __forceinline__ long long global_ns() {
    long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ bool finite_d(double v) { return isfinite(v); }

// ---- reductions ----------------------------------------------------------
// Each block writes K partial sums; after a grid barrier every block sums
// the partials in the same order, so all blocks hold identical totals.
template <int K>
__device__ __forceinline__ void write_partials(double (&acc)[K], double* part, double* scratch) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double s = block_sum(acc[k], scratch);
        if (threadIdx.x == 0) part[blockIdx.x * 4 + k] = s;
    }
}
template <int K>
__device__ __forceinline__ void read_totals(const double* part, double (&tot)[K], double* scratch) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double v = 0.0;
        for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) v += part[b * 4 + k];
        tot[k] = block_sum(v, scratch);
    }
}

// ---- phase A: t = w o (A^T src) -----------------------------------------
// src: 0 -> v, 1 -> z, 2 -> z + beta p
template <typename T, typename P>
__device__ void phase_a(const PcgArgs<T, P>& a, const T* v, int src, T beta) {
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const int gstride = gridDim.x * blockDim.x;
    const int* __restrict__ ptr = a.sp.at_ptr;
    const int* __restrict__ idx = a.sp.at_idx;
    const T* __restrict__ val = a.at_val;
    for (int j = gtid; j < a.sp.n; j += gstride) {
        const int b = ptr[j], e = ptr[j + 1];
        T s = 0;
        if (src == 0) {
            for (int k = b; k < e; ++k) s += val[k] * v[idx[k]];
        } else if (src == 1) {
            for (int k = b; k < e; ++k) s += val[k] * a.z[idx[k]];
        } else {
            for (int k = b; k < e; ++k) {
                const int i = idx[k];
                s += val[k] * (a.z[i] + beta * a.p[i]);
            }
        }
        a.t[j] = a.w[j] * s;
    }
}

// ---- phase B: rows of A t, with an epilogue per mode -----------------------
// mode 0: p = src(p'); q = At + delta p; acc += {p.q, p.p, q.q}
// mode 1: tr = rhs - (At + delta x); acc += {tr.tr, (tr-r).(tr-r)}
// mode 2: r = rhs - (At + delta x); acc += {r.r}
template <typename T, typename P>
__device__ __forceinline__ void row_epilogue(const PcgArgs<T, P>& a, int mode, int src, T beta, int i,
                                             T s, double (&acc)[3]) {
    if (mode == 0) {
        T pn = src == 1 ? a.z[i] : (src == 2 ? a.z[i] + beta * a.p[i] : a.p[i]);
        T qi = s + a.delta * pn;
        a.p[i] = pn;
        a.q[i] = qi;
        acc[0] += (double)pn * (double)qi;
        acc[1] += (double)pn * (double)pn;
        acc[2] += (double)qi * (double)qi;
    } else if (mode == 1) {
        T tri = a.rhs[i] - (s + a.delta * a.x[i]);
        a.tr[i] = tri;
        double d = (double)tri - (double)a.r[i];
        acc[0] += (double)tri * (double)tri;
        acc[1] += d * d;
    } else {
        T ri = a.rhs[i] - (s + a.delta * a.x[i]);
        a.r[i] = ri;
        acc[0] += (double)ri * (double)ri;
    }
}

template <typename T, typename P>
__device__ void phase_b(const PcgArgs<T, P>& a, int mode, int src, T beta, double (&acc)[3]) {
    const int lane = threadIdx.x & 31;
    const int gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int vw = a.sp.vw;
    const int per_warp = 32 / vw;
    const int sub = lane / vw, sl = lane % vw;
    const int* __restrict__ ptr = a.sp.a_ptr;
    const int* __restrict__ idx = a.sp.a_idx;
    const T* __restrict__ val = a.a_val;
    const T* __restrict__ t = a.t;
    for (int base = gwarp * per_warp; base < a.sp.n_short; base += nwarps * per_warp) {
        const int ri = base + sub;
        const bool valid = ri < a.sp.n_short;
        const int i = valid ? a.sp.short_rows[ri] : 0;
        T s = 0;
        if (valid) {
            const int b = ptr[i], e = ptr[i + 1];
            for (int k = b + sl; k < e; k += vw) s += val[k] * t[idx[k]];
        }
        for (int o = vw >> 1; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (valid && sl == 0) row_epilogue(a, mode, src, beta, i, s, acc);
    }
    // long rows: chunk partial sums (finished in phase_b2)
    for (int c = gwarp; c < a.sp.n_chunks; c += nwarps) {
        T s = 0;
        for (int k = a.sp.chunk_beg[c] + lane; k < a.sp.chunk_end[c]; k += 32) s += val[k] * t[idx[k]];
        s = warp_sum(s);
        if (lane == 0) a.chunk_part[c] = s;
    }
}

template <typename T, typename P>
__device__ void phase_b2(const PcgArgs<T, P>& a, int mode, int src, T beta, double (&acc)[3]) {
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const int gstride = gridDim.x * blockDim.x;
    for (int l = gtid; l < a.sp.n_long; l += gstride) {
        T s = 0;
        for (int c = a.sp.long_chunk_ptr[l]; c < a.sp.long_chunk_ptr[l + 1]; ++c) s += a.chunk_part[c];
        row_epilogue(a, mode, src, beta, a.sp.long_rows[l], s, acc);
    }
}

// ---- preconditioner apply ----------------------------------------------------
// P^{-1} = Ds Pi^T L^{-T} L^{-1} Pi Ds with L supernodal.  Each supernode s
// (c pivot columns, r rows) stores G = [L11^{-1} ; L21 L11^{-1}] (r x c,
// row-major) and its transpose GT (c x r, row-major), so both sweeps are
// dense matrix-vector products over contiguous rows:
//   forward  (levels bottom-up):  f = [b_s ; 0] + sum_children u_child
//                                 x_s = G_top f_top,  u_s = f_bot - G_bot f_top
//   backward (levels top-down):   v = [x_s ; -y(rows below)]
//                                 y_s = G^T v
// Per level and sweep: a pre-phase assembles f (or v) in global memory and
// initialises the outputs, then 2-D tasks (kApplyRows rows x kApplyChunk
// contraction entries) accumulate their partial products with atomics.
constexpr int kApplyRows = 16;
constexpr int kApplyChunk = 256;

// Four rows against one vector by one warp: lanes stride the contraction
// index, four independent accumulators, results in every lane.
template <typename T>
__device__ __forceinline__ void warp_dot4(const T* __restrict__ m0, const T* __restrict__ m1,
                                          const T* __restrict__ m2, const T* __restrict__ m3,
                                          const T* __restrict__ v, int b0, int b1, int b2, int b3,
                                          int e, T (&out)[4]) {
    const int lane = threadIdx.x & 31;
    T s0 = 0, s1 = 0, s2 = 0, s3 = 0;
    const int lo = min(min(b0, b1), min(b2, b3));
    for (int j = lo + lane; j < e; j += 32) {
        const T vj = v[j];
        if (j >= b0) s0 += m0[j] * vj;
        if (j >= b1) s1 += m1[j] * vj;
        if (j >= b2) s2 += m2[j] * vj;
        if (j >= b3) s3 += m3[j] * vj;
    }
    out[0] = warp_sum(s0);
    out[1] = warp_sum(s1);
    out[2] = warp_sum(s2);
    out[3] = warp_sum(s3);
}

// forward pre-phase: f into fvec, outputs initialised (x_s = 0, u_s = f_bot)
template <typename P, typename IT>
__device__ void prec_forward_pre(const PrecLayout<P>& pc, const IT* in, int4 task) {
    const int lane = threadIdx.x & 31;
    const int s = task.x;
    const int first = pc.sn_first[s];
    const int c = pc.sn_first[s + 1] - first;
    const long long rb = pc.sn_rowptr[s];
    for (int q = task.y + lane; q < task.z; q += 32) {
        P f = 0;
        if (q < c) {
            const int k = first + q;
            f = pc.dscp[k] * (P)in[pc.perm[k]];
        }
        for (long long g = pc.fg_ptr[rb + q]; g < pc.fg_ptr[rb + q + 1]; ++g) f += pc.uvec[pc.fg_idx[g]];
        pc.fvec[rb + q] = f;
        if (q < c)
            pc.xp[first + q] = 0;
        else
            pc.uvec[pc.uvec_off[s] + q - c] = f;
    }
}

// forward task {s, i0, i1, j0}: rows [i0, i1) of G against f[j0, j0+chunk)
template <typename P>
__device__ void prec_forward_gemv(const PrecLayout<P>& pc, int4 task) {
    const int lane = threadIdx.x & 31;
    const int s = task.x, i0 = task.y, i1 = task.z, j0 = task.w;
    const int first = pc.sn_first[s];
    const int c = pc.sn_first[s + 1] - first;
    const int j1 = min(c, j0 + kApplyChunk);
    const long long rb = pc.sn_rowptr[s];
    const P* __restrict__ Gs = pc.G + pc.panel_off[s];
    const P* __restrict__ f = pc.fvec + rb;
    for (int i = i0; i < i1; i += 4) {
        const P* rows[4];
        int end[4];
        for (int k = 0; k < 4; ++k) {
            const int ii = min(i + k, i1 - 1);
            rows[k] = Gs + (long long)ii * c;
            end[k] = i + k < i1 ? (ii < c ? min(j1, ii + 1) : j1) : j0;  // G_top is lower triangular
        }
        // rows share the loop bound j1; entries past a row's own end are masked
        P d[4];
        const int lo = j0;
        P s0 = 0, s1 = 0, s2 = 0, s3 = 0;
        for (int j = lo + lane; j < j1; j += 32) {
            const P fj = f[j];
            if (j < end[0]) s0 += rows[0][j] * fj;
            if (j < end[1]) s1 += rows[1][j] * fj;
            if (j < end[2]) s2 += rows[2][j] * fj;
            if (j < end[3]) s3 += rows[3][j] * fj;
        }
        d[0] = warp_sum(s0);
        d[1] = warp_sum(s1);
        d[2] = warp_sum(s2);
        d[3] = warp_sum(s3);
        if (lane < 4 && i + lane < i1) {
            const int ii = i + lane;
            const P v = lane == 0 ? d[0] : lane == 1 ? d[1] : lane == 2 ? d[2] : d[3];
            if (ii < c)
                atomicAdd(&pc.xp[first + ii], v);
            else
                atomicAdd(&pc.uvec[pc.uvec_off[s] + ii - c], -v);
        }
    }
}

// backward pre-phase: v into bvec, y_s = 0
template <typename P>
__device__ void prec_backward_pre(const PrecLayout<P>& pc, int4 task) {
    const int lane = threadIdx.x & 31;
    const int s = task.x;
    const int first = pc.sn_first[s];
    const int c = pc.sn_first[s + 1] - first;
    const long long rb = pc.sn_rowptr[s];
    for (int q = task.y + lane; q < task.z; q += 32) {
        pc.bvec[rb + q] = q < c ? pc.xp[first + q] : -pc.yp[pc.sn_rows[rb + q]];
        if (q < c) pc.yp[first + q] = 0;
    }
}

// backward task {s, j0, j1, i0}: columns [j0, j1) of G (rows of GT) against v[i0, i0+chunk)
template <typename P>
__device__ void prec_backward_gemv(const PrecLayout<P>& pc, int4 task) {
    const int lane = threadIdx.x & 31;
    const int s = task.x, j0 = task.y, j1 = task.z, i0 = task.w;
    const int first = pc.sn_first[s];
    const long long rb = pc.sn_rowptr[s];
    const int r = (int)(pc.sn_rowptr[s + 1] - rb);
    const int i1 = min(r, i0 + kApplyChunk);
    const P* __restrict__ GTs = pc.GT + pc.gt_off[s];
    const P* __restrict__ v = pc.bvec + rb;
    for (int j = j0; j < j1; j += 4) {
        const P* rows[4];
        int beg[4];
        for (int k = 0; k < 4; ++k) {
            const int jj = min(j + k, j1 - 1);
            rows[k] = GTs + (long long)jj * r;
            beg[k] = j + k < j1 ? max(i0, jj) : i1;  // G[i, j] = 0 for i < j
        }
        P d[4];
        warp_dot4(rows[0], rows[1], rows[2], rows[3], v, beg[0], beg[1], beg[2], beg[3], i1, d);
        if (lane < 4 && j + lane < j1) {
            const P val = lane == 0 ? d[0] : lane == 1 ? d[1] : lane == 2 ? d[2] : d[3];
            atomicAdd(&pc.yp[first + j + lane], val);
        }
    }
}

// Small supernodes (r <= kSmallRows, c <= 32): one warp does the whole
// supernode in one task, the vector staged in shared memory and one lane per
// output, so no pre-phase, no shuffles and no atomics are needed.
constexpr int kSmallRows = 64;

template <typename P, typename IT>
__device__ void prec_forward_small(const PrecLayout<P>& pc, const IT* in, int s, P* fs) {
    const int lane = threadIdx.x & 31;
    const int first = pc.sn_first[s];
    const int c = pc.sn_first[s + 1] - first;
    const long long rb = pc.sn_rowptr[s];
    const int r = (int)(pc.sn_rowptr[s + 1] - rb);
    for (int q = lane; q < r; q += 32) {
        P f = 0;
        if (q < c) {
            const int k = first + q;
            f = pc.dscp[k] * (P)in[pc.perm[k]];
        }
        for (long long g = pc.fg_ptr[rb + q]; g < pc.fg_ptr[rb + q + 1]; ++g) f += pc.uvec[pc.fg_idx[g]];
        fs[q] = f;
    }
    __syncwarp();
    const P* __restrict__ Gs = pc.G + pc.panel_off[s];
    for (int row = lane; row < r; row += 32) {
        const int jlim = row < c ? row + 1 : c;
        const P* __restrict__ g = Gs + (long long)row * c;
        P d = 0;
        for (int j = 0; j < jlim; ++j) d += g[j] * fs[j];
        if (row < c)
            pc.xp[first + row] = d;
        else
            pc.uvec[pc.uvec_off[s] + row - c] = fs[row] - d;
    }
    __syncwarp();
}

template <typename P>
__device__ void prec_backward_small(const PrecLayout<P>& pc, int s, P* fs) {
    const int lane = threadIdx.x & 31;
    const int first = pc.sn_first[s];
    const int c = pc.sn_first[s + 1] - first;
    const long long rb = pc.sn_rowptr[s];
    const int r = (int)(pc.sn_rowptr[s + 1] - rb);
    for (int q = lane; q < r; q += 32) fs[q] = q < c ? pc.xp[first + q] : -pc.yp[pc.sn_rows[rb + q]];
    __syncwarp();
    if (lane < c) {
        const P* __restrict__ gt = pc.GT + pc.panel_off[s] + (long long)lane * r;
        P d = 0;
        for (int i = lane; i < r; ++i) d += gt[i] * fs[i];
        pc.yp[first + lane] = d;
    }
    __syncwarp();
}

// z = P^{-1} in; acc_rz += in . z.  Ends without a barrier (the caller's
// reduction provides it).
template <typename P, typename IT>
__device__ void prec_apply(const PrecLayout<P>& pc, const IT* in, IT* out, double& acc_rz, P* fs,
                           cgx::grid_group& grid) {
    const int gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    int ntrace = 0;
    const bool tracer = pc.trace && blockIdx.x == 0 && threadIdx.x == 0;
    auto mark = [&]() {
        if (tracer && ntrace < pc.trace_cap) pc.trace[ntrace++] = global_ns();
    };
    mark();
    // task kind (int4.w for fused tasks is -1): fused small supernode or 2-D GEMV
    for (int lev = 0; lev < pc.nlevels; ++lev) {
        if (pc.fpre_ptr[lev + 1] > pc.fpre_ptr[lev]) {
            for (int tk = pc.fpre_ptr[lev] + gwarp; tk < pc.fpre_ptr[lev + 1]; tk += nwarps)
                prec_forward_pre(pc, in, pc.fpre_tasks[tk]);
            grid.sync();
            mark();
        }
        for (int tk = pc.fwd_ptr[lev] + gwarp; tk < pc.fwd_ptr[lev + 1]; tk += nwarps) {
            const int4 task = pc.fwd_tasks[tk];
            if (task.w < 0)
                prec_forward_small(pc, in, task.x, fs);
            else
                prec_forward_gemv(pc, task);
        }
        grid.sync();
        mark();
    }
    for (int lev = pc.nlevels - 1; lev >= 0; --lev) {
        if (pc.bpre_ptr[lev + 1] > pc.bpre_ptr[lev]) {
            for (int tk = pc.bpre_ptr[lev] + gwarp; tk < pc.bpre_ptr[lev + 1]; tk += nwarps)
                prec_backward_pre(pc, pc.bpre_tasks[tk]);
            grid.sync();
            mark();
        }
        for (int tk = pc.bwd_ptr[lev] + gwarp; tk < pc.bwd_ptr[lev + 1]; tk += nwarps) {
            const int4 task = pc.bwd_tasks[tk];
            if (task.w < 0)
                prec_backward_small(pc, task.x, fs);
            else
                prec_backward_gemv(pc, task);
        }
        grid.sync();
        mark();
    }
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const int gstride = gridDim.x * blockDim.x;
    for (int i = gtid; i < pc.m; i += gstride) {
        const int k = pc.iperm[i];
        const IT zi = (IT)(pc.dscp[k] * pc.yp[k]);
        out[i] = zi;
        acc_rz += (double)in[i] * (double)zi;
    }
}

// H v into phase-B epilogue `mode` (A, barrier, B [, barrier, B2]); ends after
// the partials are written; the caller issues the barrier.
template <typename T, typename P>
__device__ void operator_pass(const PcgArgs<T, P>& a, const T* v, int src, T beta, int mode,
                              double (&acc)[3], cgx::grid_group& grid) {
    phase_a(a, v, src, beta);
    grid.sync();
    phase_b(a, mode, src, beta, acc);
    if (a.sp.n_long) {
        grid.sync();
        phase_b2(a, mode, src, beta, acc);
    }
}

template <typename T, typename P>
__global__ void __launch_bounds__(kPcgThreads, 3) k_pcg(PcgArgs<T, P> a) {
    cgx::grid_group grid = cgx::this_grid();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double scratch[kPcgWarps + 1];
    P* fs = reinterpret_cast<P*>(smem_raw) + (threadIdx.x >> 5) * kStageChunk;
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const int gstride = gridDim.x * blockDim.x;
    const bool leader = blockIdx.x == 0 && threadIdx.x == 0;
    const bool hsd = a.variant == PSIPM_PCG_HSD;
    const double tiny = 2.2250738585072014e-308;
    long long t_start = 0;
    if (leader) t_start = global_ns();
    int info = 0, it = 0, matvecs = 0, repl = 0, checks = 0, nalpha = 0, nbeta = 0, nhist = 0, ok = 0;
    double rel = 0.0, last_r = 0.0, scale = 1.0;
    // Partial sums alternate between two buffers, so a block may write the
    // next reduction while another still reads the previous one.
    int red = 0;
    // phase clock (leader only): [0] H·p, [1] updates, [2] applies, [3] other
    double ph[4] = {0.0, 0.0, 0.0, 0.0};
    long long tmark = t_start;
    auto lap = [&](int k) {
        if (leader) {
            const long long now = global_ns();
            ph[k] += 1e-9 * (double)(now - tmark);
            tmark = now;
        }
    };
    auto reduce1 = [&](double v) -> double {
        double* pb = a.part + (size_t)(red & 1) * gridDim.x * 4;
        double acc[1] = {v}, tot[1];
        write_partials<1>(acc, pb, scratch);
        grid.sync();
        read_totals<1>(pb, tot, scratch);
        ++red;
        return tot[0];
    };
    auto reduce2 = [&](double (&acc)[3], double (&tot)[3]) {
        double* pb = a.part + (size_t)(red & 1) * gridDim.x * 4;
        double a2[2] = {acc[0], acc[1]}, t2[2];
        write_partials<2>(a2, pb, scratch);
        grid.sync();
        read_totals<2>(pb, t2, scratch);
        tot[0] = t2[0];
        tot[1] = t2[1];
        ++red;
    };
    auto reduce3 = [&](double (&acc)[3], double (&tot)[3]) {
        double* pb = a.part + (size_t)(red & 1) * gridDim.x * 4;
        write_partials<3>(acc, pb, scratch);
        grid.sync();
        read_totals<3>(pb, tot, scratch);
        ++red;
    };

    double acc3[3] = {0.0, 0.0, 0.0}, tot3[3] = {0.0, 0.0, 0.0};
    double rhs_sq = 0.0;
    for (int i = gtid; i < a.sp.m; i += gstride) rhs_sq += (double)a.rhs[i] * (double)a.rhs[i];
    const double rhs_norm = sqrt(reduce1(rhs_sq));
    scale = hsd ? rhs_norm : fmax(1.0, rhs_norm);
    const double target = hsd ? fmax(a.tol * rhs_norm, 64.0 * 2.220446049250313e-16 * rhs_norm) : a.tol;
    double rz = 0.0;
    int src = 1;  // p' = z on the first iteration
    T beta = 0;

    if (hsd && rhs_norm == 0.0) {
        for (int i = gtid; i < a.sp.m; i += gstride) a.x[i] = 0;
        ok = 1;
        goto done;
    }
    {
        // x = P^-1 rhs ; r = rhs - H x
        double dummy = 0.0;
        prec_apply(a.pc, a.rhs, a.x, dummy, fs, grid);
        grid.sync();
        acc3[0] = acc3[1] = acc3[2] = 0.0;
        operator_pass(a, a.x, 0, (T)0, 2, acc3, grid);
        const double rnorm = sqrt(reduce1(acc3[0]));
        matvecs = 1;
        last_r = rnorm;
        if (hsd) {
            if (rnorm <= target) {
                ok = 1;
                goto done;
            }
        } else {
            if (leader && a.history) a.history[0] = rnorm / scale;
            nhist = 1;
        }
        double rzacc = 0.0;
        prec_apply(a.pc, a.r, a.z, rzacc, fs, grid);
        rz = reduce1(rzacc);
        if (hsd) {
            if (!finite_d(rz) || rz <= 0.0) goto done;
        } else {
            info = a.maxit;
            if (rnorm / scale <= target)
                info = 0;
            else if (!finite_d(rz) || rz <= 0.0)
                info = -1;
        }
    }
    while ((hsd || info > 0) && it < a.maxit) {
        // q = H p'   (p <- p' inside phase B)
        acc3[0] = acc3[1] = acc3[2] = 0.0;
        lap(3);
        operator_pass(a, a.p, src, beta, 0, acc3, grid);
        reduce3(acc3, tot3);
        lap(0);
        ++matvecs;
        const double curv = tot3[0];
        double alpha;
        if (hsd) {
            if (!finite_d(curv) || curv <= 0.0) {
                ++it;
                goto done;
            }
            alpha = rz / curv;
        } else {
            const double floor_ = tiny * fmax(1.0, sqrt(tot3[1]) * sqrt(tot3[2]));
            if (!finite_d(curv) || curv <= floor_) {
                info = -2;
                break;
            }
            alpha = rz / curv;
            if (!finite_d(alpha) || alpha <= 0.0) {
                info = -3;
                break;
            }
        }
        // x += alpha p ; r -= alpha q
        double rr;
        {
            double acc = 0.0;
            const T al = (T)alpha;
            for (int i = gtid; i < a.sp.m; i += gstride) {
                a.x[i] += al * a.p[i];
                const T ri = a.r[i] - al * a.q[i];
                a.r[i] = ri;
                acc += (double)ri * (double)ri;
            }
            if (leader && a.budget_ns > 0 && global_ns() - t_start > a.budget_ns) a.ctrl[0] = 1;
            rr = reduce1(acc);
        }
        lap(1);
        ++it;
        if (leader && a.alphas) a.alphas[nalpha] = alpha;
        ++nalpha;
        const int timed_out = *((volatile int*)a.ctrl);
        if (hsd) {
            if (it % 10 == 0) {
                acc3[0] = acc3[1] = acc3[2] = 0.0;
                operator_pass(a, a.x, 0, (T)0, 2, acc3, grid);
                rr = reduce1(acc3[0]);
                ++matvecs;
            }
            last_r = sqrt(rr);
            if (last_r <= target) {
                ok = 1;
                goto done;
            }
            if (timed_out) goto done;
        } else {
            const double rec = sqrt(rr) / scale;
            const bool replace = a.replacement > 0 && it % a.replacement == 0;
            if (timed_out) {
                info = -8;  // deadline: not a reference code; the host reports a timeout
                break;
            }
            if (replace || rec <= target) {
                acc3[0] = acc3[1] = acc3[2] = 0.0;
                operator_pass(a, a.x, 0, (T)0, 1, acc3, grid);
                reduce2(acc3, tot3);
                ++matvecs;
                ++checks;
                const double tnorm = sqrt(tot3[0]);
                const double relc = tnorm / scale;
                if (leader && a.history) a.history[nhist] = relc;
                ++nhist;
                if (!finite_d(relc)) {
                    info = -4;
                    break;
                }
                if (relc <= target) {
                    info = 0;
                    break;
                }
                const double gap = sqrt(tot3[1]);
                if (gap > a.gap_tol * fmax(tnorm, target * scale)) {
                    // residual replacement: r = tr and restart the recurrence
                    for (int i = gtid; i < a.sp.m; i += gstride) a.r[i] = a.tr[i];
                    ++repl;
                    grid.sync();
                    double rzr = 0.0;
                    prec_apply(a.pc, a.r, a.z, rzr, fs, grid);
                    rz = reduce1(rzr);
                    if (!finite_d(rz) || rz <= 0.0) {
                        info = -5;
                        break;
                    }
                    src = 1;
                    nalpha = 0;
                    nbeta = 0;
                    continue;
                }
            }
        }
        // z = P^-1 r ; beta
        lap(3);
        double rzn = 0.0;
        prec_apply(a.pc, a.r, a.z, rzn, fs, grid);
        const double rz_next = reduce1(rzn);
        lap(2);
        if (!finite_d(rz_next) || rz_next <= 0.0) {
            if (hsd) goto done;
            info = -6;
            break;
        }
        const double bt = rz_next / rz;
        if (!hsd && (!finite_d(bt) || bt < 0.0)) {
            info = -7;
            break;
        }
        if (leader && a.betas) a.betas[nbeta] = bt;
        ++nbeta;
        beta = (T)bt;
        src = 2;
        rz = rz_next;
    }
    if (!hsd) {
        // explicit final residual (psipm_spectral_preconditioner.py:558-561)
        acc3[0] = acc3[1] = acc3[2] = 0.0;
        operator_pass(a, a.x, 0, (T)0, 1, acc3, grid);
        const double fin = reduce1(acc3[0]);
        ++matvecs;
        last_r = sqrt(fin);
        rel = last_r / scale;
        if (info > 0 && rel <= target) info = 0;
    }
done:
    if (hsd) rel = scale > 0.0 ? last_r / scale : 0.0;
    if (leader) {
        a.iout[0] = info;
        a.iout[1] = it;
        a.iout[2] = matvecs;
        a.iout[3] = repl;
        a.iout[4] = checks;
        a.iout[5] = nalpha;
        a.iout[6] = nbeta;
        a.iout[7] = nhist;
        a.iout[8] = ok;
        a.dout[0] = rel;
        a.dout[1] = last_r;
        lap(3);
        for (int k = 0; k < 4; ++k) a.dout[2 + k] = ph[k];
    }
}

// Grid-barrier cost probe: `count` barriers, nothing else.
__global__ void k_barrier_probe(int count, long long* out) {
    cgx::grid_group grid = cgx::this_grid();
    const long long t0 = global_ns();
    for (int i = 0; i < count; ++i) grid.sync();
    if (blockIdx.x == 0 && threadIdx.x == 0) *out = global_ns() - t0;
}

// Standalone preconditioner apply / operator kernels (cooperative as well)
template <typename T, typename P>
__global__ void __launch_bounds__(kPcgThreads, 3) k_apply(PcgArgs<T, P> a, const T* in, T* out) {
    cgx::grid_group grid = cgx::this_grid();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    P* fs = reinterpret_cast<P*>(smem_raw) + (threadIdx.x >> 5) * kStageChunk;
    double dummy = 0.0;
    prec_apply(a.pc, in, out, dummy, fs, grid);
}

// y = H v  (mode 0 with src = v copied into p first by the host)
template <typename T, typename P>
__global__ void __launch_bounds__(kPcgThreads, 3) k_matvec(PcgArgs<T, P> a) {
    cgx::grid_group grid = cgx::this_grid();
    double acc[3] = {0.0, 0.0, 0.0};
    operator_pass(a, a.p, 0, (T)0, 0, acc, grid);
}

}  // namespace psipm
