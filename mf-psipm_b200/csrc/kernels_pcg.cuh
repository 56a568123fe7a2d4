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
    T* xp = nullptr;
    T* yp = nullptr;
    T* uvec = nullptr;
};

template <typename T>
struct PcgArgs {
    SpmvLayout sp;
    const T* at_val = nullptr;
    const T* a_val = nullptr;
    const T* w = nullptr;
    T delta = 0;
    PrecLayout<T> pc;
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
template <typename T>
__device__ void phase_a(const PcgArgs<T>& a, const T* v, int src, T beta) {
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
template <typename T>
__device__ __forceinline__ void row_epilogue(const PcgArgs<T>& a, int mode, int src, T beta, int i,
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

template <typename T>
__device__ void phase_b(const PcgArgs<T>& a, int mode, int src, T beta, double (&acc)[3]) {
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

template <typename T>
__device__ void phase_b2(const PcgArgs<T>& a, int mode, int src, T beta, double (&acc)[3]) {
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const int gstride = gridDim.x * blockDim.x;
    for (int l = gtid; l < a.sp.n_long; l += gstride) {
        T s = 0;
        for (int c = a.sp.long_chunk_ptr[l]; c < a.sp.long_chunk_ptr[l + 1]; ++c) s += a.chunk_part[c];
        row_epilogue(a, mode, src, beta, a.sp.long_rows[l], s, acc);
    }
}

// ---- preconditioner apply ----------------------------------------------------
template <typename T>
__device__ void prec_forward_task(const PcgArgs<T>& a, const T* in, int4 task, T* fs) {
    const PrecLayout<T>& pc = a.pc;
    const int lane = threadIdx.x & 31;
    const int s = task.x, r0 = task.y, r1 = task.z;
    const int first = pc.sn_first[s];
    const int c = pc.sn_first[s + 1] - first;
    const long long rb = pc.sn_rowptr[s];
    const T* __restrict__ Gs = pc.G + pc.panel_off[s];
    T acc = 0;
    for (int j0 = 0; j0 < c; j0 += kStageChunk) {
        const int jn = min(kStageChunk, c - j0);
        if (r1 <= c && r1 - 1 < j0) break;  // all rows of the task are above this chunk
        for (int jj = lane; jj < jn; jj += 32) {
            const int j = j0 + jj, k = first + j;
            T f = pc.dscp[k] * in[pc.perm[k]];
            for (long long g = pc.fg_ptr[rb + j]; g < pc.fg_ptr[rb + j + 1]; ++g) f += pc.uvec[pc.fg_idx[g]];
            fs[jj] = f;
        }
        __syncwarp();
        for (int rr = r0; rr < r1; ++rr) {
            const int jlim = rr < c ? min(jn, rr - j0 + 1) : jn;
            T d = 0;
            const T* __restrict__ grow = Gs + (long long)rr * c + j0;
            for (int jj = lane; jj < jlim; jj += 32) d += grow[jj] * fs[jj];
            d = warp_sum(d);
            if (lane == rr - r0) acc += d;
        }
        __syncwarp();
    }
    const int rr = r0 + lane;
    if (rr < r1) {
        if (rr < c) {
            pc.xp[first + rr] = acc;
        } else {
            T fb = 0;
            for (long long g = pc.fg_ptr[rb + rr]; g < pc.fg_ptr[rb + rr + 1]; ++g) fb += pc.uvec[pc.fg_idx[g]];
            pc.uvec[pc.uvec_off[s] + rr - c] = fb - acc;
        }
    }
}

template <typename T>
__device__ void prec_backward_task(const PcgArgs<T>& a, int4 task) {
    const PrecLayout<T>& pc = a.pc;
    const int lane = threadIdx.x & 31;
    const int s = task.x, j0 = task.y, j1 = task.z;
    const int first = pc.sn_first[s];
    const int c = pc.sn_first[s + 1] - first;
    const long long rb = pc.sn_rowptr[s];
    const int r = (int)(pc.sn_rowptr[s + 1] - rb);
    const T* __restrict__ Gs = pc.G + pc.panel_off[s];
    const int j = j0 + lane;
    const bool valid = j < j1;
    T acc = 0;
    for (int i = j0; i < c; ++i) {
        const T v = pc.xp[first + i];
        if (valid) acc += Gs[(long long)i * c + j] * v;
    }
    for (int i = c; i < r; ++i) {
        const T v = pc.yp[pc.sn_rows[rb + i]];
        if (valid) acc -= Gs[(long long)i * c + j] * v;
    }
    if (valid) pc.yp[first + j] = acc;
}

// Big supernodes (task kind 2): the front vector is assembled in global
// memory by a pre-phase, then each warp computes a few rows of G f.
template <typename T>
__device__ void prec_forward_pre(const PcgArgs<T>& a, const T* in, int4 task) {
    const PrecLayout<T>& pc = a.pc;
    const int lane = threadIdx.x & 31;
    const int s = task.x;
    const int first = pc.sn_first[s];
    const int c = pc.sn_first[s + 1] - first;
    const long long rb = pc.sn_rowptr[s];
    for (int q = task.y + lane; q < task.z; q += 32) {
        T f = 0;
        if (q < c) {
            const int k = first + q;
            f = pc.dscp[k] * in[pc.perm[k]];
        }
        for (long long g = pc.fg_ptr[rb + q]; g < pc.fg_ptr[rb + q + 1]; ++g) f += pc.uvec[pc.fg_idx[g]];
        pc.fvec[rb + q] = f;
    }
}

template <typename T>
__device__ void prec_forward_rows(const PcgArgs<T>& a, int4 task) {
    const PrecLayout<T>& pc = a.pc;
    const int lane = threadIdx.x & 31;
    const int s = task.x;
    const int first = pc.sn_first[s];
    const int c = pc.sn_first[s + 1] - first;
    const long long rb = pc.sn_rowptr[s];
    const T* __restrict__ Gs = pc.G + pc.panel_off[s];
    const T* __restrict__ f = pc.fvec + rb;
    for (int rr = task.y; rr < task.z; ++rr) {
        const int jlim = rr < c ? rr + 1 : c;
        const T* __restrict__ grow = Gs + (long long)rr * c;
        T d = 0;
        for (int j = lane; j < jlim; j += 32) d += grow[j] * f[j];
        d = warp_sum(d);
        if (lane == 0) {
            if (rr < c)
                pc.xp[first + rr] = d;
            else
                pc.uvec[pc.uvec_off[s] + rr - c] = f[rr] - d;
        }
    }
}

template <typename T>
__device__ void prec_backward_pre(const PcgArgs<T>& a, int4 task) {
    const PrecLayout<T>& pc = a.pc;
    const int lane = threadIdx.x & 31;
    const int s = task.x;
    const int first = pc.sn_first[s];
    const int c = pc.sn_first[s + 1] - first;
    const long long rb = pc.sn_rowptr[s];
    for (int q = task.y + lane; q < task.z; q += 32)
        pc.bvec[rb + q] = q < c ? pc.xp[first + q] : -pc.yp[pc.sn_rows[rb + q]];
}

template <typename T>
__device__ void prec_backward_rows(const PcgArgs<T>& a, int4 task) {
    const PrecLayout<T>& pc = a.pc;
    const int lane = threadIdx.x & 31;
    const int s = task.x;
    const int first = pc.sn_first[s];
    const long long rb = pc.sn_rowptr[s];
    const int r = (int)(pc.sn_rowptr[s + 1] - rb);
    const T* __restrict__ GTs = pc.GT + pc.gt_off[s];
    const T* __restrict__ v = pc.bvec + rb;
    for (int j = task.y; j < task.z; ++j) {
        const T* __restrict__ grow = GTs + (long long)j * r;
        T d = 0;
        for (int i = (j & ~31) + lane; i < r; i += 32)
            if (i >= j) d += grow[i] * v[i];
        d = warp_sum(d);
        if (lane == 0) pc.yp[first + j] = d;
    }
}

// z = P^{-1} in; acc_rz += in . z.  Ends without a barrier (the caller's
// reduction provides it).
template <typename T>
__device__ void prec_apply(const PcgArgs<T>& a, const T* in, T* out, double& acc_rz, T* fs,
                           cgx::grid_group& grid) {
    const PrecLayout<T>& pc = a.pc;
    const int gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int lev = 0; lev < pc.nlevels; ++lev) {
        if (pc.fpre_ptr[lev + 1] > pc.fpre_ptr[lev]) {
            for (int tk = pc.fpre_ptr[lev] + gwarp; tk < pc.fpre_ptr[lev + 1]; tk += nwarps)
                prec_forward_pre(a, in, pc.fpre_tasks[tk]);
            grid.sync();
        }
        for (int tk = pc.fwd_ptr[lev] + gwarp; tk < pc.fwd_ptr[lev + 1]; tk += nwarps) {
            const int4 task = pc.fwd_tasks[tk];
            if (task.w == 2)
                prec_forward_rows(a, task);
            else
                prec_forward_task(a, in, task, fs);
        }
        grid.sync();
    }
    for (int lev = pc.nlevels - 1; lev >= 0; --lev) {
        if (pc.bpre_ptr[lev + 1] > pc.bpre_ptr[lev]) {
            for (int tk = pc.bpre_ptr[lev] + gwarp; tk < pc.bpre_ptr[lev + 1]; tk += nwarps)
                prec_backward_pre(a, pc.bpre_tasks[tk]);
            grid.sync();
        }
        for (int tk = pc.bwd_ptr[lev] + gwarp; tk < pc.bwd_ptr[lev + 1]; tk += nwarps) {
            const int4 task = pc.bwd_tasks[tk];
            if (task.w == 2)
                prec_backward_rows(a, task);
            else
                prec_backward_task(a, task);
        }
        grid.sync();
    }
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const int gstride = gridDim.x * blockDim.x;
    for (int i = gtid; i < pc.m; i += gstride) {
        const int k = pc.iperm[i];
        const T zi = pc.dscp[k] * pc.yp[k];
        out[i] = zi;
        acc_rz += (double)in[i] * (double)zi;
    }
}

// H v into phase-B epilogue `mode` (A, barrier, B [, barrier, B2]); ends after
// the partials are written; the caller issues the barrier.
template <typename T>
__device__ void operator_pass(const PcgArgs<T>& a, const T* v, int src, T beta, int mode,
                              double (&acc)[3], cgx::grid_group& grid) {
    phase_a(a, v, src, beta);
    grid.sync();
    phase_b(a, mode, src, beta, acc);
    if (a.sp.n_long) {
        grid.sync();
        phase_b2(a, mode, src, beta, acc);
    }
}

template <typename T>
__global__ void __launch_bounds__(kPcgThreads) k_pcg(PcgArgs<T> a) {
    cgx::grid_group grid = cgx::this_grid();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double scratch[kPcgWarps + 1];
    T* fs = reinterpret_cast<T*>(smem_raw) + (threadIdx.x >> 5) * kStageChunk;
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
        double* P = a.part + (size_t)(red & 1) * gridDim.x * 4;
        double acc[1] = {v}, tot[1];
        write_partials<1>(acc, P, scratch);
        grid.sync();
        read_totals<1>(P, tot, scratch);
        ++red;
        return tot[0];
    };
    auto reduce2 = [&](double (&acc)[3], double (&tot)[3]) {
        double* P = a.part + (size_t)(red & 1) * gridDim.x * 4;
        double a2[2] = {acc[0], acc[1]}, t2[2];
        write_partials<2>(a2, P, scratch);
        grid.sync();
        read_totals<2>(P, t2, scratch);
        tot[0] = t2[0];
        tot[1] = t2[1];
        ++red;
    };
    auto reduce3 = [&](double (&acc)[3], double (&tot)[3]) {
        double* P = a.part + (size_t)(red & 1) * gridDim.x * 4;
        write_partials<3>(acc, P, scratch);
        grid.sync();
        read_totals<3>(P, tot, scratch);
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
        prec_apply(a, a.rhs, a.x, dummy, fs, grid);
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
        prec_apply(a, a.r, a.z, rzacc, fs, grid);
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
                    prec_apply(a, a.r, a.z, rzr, fs, grid);
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
        prec_apply(a, a.r, a.z, rzn, fs, grid);
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

// Standalone preconditioner apply / operator kernels (cooperative as well)
template <typename T>
__global__ void __launch_bounds__(kPcgThreads) k_apply(PcgArgs<T> a, const T* in, T* out) {
    cgx::grid_group grid = cgx::this_grid();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* fs = reinterpret_cast<T*>(smem_raw) + (threadIdx.x >> 5) * kStageChunk;
    double dummy = 0.0;
    prec_apply(a, in, out, dummy, fs, grid);
}

// y = H v  (mode 0 with src = v copied into p first by the host)
template <typename T>
__global__ void __launch_bounds__(kPcgThreads) k_matvec(PcgArgs<T> a) {
    cgx::grid_group grid = cgx::this_grid();
    double acc[3] = {0.0, 0.0, 0.0};
    operator_pass(a, a.p, 0, (T)0, 0, acc, grid);
}

}  // namespace psipm
