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
#include "kernels_tree.cuh"

namespace psipm {

namespace cgx = cooperative_groups;

constexpr int kPcgThreads = 256;
constexpr int kPcgWarps = kPcgThreads / 32;
constexpr int kStageChunk = 64;   // per-warp staging of a small supernode's vector (elements)
// Rows with more nonzeros are split into chunks of this many entries, one
// warp each (16 entries per lane: short dependent-load chains).  Each lane
// sums its entries in index order with one accumulator.  Four interleaved
// accumulators per lane (more loads in flight) were tried: single products
// agreed with these to 1e-14, but on the 4,000 x 1,004,000 set-cover LP the
// PCG then reached its iteration limit 95-285 times per IPM solve instead of
// twice (five runs against three), so this summation order is kept.
constexpr int kLongRow = 512;

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

// Grid barrier of the persistent kernels (cooperative launches: every block
// is resident).  Each block leader adds to one arrival word with a release
// atomic: block 0 adds 2^31 - (blocks - 1), every other block adds 1, so when
// the last block has arrived the word has grown by exactly 2^31 and its top
// bit has flipped, with no reset and no second word.  The leaders poll the top
// bit with acquire loads and a short sleep between them.  Without the sleep
// several hundred leaders spinning on one word keep its L2 slice busy and slow
// down the memory accesses of the blocks that are still working.  A wait
// longer than `polls` polls sets *err and returns.  Once *err is set every
// later wait gives up within kBarrierErrCheck polls (the flag is read every
// kBarrierErrCheck polls, never on the fast path), and the persistent kernels
// leave their iteration loops when they see the flag, so a timed-out kernel
// ends after a few more phases instead of waiting out every later barrier.
// The host clears the word before every launch and reports the flag.
constexpr unsigned int kBarrierPolls = 1u << 24;
constexpr unsigned int kBarrierSleepNs = 64;
constexpr unsigned int kBarrierErrCheck = 16;

struct GridBarrier {
    unsigned int* bar = nullptr;  // [0] arrival word ([1] unused)
    int* err = nullptr;
    unsigned int polls = kBarrierPolls;  // poll limit of one wait

    __device__ __forceinline__ bool failed() const { return *((volatile const int*)err) != 0; }

    __device__ __forceinline__ void sync() const {
        __syncthreads();
        if (threadIdx.x == 0) {
            const unsigned int add = blockIdx.x == 0 ? 0x80000000u - (gridDim.x - 1) : 1u;
            unsigned int old, cur;
            asm volatile("atom.add.release.gpu.u32 %0, [%1], %2;" : "=r"(old) : "l"(bar), "r"(add) : "memory");
            for (unsigned int n = 0;; ++n) {
                asm volatile("ld.acquire.gpu.u32 %0, [%1];" : "=r"(cur) : "l"(bar) : "memory");
                if ((cur ^ old) & 0x80000000u) break;
                if (n >= polls) {
                    atomicExch(err, 1);
                    break;
                }
                if (n % kBarrierErrCheck == kBarrierErrCheck - 1 && failed()) break;
                __nanosleep(kBarrierSleepNs);
            }
        }
        __syncthreads();
    }
};

// Triangular-solve task records: everything a task needs sits in one
// 48-byte record, so a warp reaches its data after a single load.
struct __align__(16) FwdTask {
    long long g;      // panel offset of the task's first row (G, row-major r x c)
    long long f;      // front-vector offset of the supernode (sn_rowptr)
    long long u;      // update-vector offset of the supernode (fdst base)
    int first, c;     // first pivot column (permuted), pivot columns
    int i0, i1;       // rows [i0, i1) of the supernode
    int j0, s;        // first column of the chunk; s >= 0 marks a fused small supernode
};
struct __align__(16) BwdTask {
    long long g;      // GT offset of the task's first row (GT, row-major c x r)
    long long rb;     // sn_rowptr of the supernode
    int first, c, r;  // first pivot column, pivot columns, front rows
    int j0, j1;       // GT rows [j0, j1) (pivot columns of the supernode)
    int i0;           // first front row of the chunk
    int s, pad;       // s >= 0 marks a fused small supernode
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
    const int* fown = nullptr;   // per front row: permuted column of a pivot row, -1 below
    const int* fdst = nullptr;   // per update-vector entry: the parent's front row, -1 at roots
    long long nfront = 0;        // front rows of all supernodes
    int nlevels = 0;
    const int* fwd_ptr = nullptr;
    const FwdTask* fwd_tasks = nullptr;
    const int* bwd_ptr = nullptr;
    const BwdTask* bwd_tasks = nullptr;
    T* fvec = nullptr;                // front vectors f, indexed like sn_rows
    const T* GT = nullptr;             // transposed panels of big supernodes (c x r row-major)
    const long long* gt_off = nullptr;
    long long* trace = nullptr;  // optional: %globaltimer after every barrier of an apply
    int trace_cap = 0;
    T* xp = nullptr;
    T* yp = nullptr;
    // fixed-order accumulation (deterministic != 0; no floating-point atomics):
    // every partial sum goes to its own slot and the contributor that completes
    // a destination (an atomic arrival count) adds the slots in slot order.
    // Otherwise partial sums are added with FP64 atomics (faster; the order,
    // and so the last bits, can change from run to run).
    int deterministic = 0;
    const int* frow_nch = nullptr;       // per front row: forward tasks that cover it (0: fused supernode)
    const long long* frow_slot = nullptr;
    int* fcount = nullptr;               // per front row: arrivals
    T* fslots = nullptr;
    const int* ecnt = nullptr;           // per front row: child update rows that add into it
    const long long* eslot_off = nullptr;
    const long long* uslot = nullptr;    // per update row: its slot in the parent's list
    int* ecount = nullptr;
    T* eslots = nullptr;
    const int* brow_nch = nullptr;       // per permuted column: backward tasks that cover it (0: fused)
    const long long* brow_slot = nullptr;
    int* bcount = nullptr;
    T* bslots = nullptr;
    // extracted dense columns: the Woodbury correction of the apply (lr_q = 0: none)
    int lr_q = 0;
    const int* lr_ptr = nullptr;      // q + 1 offsets into lr_row / lr_val
    const int* lr_row = nullptr;
    const double* lr_val = nullptr;
    const double* lr_B = nullptr;     // P_base^{-1} A_L, m x q column-major
    const double* lr_chol = nullptr;  // Cholesky factor of the q x q core, row-major lower
    double* lr_part = nullptr;        // per-block partial sums, gridDim.x x kLowRankMax
    // network tree-plus-diagonal preconditioner instead of the supernodal factor
    // (tree.nlevels > 0; FP64 handles only)
    TreeLayout tree;
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
    GridBarrier gb;
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
    const T* t = a.t;  // rewritten by phase A every pass: not __restrict__
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

// one warp per long row adds its chunk sums (lane-strided, then a butterfly:
// a fixed order) and runs the row's epilogue
template <typename T, typename P>
__device__ void phase_b2(const PcgArgs<T, P>& a, int mode, int src, T beta, double (&acc)[3]) {
    const int lane = threadIdx.x & 31;
    const int gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int l = gwarp; l < a.sp.n_long; l += nwarps) {
        T s = 0;
        for (int c = a.sp.long_chunk_ptr[l] + lane; c < a.sp.long_chunk_ptr[l + 1]; c += 32) s += a.chunk_part[c];
        s = warp_sum(s);
        if (lane == 0) row_epilogue(a, mode, src, beta, a.sp.long_rows[l], s, acc);
    }
}

// ---- preconditioner apply ----------------------------------------------------
// P^{-1} = Ds Pi^T L^{-T} L^{-1} Pi Ds with L supernodal.  Each supernode s
// (c pivot columns, r rows) stores G = [L11^{-1} ; L21 L11^{-1}] (r x c,
// row-major) and its transpose GT (c x r, row-major), so both sweeps are
// dense matrix-vector products over contiguous rows:
//   forward  (levels bottom-up):  f_s = [b_s ; 0] + sum_children u_child
//                                 x_s = G_top f_top,  u_s = f_bot - G_bot f_top
//   backward (levels top-down):   v = [x_s ; -y(rows below)]
//                                 y_s = G^T v
// The forward sweep pushes: every supernode's update rows u_s go to their
// parent's f (fvec at fdst), so a level needs no gather phase, and one flat
// pass before the first level writes every f = [b_s ; 0] and clears x, y (and
// the arrival counts).  Partial sums (a chunk of a row, a child's update row)
// are added with FP64 atomics, or, on a handle set to be deterministic, each
// is stored in its own slot and whichever contributor completes a destination
// adds that destination's slots in slot order, so an application gives the
// same bits on every run.  The backward sweep gathers v into registers inside
// each task.
// Big supernodes are cut into 2-D tasks of kApplyRows output rows x
// kApplyChunk contraction entries; each lane holds kLaneCols entries of the
// vector chunk and loads its kLaneCols columns of four rows at once.
constexpr int kApplyRows = 4;
constexpr int kApplyChunk = 128;
constexpr int kLaneCols = kApplyChunk / 32;

// warp sums of four values; lane k (k < 4) returns the total of v[k]
template <typename P>
__device__ __forceinline__ P warp_sum4(P (&v)[4]) {
    const int lane = threadIdx.x & 31;
    // exchange halves so that each lane keeps two of the four partial sums
    const bool hi16 = lane & 16;
    P a0 = hi16 ? v[0] : v[2], a1 = hi16 ? v[1] : v[3];
    P k0 = hi16 ? v[2] : v[0], k1 = hi16 ? v[3] : v[1];
    k0 += __shfl_xor_sync(0xffffffffu, a0, 16);
    k1 += __shfl_xor_sync(0xffffffffu, a1, 16);
    // lanes < 16 hold rows {0,1}, lanes >= 16 rows {2,3}
    const bool hi8 = lane & 8;
    P s = hi8 ? k0 : k1;
    P keep = hi8 ? k1 : k0;
    keep += __shfl_xor_sync(0xffffffffu, s, 8);
    // lane group (bit4, bit3) now holds row 2*bit4 + bit3
    keep += __shfl_xor_sync(0xffffffffu, keep, 4);
    keep += __shfl_xor_sync(0xffffffffu, keep, 2);
    keep += __shfl_xor_sync(0xffffffffu, keep, 1);
    // row k lives in lanes 8k .. 8k+7: bring it to lane k
    return __shfl_sync(0xffffffffu, keep, (lane & 3) * 8);
}

__device__ __forceinline__ void prefetch_l2(const void* p) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// Slot protocol: store this contribution in its slot; when the destination
// expects more than one, publish it (fence, arrival count) and report whether
// this was the last one, which then sees every slot (fence) and sums them in
// slot order.
template <typename P>
__device__ __forceinline__ bool slot_arrive(P* slots, long long slot, P v, int expected, int* count) {
    slots[slot] = v;
    if (expected <= 1) return true;
    __threadfence();
    const bool last = atomicAdd(count, 1) == expected - 1;
    if (last) __threadfence();
    return last;
}
template <typename P>
__device__ __forceinline__ P slot_sum(const P* slots, long long base, int count, P init) {
    P s = init;
    for (int k = 0; k < count; ++k) s += __ldcg(slots + base + k);
    return s;
}

// An update row u of a child adds into its parent's front row fdst[u]; the
// last of the parent row's contributors writes f = base + sum of the slots.
template <typename P>
__device__ __forceinline__ void deliver_update(const PrecLayout<P>& pc, long long u, P val) {
    const int e = pc.fdst[u];
    if (e < 0) return;
    if (!pc.deterministic) {
        atomicAdd(&pc.fvec[e], val);
        return;
    }
    const int ne = pc.ecnt[e];
    if (slot_arrive(pc.eslots, pc.uslot[u], val, ne, pc.ecount + e))
        pc.fvec[e] = slot_sum(pc.eslots, pc.eslot_off[e], ne, __ldcg(pc.fvec + e));
}

// forward task: rows [i0, i1) (at most four) of G against f[j0, j0 + kApplyChunk).
// Every lane loads a clamped in-row index and masks the product, so the
// sixteen loads carry no branches and issue together.
template <typename P>
__device__ void prec_forward_gemv(const PrecLayout<P>& pc, const FwdTask& t) {
    const int lane = threadIdx.x & 31;
    const int c = t.c, i0 = t.i0, i1 = t.i1, j0 = t.j0;
    const P* __restrict__ G = pc.G + t.g;
    const P* f = pc.fvec + t.f;
    const int j1 = min(c, j0 + kApplyChunk);
    const int ii = i0 + lane;  // the row lane k < 4 finishes
    P fr[kLaneCols];
#pragma unroll
    for (int q = 0; q < kLaneCols; ++q) {
        const int j = j0 + lane + 32 * q;
        const P fv = f[min(j, c - 1)];
        fr[q] = j < j1 ? fv : (P)0;
    }
    P d[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int row = i0 + k;
        // G_top is lower triangular; rows past i1 contribute nothing
        const int jend = row < i1 ? (row < c ? min(j1, row + 1) : j1) : j0;
        const P* __restrict__ g = G + (long long)min(k, i1 - i0 - 1) * c;
        P acc = 0;
#pragma unroll
        for (int q = 0; q < kLaneCols; ++q) {
            const int j = j0 + lane + 32 * q;
            const P gv = g[min(j, c - 1)];
            acc += j < jend ? gv * fr[q] : (P)0;
        }
        d[k] = acc;
    }
    const P v = warp_sum4(d);
    if (lane < 4 && ii < i1 && !pc.deterministic) {
        if (ii < c)
            atomicAdd(&pc.xp[t.first + ii], v);
        else  // u pushed into the parent's front vector; f_bot once, with the first chunk
            deliver_update(pc, t.u + ii - c, (j0 == 0 ? f[ii] : (P)0) - v);
    } else if (lane < 4 && ii < i1) {
        // this chunk's part of row ii; the row's last chunk finishes it:
        // x = G_top f_top (pivot rows), u = f_bot - G_bot f_top (update rows)
        const long long g = t.f + ii;
        const int nch = pc.frow_nch[g];
        if (slot_arrive(pc.fslots, pc.frow_slot[g] + j0 / kApplyChunk, v, nch, pc.fcount + g)) {
            const P sum = slot_sum(pc.fslots, pc.frow_slot[g], nch, (P)0);
            if (ii < c)
                pc.xp[t.first + ii] = sum;
            else
                deliver_update(pc, t.u + ii - c, __ldcg(pc.fvec + g) - sum);
        }
    }
}

// backward task: GT rows [j0, j1) (at most four) against v[i0, i0 + kApplyChunk)
template <typename P>
__device__ void prec_backward_gemv(const PrecLayout<P>& pc, const BwdTask& t) {
    const int lane = threadIdx.x & 31;
    const int c = t.c, r = t.r, j0 = t.j0, j1 = t.j1, i0 = t.i0;
    const int i1 = min(r, i0 + kApplyChunk);
    const P* __restrict__ GT = pc.GT + t.g;
    P vr[kLaneCols];
#pragma unroll
    for (int q = 0; q < kLaneCols; ++q) {
        const int i = i0 + lane + 32 * q;
        vr[q] = i < i1 ? (i < c ? pc.xp[t.first + i] : -pc.yp[pc.sn_rows[t.rb + i]]) : (P)0;
    }
    P d[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int jj = j0 + k;
        const int ibeg = jj < j1 ? max(i0, jj) : i1;  // G[i, j] = 0 for i < j
        const P* __restrict__ g = GT + (long long)min(k, j1 - j0 - 1) * r;
        P acc = 0;
#pragma unroll
        for (int q = 0; q < kLaneCols; ++q) {
            const int i = i0 + lane + 32 * q;
            const P gv = g[min(i, r - 1)];
            acc += (i >= ibeg && i < i1) ? gv * vr[q] : (P)0;
        }
        d[k] = acc;
    }
    const P v = warp_sum4(d);
    if (lane < 4 && j0 + lane < j1 && !pc.deterministic) {
        atomicAdd(&pc.yp[t.first + j0 + lane], v);
    } else if (lane < 4 && j0 + lane < j1) {
        const int col = t.first + j0 + lane;
        const int nch = pc.brow_nch[col];
        if (slot_arrive(pc.bslots, pc.brow_slot[col] + (i0 / kApplyChunk - j0 / kApplyChunk), v, nch,
                        pc.bcount + col))
            pc.yp[col] = slot_sum(pc.bslots, pc.brow_slot[col], nch, (P)0);
    }
}

// Small supernodes (r <= kSmallRows, c <= 32): one warp does the whole
// supernode in one task with the vector staged in shared memory and one lane
// per output row.
constexpr int kSmallRows = 64;

template <typename P>
__device__ void prec_forward_small(const PrecLayout<P>& pc, int s, P* fs) {
    const int lane = threadIdx.x & 31;
    const int first = pc.sn_first[s];
    const int c = pc.sn_first[s + 1] - first;
    const long long rb = pc.sn_rowptr[s];
    const int r = (int)(pc.sn_rowptr[s + 1] - rb);
    const long long uo = pc.uvec_off[s];
    for (int q = lane; q < r; q += 32) fs[q] = pc.fvec[rb + q];
    __syncwarp();
    const P* __restrict__ Gs = pc.G + pc.panel_off[s];
    for (int row = lane; row < r; row += 32) {
        const int jlim = row < c ? row + 1 : c;
        const P* __restrict__ g = Gs + (long long)row * c;
        P d = 0;
#pragma unroll 8
        for (int j = 0; j < jlim; ++j) d += g[j] * fs[j];
        if (row < c)
            pc.xp[first + row] = d;
        else
            deliver_update(pc, uo + row - c, fs[row] - d);
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
#pragma unroll 8
        for (int i = lane; i < r; ++i) d += gt[i] * fs[i];
        pc.yp[first + lane] = d;
    }
    __syncwarp();
}

constexpr int kLowRankMax = 8;

// Woodbury correction for the extracted dense columns A_L
// (psipm_active_pool.py:949-956): with z0 = P_base^{-1} r already in out,
//   z = z0 - B C^{-1} (A_L^T z0),  B = P_base^{-1} A_L,  C = Theta_L + A_L^T B.
// The q dot products go through per-block partials that every block sums in
// the same order, so all blocks hold the same coefficients.
template <typename P, typename IT>
__device__ void prec_low_rank(const PrecLayout<P>& pc, const IT* in, IT* out, double& acc_rz,
                              const GridBarrier& grid) {
    __shared__ double scr[32];
    __shared__ double coef[2 * kLowRankMax];
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const int gstride = gridDim.x * blockDim.x;
    const int q = pc.lr_q;
    grid.sync();  // z0 complete
    for (int a = 0; a < q; ++a) {
        double t = 0.0;
        for (int e = pc.lr_ptr[a] + gtid; e < pc.lr_ptr[a + 1]; e += gstride)
            t += pc.lr_val[e] * (double)__ldcg(out + pc.lr_row[e]);
        t = block_sum(t, scr);
        if (threadIdx.x == 0) pc.lr_part[blockIdx.x * kLowRankMax + a] = t;
    }
    grid.sync();
    if (threadIdx.x < q) {
        double t = 0.0;
        for (int b = 0; b < (int)gridDim.x; ++b) t += __ldcg(pc.lr_part + b * kLowRankMax + threadIdx.x);
        coef[threadIdx.x] = t;
    }
    __syncthreads();
    if (threadIdx.x == 0) {  // c = L^{-T} L^{-1} t
        double* c = coef + kLowRankMax;
        for (int i = 0; i < q; ++i) {
            double v = coef[i];
            for (int j = 0; j < i; ++j) v -= pc.lr_chol[i * q + j] * c[j];
            c[i] = v / pc.lr_chol[i * q + i];
        }
        for (int i = q - 1; i >= 0; --i) {
            double v = c[i];
            for (int j = i + 1; j < q; ++j) v -= pc.lr_chol[j * q + i] * c[j];
            c[i] = v / pc.lr_chol[i * q + i];
        }
    }
    __syncthreads();
    for (int i = gtid; i < pc.m; i += gstride) {
        double z = (double)out[i];
        for (int a = 0; a < q; ++a) z -= pc.lr_B[(long long)a * pc.m + i] * coef[kLowRankMax + a];
        out[i] = (IT)z;
        acc_rz += (double)in[i] * z;
    }
}

// Tree-plus-diagonal solve (kernels_tree.cuh) over the whole grid: one grid
// barrier per level and direction; the same operations in the same order as
// the reference's TreePreconditioner.solve (psipm_v3_1_hsd.py:764-776).
template <typename IT>
__device__ void prec_tree(const TreeLayout& t, const IT* in, IT* out, double& acc_rz, const GridBarrier& grid) {
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const int gstride = gridDim.x * blockDim.x;
    double* v = t.val;
    for (int i = gtid; i < t.m; i += gstride) v[i] = (double)in[i];
    grid.sync();
    for (int l = t.nlevels - 2; l >= 0; --l) {  // parents at level l gather their children
        for (int q = t.level_ptr[l] + gtid; q < t.level_ptr[l + 1]; q += gstride) {
            const int p = t.level_nodes[q];
            double a = v[p];
            for (int k = t.kid_ptr[p]; k < t.kid_ptr[p + 1]; ++k) {
                const int c = t.kids[k];
                a = __dadd_rn(a, __dmul_rn(-t.mult[c], v[c]));
            }
            v[p] = a;
        }
        grid.sync();
    }
    for (int i = gtid; i < t.m; i += gstride) v[i] = __ddiv_rn(v[i], t.pivot[i]);
    grid.sync();
    for (int l = 1; l < t.nlevels; ++l) {
        for (int q = t.level_ptr[l] + gtid; q < t.level_ptr[l + 1]; q += gstride) {
            const int c = t.level_nodes[q];
            v[c] = __dsub_rn(v[c], __dmul_rn(t.mult[c], v[t.parent[c]]));
        }
        grid.sync();
    }
    for (int i = gtid; i < t.m; i += gstride) {
        const IT zi = (IT)v[i];
        out[i] = zi;
        acc_rz += (double)in[i] * (double)zi;
    }
}

// z = P^{-1} in; acc_rz += in . z.  Ends without a barrier (the caller's
// reduction provides it).
template <typename P, typename IT>
__device__ void prec_apply(const PrecLayout<P>& pc, const IT* in, IT* out, double& acc_rz, P* fs,
                           const GridBarrier& grid) {
    if (pc.tree.nlevels > 0) {
        prec_tree(pc.tree, in, out, acc_rz, grid);
        return;
    }
    const int gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const int gstride = gridDim.x * blockDim.x;
    int ntrace = 0;
    const bool tracer = pc.trace && blockIdx.x == 0 && threadIdx.x == 0;
    auto mark = [&]() {
        if (tracer && ntrace < pc.trace_cap) pc.trace[ntrace++] = global_ns();
    };
    mark();
    // f = [Ds Pi in ; 0] for every supernode, x = y = 0
    for (long long g = gtid; g < pc.nfront; g += gstride) {
        const int k = pc.fown[g];
        pc.fvec[g] = k >= 0 ? pc.dscp[k] * (P)in[pc.perm[k]] : (P)0;
    }
    if (pc.deterministic)
        for (long long g = gtid; g < pc.nfront; g += gstride) {
            pc.fcount[g] = 0;
            pc.ecount[g] = 0;
        }
    for (int k = gtid; k < pc.m; k += gstride) {
        pc.xp[k] = 0;
        pc.yp[k] = 0;
        if (pc.deterministic) pc.bcount[k] = 0;
    }
    grid.sync();
    mark();
    // task kind (int4.w for fused tasks is -1): fused small supernode or 2-D GEMV
    for (int lev = 0; lev < pc.nlevels; ++lev) {
        for (int tk = pc.fwd_ptr[lev] + gwarp; tk < pc.fwd_ptr[lev + 1]; tk += nwarps) {
            // the record of this warp's next task is pulled into L2 meanwhile
            if ((threadIdx.x & 31) == 0 && tk + nwarps < pc.fwd_ptr[lev + 1]) prefetch_l2(pc.fwd_tasks + tk + nwarps);
            const FwdTask task = pc.fwd_tasks[tk];
            if (task.s >= 0)
                prec_forward_small(pc, task.s, fs);
            else
                prec_forward_gemv(pc, task);
        }
        grid.sync();
        mark();
    }
    for (int lev = pc.nlevels - 1; lev >= 0; --lev) {
        for (int tk = pc.bwd_ptr[lev] + gwarp; tk < pc.bwd_ptr[lev + 1]; tk += nwarps) {
            if ((threadIdx.x & 31) == 0 && tk + nwarps < pc.bwd_ptr[lev + 1]) prefetch_l2(pc.bwd_tasks + tk + nwarps);
            const BwdTask task = pc.bwd_tasks[tk];
            if (task.s >= 0)
                prec_backward_small(pc, task.s, fs);
            else
                prec_backward_gemv(pc, task);
        }
        grid.sync();
        mark();
    }
    const bool lr = pc.lr_q > 0;
    for (int i = gtid; i < pc.m; i += gstride) {
        const int k = pc.iperm[i];
        const IT zi = (IT)(pc.dscp[k] * pc.yp[k]);
        out[i] = zi;
        if (!lr) acc_rz += (double)in[i] * (double)zi;
    }
    if (lr) prec_low_rank(pc, in, out, acc_rz, grid);
}

// H v into phase-B epilogue `mode` (A, barrier, B [, barrier, B2]); ends after
// the partials are written; the caller issues the barrier.
template <typename T, typename P>
__device__ void operator_pass(const PcgArgs<T, P>& a, const T* v, int src, T beta, int mode,
                              double (&acc)[3], const GridBarrier& grid) {
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
    const GridBarrier grid = a.gb;
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
        if (grid.failed()) break;  // a barrier wait timed out: the host reports it
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
        ok = info == 0;
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

// Grid-barrier cost probe: `count` barriers, nothing else.  Block
// `skip_block` (-1: none) returns without arriving, so the other blocks'
// first wait runs out its poll limit: the timeout path, without a fault.
__global__ void k_barrier_probe(int count, long long* out, GridBarrier grid, int skip_block) {
    if ((int)blockIdx.x == skip_block) return;
    const long long t0 = global_ns();
    for (int i = 0; i < count; ++i) grid.sync();
    if (blockIdx.x == 0 && threadIdx.x == 0) *out = global_ns() - t0;
}

// Standalone preconditioner apply / operator kernels (cooperative as well)
template <typename T, typename P>
__global__ void __launch_bounds__(kPcgThreads, 3) k_apply(PcgArgs<T, P> a, const T* in, T* out) {
    const GridBarrier grid = a.gb;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    P* fs = reinterpret_cast<P*>(smem_raw) + (threadIdx.x >> 5) * kStageChunk;
    double dummy = 0.0;
    prec_apply(a.pc, in, out, dummy, fs, grid);
}

// y = H v  (mode 0 with src = v copied into p first by the host)
template <typename T, typename P>
__global__ void __launch_bounds__(kPcgThreads, 3) k_matvec(PcgArgs<T, P> a) {
    const GridBarrier grid = a.gb;
    double acc[3] = {0.0, 0.0, 0.0};
    operator_pass(a, a.p, 0, (T)0, 0, acc, grid);
}

}  // namespace psipm
