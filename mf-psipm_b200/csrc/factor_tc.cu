// Trailing updates of the FP32 factor's large fronts on the 5th-generation
// tensor cores (tcgen05.mma kind::tf32, accumulators in tensor memory).
//
// One CTA of 256 threads computes one 128 x 128 tile of the blocked
// right-looking Cholesky's SYRK step
//     F[i, j] -= sum_k P[i, k] P[j, k],   P = F[:, k0 : k0 + kb]
// (the reference factors the same matrix with CHOLMOD on the CPU,
// psipm_active_pool.py:839-897).  K runs in stages of 32 FP32 values, the
// width of one 128-byte swizzled shared-memory row; while the tensor core
// works on one stage, the threads already hold the next stage's values in
// registers.  The threads load the column-major panel with coalesced 4-byte
// loads (consecutive threads, consecutive rows), split each value into a TF32
// head (round to nearest) and its FP32 remainder, and store both as K-major
// tiles in the canonical 128-byte swizzle; one thread issues hi*hi + hi*lo +
// lo*hi (3xTF32: the products carry ~22 significant bits, FP32-level) or
// hi*hi alone, and commits to a shared-memory barrier.  The epilogue reads
// the accumulator out of tensor memory (32x32b.x32 loads) and subtracts it
// from the front's lower triangle with coalesced accesses.
//
// Every wait on the completion barrier is bounded (2 s of %globaltimer): on
// expiry the CTA records kTcErrWait, waits once more with the same bound, frees
// its tensor memory and returns.
#include "common.cuh"
#include "factor_tc.h"

namespace psipm {
namespace {

constexpr int kTm = 128;                 // tile rows = tensor-memory lanes
constexpr int kTn = 128;                 // tile columns = tensor-memory columns (FP32)
constexpr int kKc = 32;                  // K per stage (one 128-byte row of FP32)
constexpr int kOpBytes = kTm * kKc * 4;  // one operand tile of one stage: 16 KB
constexpr int kTcThreads = 256;
// 3 passes: one stage of A hi/lo and B hi/lo; 1 pass: two stages of A and B
// heads.  65 KB either way (1 KB for alignment): up to three CTAs per SM.
constexpr int kStages3 = 1, kStages1 = 2;
constexpr size_t kTcSmem = (size_t)4 * kOpBytes + 1024;
constexpr unsigned long long kWaitNs = 2000000000ull;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long now_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Byte offset of the 16-byte chunk `kchunk` (K values 4 kchunk .. 4 kchunk + 3)
// of row m in a 128 x 32 FP32 K-major tile, 128-byte swizzle: 8-row groups
// 1024 B apart, rows 128 B apart, chunk index XOR row-in-group.
__device__ __forceinline__ uint32_t sw128_offset(int m, int kchunk) {
    return (uint32_t)((m >> 3) * 1024 + (m & 7) * 128 + (((kchunk ^ m) & 7) << 4));
}

// Shared-memory matrix descriptor of a K-major, 128-byte-swizzled operand
// starting at `addr` (the tile base is 1024-byte aligned; a K offset inside
// the swizzle row is added to the start address).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr) {
    return (uint64_t)((addr >> 4) & 0x3FFF)  // start address, 16-byte units
           | ((uint64_t)1 << 16)             // leading-dimension offset (unused: swizzled K-major)
           | ((uint64_t)(1024 >> 4) << 32)   // stride-dimension offset: 8-row groups
           | ((uint64_t)1 << 46)             // descriptor version
           | ((uint64_t)2 << 61);            // 128-byte swizzle
}

// Instruction descriptor: D FP32, A and B TF32, both K-major, N = 128, M = 128.
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kTn >> 3) << 17) |
                            ((uint32_t)(kTm >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t"
        "}\n" ::"r"(tmem),
        "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t parity) {
    const unsigned long long t0 = now_ns();
    while (true) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t"
            "}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
        if (now_ns() - t0 > kWaitNs) return false;
    }
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
          "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ float tf32_round(float x) {
    uint32_t u;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(u) : "f"(x));
    return __uint_as_float(u);
}

// The 16 K values (chunks kc .. kc + 3) of operand row m: front row `row` of
// the panel columns k0 + kbase + 4 kc ...; zero past kb or outside the front.
__device__ __forceinline__ void load_row(const float* __restrict__ F, long long r, int row, bool valid, int k0,
                                         int kbase, int kb, int kc, float (&v)[16]) {
#pragma unroll
    for (int q = 0; q < 16; ++q) {
        const int k = kbase + kc * 4 + q;
        v[q] = (valid && k < kb) ? __ldg(F + (long long)(k0 + k) * r + row) : 0.0f;
    }
}

// Store them as TF32 heads (and, for 3 passes, FP32 remainders) into the
// swizzled K-major tiles.
template <int PASSES>
__device__ __forceinline__ void store_row(const float (&v)[16], int m, int kc, unsigned char* hi,
                                          unsigned char* lo) {
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        float4 h, l;
        h.x = tf32_round(v[4 * c + 0]);
        h.y = tf32_round(v[4 * c + 1]);
        h.z = tf32_round(v[4 * c + 2]);
        h.w = tf32_round(v[4 * c + 3]);
        const uint32_t off = sw128_offset(m, kc + c);
        *reinterpret_cast<float4*>(hi + off) = h;
        if (PASSES == 3) {
            l.x = v[4 * c + 0] - h.x;
            l.y = v[4 * c + 1] - h.y;
            l.z = v[4 * c + 2] - h.z;
            l.w = v[4 * c + 3] - h.w;
            *reinterpret_cast<float4*>(lo + off) = l;
        }
    }
}

template <int PASSES, int STAGES>
__global__ void __launch_bounds__(kTcThreads, 2)
    k_syrk_tc(float* __restrict__ F, int r, int k0, int kb, int jend, int nti, int* err) {
    extern __shared__ __align__(1024) unsigned char tc_smem_raw[];
    __shared__ uint64_t bars[STAGES];
    __shared__ uint32_t tmem_slot;
    unsigned char* smem = tc_smem_raw + ((1024u - (smem_u32(tc_smem_raw) & 1023u)) & 1023u);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    // tile (ti, tj) with ti >= tj, enumerated column by column
    int t = blockIdx.x, tj = 0;
    while (t >= nti - tj) {
        t -= nti - tj;
        ++tj;
    }
    const int ti = tj + t;
    const int base = k0 + kb;
    const int i0 = base + ti * kTm, j0 = base + tj * kTn;
    const bool diag = ti == tj;

    if (tid == 0) {
        for (int s = 0; s < STAGES; ++s) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bars[s])));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                     "r"(kTn));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;

    const int m = tid & (kTm - 1);  // operand row this thread fills
    const int kc = (tid >> 7) * 4;  // first 16-byte chunk it fills (of 8 per row)
    const int nchunk = (kb + kKc - 1) / kKc;
    uint32_t parity = 0;  // bit s: parity of the next completion of stage s (thread 0's view)
    int committed = 0;    // stages committed so far (thread 0's view)
    bool ok = true;
    constexpr int kStageBytes = (PASSES == 3 ? 4 : 2) * kOpBytes;  // A hi [lo], B hi [lo]
    // the next stage's values are loaded into registers while the tensor core
    // works on the current one
    float va[16], vb[16];
    load_row(F, r, i0 + m, i0 + m < r, k0, 0, kb, kc, va);
    if (!diag) load_row(F, r, j0 + m, j0 + m < jend, k0, 0, kb, kc, vb);
    for (int q = 0; q < nchunk; ++q) {
        const int s = q % STAGES;
        unsigned char* st = smem + s * kStageBytes;
        unsigned char* sb = st + (PASSES == 3 ? 2 : 1) * kOpBytes;
        if (q >= STAGES) {  // the tensor core has finished reading this stage
            bool mine = true;
            if (tid == 0) {
                mine = bar_wait(smem_u32(&bars[s]), (parity >> s) & 1u);
                parity ^= 1u << s;
            }
            ok = __syncthreads_and(mine);
            if (!ok) break;
        }
        store_row<PASSES>(va, m, kc, st, st + kOpBytes);
        if (!diag) store_row<PASSES>(vb, m, kc, sb, sb + kOpBytes);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (q + 1 < nchunk) {
            load_row(F, r, i0 + m, i0 + m < r, k0, (q + 1) * kKc, kb, kc, va);
            if (!diag) load_row(F, r, j0 + m, j0 + m < jend, k0, (q + 1) * kKc, kb, kc, vb);
        }
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t a_hi = smem_u32(st), a_lo = a_hi + kOpBytes;
            const uint32_t b_hi = diag ? a_hi : smem_u32(sb), b_lo = b_hi + kOpBytes;
#pragma unroll
            for (int ks = 0; ks < kKc / 8; ++ks) {  // K = 8 TF32 values (32 bytes) per instruction
                const uint32_t off = ks * 32;
                const uint32_t acc = (q > 0 || ks > 0) ? 1u : 0u;
                if (PASSES == 3) {
                    mma_tf32(tmem, sw128_desc(a_lo + off), sw128_desc(b_hi + off), acc);
                    mma_tf32(tmem, sw128_desc(a_hi + off), sw128_desc(b_lo + off), 1u);
                    mma_tf32(tmem, sw128_desc(a_hi + off), sw128_desc(b_hi + off), 1u);
                } else {
                    mma_tf32(tmem, sw128_desc(a_hi + off), sw128_desc(b_hi + off), acc);
                }
            }
            mma_commit(smem_u32(&bars[s]));
            ++committed;
        }
    }
    {  // the last commit covers every MMA issued before it (also after a failed wait)
        bool mine = true;
        if (tid == 0 && committed > 0) {
            const int sl = (committed - 1) % STAGES;
            mine = bar_wait(smem_u32(&bars[sl]), (parity >> sl) & 1u);
            if (!mine || !ok) atomicOr(err, kTcErrWait);
        }
        ok = __syncthreads_and(mine && ok);
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (ok) {
        // warp w reads lanes 32 (w % 4) .. + 31 (its rows) and columns 64 (w / 4) .. + 63
        const int row = (warp & 3) * 32 + lane;
        const int i = i0 + row;
        const uint32_t lane_base = tmem + ((uint32_t)((warp & 3) * 32) << 16);
#pragma unroll 1
        for (int c0 = (warp >> 2) * 64; c0 < (warp >> 2) * 64 + 64; c0 += 32) {
            uint32_t v[32];
            tmem_ld32(lane_base + (uint32_t)c0, v);
            if (i < r) {
#pragma unroll
                for (int qq = 0; qq < 32; ++qq) {
                    const int j = j0 + c0 + qq;
                    if (j < jend && j <= i) {
                        float* p = F + (long long)j * r + i;
                        *p -= __uint_as_float(v[qq]);
                    }
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTn));
    }
}

}  // namespace

size_t syrk_update_tc_smem() { return kTcSmem; }

void syrk_update_tc(float* F, int r, int k0, int kb, int jend, int passes, int* err, cudaStream_t st) {
    static bool attributes_set = false;
    if (!attributes_set) {
        PSIPM_CUDA(cudaFuncSetAttribute(k_syrk_tc<3, kStages3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)kTcSmem));
        PSIPM_CUDA(cudaFuncSetAttribute(k_syrk_tc<1, kStages1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)kTcSmem));
        // the largest shared-memory carveout: three 65 KB CTAs per SM
        PSIPM_CUDA(cudaFuncSetAttribute(k_syrk_tc<3, kStages3>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                        (int)cudaSharedmemCarveoutMaxShared));
        PSIPM_CUDA(cudaFuncSetAttribute(k_syrk_tc<1, kStages1>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                        (int)cudaSharedmemCarveoutMaxShared));
        attributes_set = true;
    }
    const int base = k0 + kb;
    if (kb <= 0 || base >= r || jend <= base) return;
    const int nti = (r - base + kTm - 1) / kTm;
    const int ntj = (jend - base + kTn - 1) / kTn;
    // tiles (ti, tj), tj < ntj <= nti, ti >= tj
    const long long tiles = (long long)ntj * nti - (long long)ntj * (ntj - 1) / 2;
    if (tiles > 0x7fffffffLL) throw Failure(PSIPM_ERR_UNSUPPORTED, "front too large for the tensor-core update");
    if (passes == 1)
        k_syrk_tc<1, kStages1><<<(unsigned)tiles, kTcThreads, kTcSmem, st>>>(F, r, k0, kb, jend, nti, err);
    else
        k_syrk_tc<3, kStages3><<<(unsigned)tiles, kTcThreads, kTcSmem, st>>>(F, r, k0, kb, jend, nti, err);
    PSIPM_CHECK_LAUNCH();
}

}  // namespace psipm
