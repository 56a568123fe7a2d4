// Allocation-free operator product y = A diag(w) A^T v + delta v.
//
// Some callers of this library cannot allocate device memory: an
// interior-point loop that runs inside a host framework which owns the whole
// device pool (every byte pre-reserved by its allocator), code that must not
// call cudaMalloc/cudaFree because those calls synchronise the device, or a
// real-time solver that has to prove a fixed memory footprint up front.
// psipm_normal_matvec_static serves them: the caller passes every input and
// the output in its own device memory, and the one intermediate vector
// t = w o (A^T v) lives in a fixed array in this file, g_matvec_scratch, that
// every GPU loading the library holds until the process exits.
//
// Rules of use:
//  * n must not exceed PSIPM_STATIC_SCRATCH_MAX (1,048,576 columns, 8 MiB of
//    FP64 scratch); larger calls are rejected with PSIPM_ERR_ARGUMENT.
//  * The first call on a device looks up the array's device address
//    (cudaGetSymbolAddress) with that device current and caches it; make that
//    first call before any stream capture.
//  * All calls share the array and it keeps the last call's contents.  Each
//    call writes every scratch entry before reading it, so nothing has to be
//    cleared, but two calls whose kernels overlap on the GPU (different
//    streams, no ordering between them) race on the scratch.
//  * The cached address belongs to the device's current primary context:
//    calls must not cross a cudaDeviceReset of that device (after one, the
//    cached address would point into a context that no longer exists).
//  * A launch error that the caller left pending makes the call return
//    PSIPM_ERR_CUDA before it launches anything; the pending error is left in
//    place for the caller (it is read with cudaPeekAtLastError, not cleared).
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "psipm_b200.h"

namespace {

constexpr long long kStaticScratchMax = PSIPM_STATIC_SCRATCH_MAX;

// The scratch itself.  In host code this name is only a stand-in for the
// symbol, not a device address: kernels receive the address looked up below.
static __device__ __align__(256) double g_matvec_scratch[kStaticScratchMax];

std::mutex g_lock;
constexpr int kMaxDevices = 64;
double* g_scratch_addr[kMaxDevices] = {nullptr};

// t_j = w_j * sum_k A_kj v_k   (A^T in CSR, one thread per column)
__global__ void k_static_at(long long n, const int* __restrict__ at_ptr, const int* __restrict__ at_idx,
                            const double* __restrict__ at_val, const double* __restrict__ w,
                            const double* __restrict__ v, double* __restrict__ t) {
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n;
         j += (long long)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int k = at_ptr[j]; k < at_ptr[j + 1]; ++k) s += at_val[k] * v[at_idx[k]];
        t[j] = w[j] * s;
    }
}

// y_i = sum_j A_ij t_j + delta v_i   (A in CSR, one warp per row)
__global__ void k_static_a(long long m, const int* __restrict__ a_ptr, const int* __restrict__ a_idx,
                           const double* __restrict__ a_val, const double* __restrict__ t, double delta,
                           const double* __restrict__ v, double* __restrict__ y) {
    const int lane = threadIdx.x & 31;
    const long long warps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long i = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; i < m; i += warps) {
        double s = 0.0;
        for (int k = a_ptr[i] + lane; k < a_ptr[i + 1]; k += 32) s += a_val[k] * t[a_idx[k]];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) y[i] = s + delta * v[i];
    }
}

}  // namespace

extern "C" int psipm_normal_matvec_static(int64_t m, int64_t n, const int32_t* at_ptr, const int32_t* at_idx,
                                          const double* at_val, const int32_t* a_ptr, const int32_t* a_idx,
                                          const double* a_val, const double* w, double delta, const double* v,
                                          double* y, void* stream) {
    if (m <= 0 || n <= 0 || !at_ptr || !at_idx || !at_val || !a_ptr || !a_idx || !a_val || !w || !v || !y)
        return PSIPM_ERR_ARGUMENT;
    if (n > kStaticScratchMax) return PSIPM_ERR_ARGUMENT;  // scratch holds at most this many columns
    int device = -1;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices) return PSIPM_ERR_CUDA;
    double* scratch = nullptr;
    {
        std::lock_guard<std::mutex> guard(g_lock);
        if (!g_scratch_addr[device]) {
            void* addr = nullptr;
            if (cudaGetSymbolAddress(&addr, g_matvec_scratch) != cudaSuccess || !addr) return PSIPM_ERR_CUDA;
            g_scratch_addr[device] = static_cast<double*>(addr);
        }
        scratch = g_scratch_addr[device];
    }
    // an earlier, unrelated launch error of the caller: report it, keep it pending
    if (cudaPeekAtLastError() != cudaSuccess) return PSIPM_ERR_CUDA;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int threads = 256;
    const long long col_blocks = std::min<long long>((n + threads - 1) / threads, 65535);
    const long long row_blocks = std::min<long long>((m * 32 + threads - 1) / threads, 65535);
    k_static_at<<<(unsigned)col_blocks, threads, 0, s>>>(n, at_ptr, at_idx, at_val, w, v, scratch);
    k_static_a<<<(unsigned)row_blocks, threads, 0, s>>>(m, a_ptr, a_idx, a_val, scratch, delta, v, y);
    return cudaGetLastError() == cudaSuccess ? PSIPM_OK : PSIPM_ERR_CUDA;
}
