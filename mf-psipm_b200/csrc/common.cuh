// Shared device/host helpers for libpsipm_b200.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "psipm_b200.h"

namespace psipm {

// An exception that carries one of the PSIPM_ERR_* status codes; the C ABI
// catches it at the boundary and returns the code.
struct Failure : std::runtime_error {
    int code;
    Failure(int c, const std::string& what) : std::runtime_error(what), code(c) {}
};

#define PSIPM_CUDA(call)                                                                   \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            throw ::psipm::Failure(PSIPM_ERR_CUDA, std::string(#call) + ": " +             \
                                                       cudaGetErrorString(e_));            \
    } while (0)

#define PSIPM_CHECK_LAUNCH() PSIPM_CUDA(cudaGetLastError())

// Device buffer owned by a handle (plain cudaMalloc; freed on destruction).
template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    // (Re)allocate to hold at least `count` elements; contents are not kept.
    void reserve(size_t count) {
        if (count <= n && p) return;
        release();
        if (count == 0) return;
        cudaError_t e = cudaMalloc(&p, count * sizeof(T));
        if (e != cudaSuccess) {
            p = nullptr;
            throw Failure(PSIPM_ERR_MEMORY, "cudaMalloc of " + std::to_string(count * sizeof(T)) +
                                                " bytes failed: " + cudaGetErrorString(e));
        }
        n = count;
    }
    // As reserve, but a buffer more than twice the size asked for (and above
    // 64 MB) is given back first: a smaller factor after a larger one does
    // not keep the larger one's memory.
    void fit(size_t count) {
        if (p && n > 2 * count && n * sizeof(T) > (size_t(64) << 20)) release();
        reserve(count);
    }
    void upload(const T* host, size_t count, cudaStream_t s) {
        reserve(count);
        if (count) PSIPM_CUDA(cudaMemcpyAsync(p, host, count * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    void upload(const std::vector<T>& v, cudaStream_t s) { upload(v.data(), v.size(), s); }
    void zero(size_t count, cudaStream_t s) {
        reserve(count);
        if (count) PSIPM_CUDA(cudaMemsetAsync(p, 0, count * sizeof(T), s));
    }
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Deterministic block sum (fixed tree); every thread receives the result.
// `scratch` must hold blockDim.x/32 doubles and is reused after a barrier.
__device__ __forceinline__ double block_sum(double v, double* scratch) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    double s = 0.0;
    if (warp == 0) {
        s = lane < nw ? scratch[lane] : 0.0;
        s = warp_sum(s);
        if (lane == 0) scratch[0] = s;
    }
    __syncthreads();
    s = scratch[0];
    __syncthreads();
    return s;
}

inline int ceil_div(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }

}  // namespace psipm
