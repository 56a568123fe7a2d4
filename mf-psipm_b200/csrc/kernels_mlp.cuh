// Learned active-column selector: a 6 -> 64 -> 64 -> 2 perceptron scored per
// candidate column, with BF16 weights, FP32 biases and FP32 accumulation.
//
// Inputs per column (k_mlp_features): log theta_j, log nnz_j, log |a_j|_2,
// log mu, previous core membership, and the spectral rule's own log score
// (psipm_stable_preconditioner.py:293-309), so the network learns a
// correction to the rule rather than a rule of its own.  Outputs: [0] the
// column's score (a predicted leverage), [1] a per-column vote for the
// factor's first diagonal-shift index, averaged over the candidates.
//
// Parameter layout (kMlpParams floats, gradients in the same order):
//   W1[64][6], W2[64][64], W3[2][64]   (row-major, output x input)  BF16 in use
//   b1[64], b2[64], b3[2]                                            FP32
//
// Training (k_mlp_grad) runs tiles of kMlpTile samples per block: every thread
// takes one sample through the forward pass, keeps its activations and
// back-propagated errors in shared-memory tiles, then the block forms the
// tile's weight gradients as dot products over the tile's samples and adds
// them to per-thread register accumulators.  Each block writes one partial
// gradient; k_mlp_reduce adds the partials in block order, so a gradient is
// the same on every run.
#pragma once

#include <cuda_bf16.h>

#include "common.cuh"

namespace psipm {

constexpr int kMlpIn = 6;
constexpr int kMlpHid = 64;
constexpr int kMlpOut = 2;
constexpr int kMlpW1 = kMlpHid * kMlpIn;        // 384
constexpr int kMlpW2 = kMlpHid * kMlpHid;       // 4096
constexpr int kMlpW3 = kMlpOut * kMlpHid;       // 128
constexpr int kMlpWeights = kMlpW1 + kMlpW2 + kMlpW3;  // 4608 (BF16)
constexpr int kMlpBiases = kMlpHid + kMlpHid + kMlpOut;  // 130 (FP32)
constexpr int kMlpParams = kMlpWeights + kMlpBiases;     // 4738
constexpr int kMlpTile = 128;                  // samples per training tile (= threads)
constexpr int kMlpRow = kMlpHid + 1;           // padded shared-memory row (no bank conflicts)

struct MlpShared {  // weights as FP32 in shared memory
    float w1[kMlpW1], w2[kMlpW2], w3[kMlpW3], b1[kMlpHid], b2[kMlpHid], b3[kMlpOut];
};

__device__ __forceinline__ void mlp_stage(MlpShared& s, const __nv_bfloat16* __restrict__ w,
                                          const float* __restrict__ b) {
    for (int i = threadIdx.x; i < kMlpWeights; i += blockDim.x) {
        const float v = __bfloat162float(w[i]);
        if (i < kMlpW1)
            s.w1[i] = v;
        else if (i < kMlpW1 + kMlpW2)
            s.w2[i - kMlpW1] = v;
        else
            s.w3[i - kMlpW1 - kMlpW2] = v;
    }
    for (int i = threadIdx.x; i < kMlpBiases; i += blockDim.x) {
        const float v = b[i];
        if (i < kMlpHid)
            s.b1[i] = v;
        else if (i < 2 * kMlpHid)
            s.b2[i - kMlpHid] = v;
        else
            s.b3[i - 2 * kMlpHid] = v;
    }
    __syncthreads();
}

// first layer: h1 = relu(W1 x + b1)
__device__ __forceinline__ void mlp_layer1(const MlpShared& s, const float (&x)[kMlpIn], float (&h1)[kMlpHid]) {
#pragma unroll
    for (int o = 0; o < kMlpHid; ++o) {
        float a = s.b1[o];
#pragma unroll
        for (int k = 0; k < kMlpIn; ++k) a = fmaf(s.w1[o * kMlpIn + k], x[k], a);
        h1[o] = fmaxf(a, 0.0f);
    }
}

// second layer pre-activation of unit o
__device__ __forceinline__ float mlp_z2(const MlpShared& s, const float (&h1)[kMlpHid], int o) {
    float a = s.b2[o];
    const float4* row = reinterpret_cast<const float4*>(s.w2 + o * kMlpHid);
#pragma unroll
    for (int k = 0; k < kMlpHid / 4; ++k) {
        const float4 wv = row[k];
        a = fmaf(wv.x, h1[4 * k + 0], a);
        a = fmaf(wv.y, h1[4 * k + 1], a);
        a = fmaf(wv.z, h1[4 * k + 2], a);
        a = fmaf(wv.w, h1[4 * k + 3], a);
    }
    return a;
}

// Forward pass, one thread per sample (no grid-stride loop: a loop would let
// the compiler hoist the staged weights into registers and spill them):
// x (count x 6, row-major) -> out (count x 2)
__global__ void __launch_bounds__(256) k_mlp_forward(long long count, const float* __restrict__ x,
                                                     const __nv_bfloat16* __restrict__ w,
                                                     const float* __restrict__ b, float* __restrict__ out) {
    __shared__ __align__(16) MlpShared s;
    mlp_stage(s, w, b);
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < count) {
        float in[kMlpIn], h1[kMlpHid];
#pragma unroll
        for (int k = 0; k < kMlpIn; ++k) in[k] = x[i * kMlpIn + k];
        mlp_layer1(s, in, h1);
        float o0 = s.b3[0], o1 = s.b3[1];
#pragma unroll 1
        for (int o = 0; o < kMlpHid; ++o) {
            const float a = fmaxf(mlp_z2(s, h1, o), 0.0f);
            o0 = fmaf(s.w3[o], a, o0);
            o1 = fmaf(s.w3[kMlpHid + o], a, o1);
        }
        out[2 * i] = o0;
        out[2 * i + 1] = o1;
    }
}

struct MlpTiles {  // per-block training tiles (dynamic shared memory)
    float x[kMlpTile][kMlpIn];
    float h1[kMlpTile][kMlpRow];   // relu(z1)
    float a2[kMlpTile][kMlpRow];   // relu(z2)
    float d2[kMlpTile][kMlpRow];   // dL/dz2
    float d1[kMlpTile][kMlpRow];   // dL/dz1
    float d3[kMlpTile][kMlpOut];   // dL/dout
};
constexpr size_t kMlpGradSmem = sizeof(MlpShared) + sizeof(MlpTiles);
constexpr int kMlpPerThread = (kMlpParams + kMlpTile - 1) / kMlpTile;  // 38 accumulators

// Loss over the samples: sum_i c0 (out0_i - y0_i)^2 + c1 (out1_i - y1_i)^2, with
// per-sample targets y (count x 2); gradient of the loss w.r.t. every parameter
// (the BF16 weights as used) into part[block][kMlpParams], the block's loss
// into loss_part[block].
__global__ void __launch_bounds__(kMlpTile, 1)
    k_mlp_grad(long long count, const float* __restrict__ x, const float* __restrict__ y, float c0, float c1,
               const __nv_bfloat16* __restrict__ w, const float* __restrict__ b, float* __restrict__ part,
               float* __restrict__ loss_part) {
    extern __shared__ __align__(16) unsigned char mlp_smem[];
    MlpShared& s = *reinterpret_cast<MlpShared*>(mlp_smem);
    MlpTiles& T = *reinterpret_cast<MlpTiles*>(mlp_smem + sizeof(MlpShared));
    mlp_stage(s, w, b);
    const int t = threadIdx.x;
    float acc[kMlpPerThread];
#pragma unroll
    for (int q = 0; q < kMlpPerThread; ++q) acc[q] = 0.0f;
    float loss = 0.0f;
    const long long ntiles = (count + kMlpTile - 1) / kMlpTile;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const long long i = tile * kMlpTile + t;
        const bool live = i < count;
        // ---- forward + output error of this thread's sample ------------------
        float in[kMlpIn], h1[kMlpHid];
#pragma unroll
        for (int k = 0; k < kMlpIn; ++k) {
            in[k] = live ? x[i * kMlpIn + k] : 0.0f;
            T.x[t][k] = in[k];
        }
        mlp_layer1(s, in, h1);
#pragma unroll
        for (int o = 0; o < kMlpHid; ++o) T.h1[t][o] = h1[o];
        float o0 = s.b3[0], o1 = s.b3[1];
#pragma unroll 1
        for (int o = 0; o < kMlpHid; ++o) {
            const float z = mlp_z2(s, h1, o);
            const float a = fmaxf(z, 0.0f);
            T.a2[t][o] = a;
            T.d2[t][o] = z;  // pre-activation for now
            o0 = fmaf(s.w3[o], a, o0);
            o1 = fmaf(s.w3[kMlpHid + o], a, o1);
        }
        float e0 = 0.0f, e1 = 0.0f;
        if (live) {
            const float r0 = o0 - y[2 * i], r1 = o1 - y[2 * i + 1];
            loss += c0 * r0 * r0 + c1 * r1 * r1;
            e0 = 2.0f * c0 * r0;
            e1 = 2.0f * c1 * r1;
        }
        T.d3[t][0] = e0;
        T.d3[t][1] = e1;
        // dL/dz2 = W3^T e * [z2 > 0]
        for (int o = 0; o < kMlpHid; ++o) {
            const float z = T.d2[t][o];
            T.d2[t][o] = z > 0.0f ? fmaf(s.w3[o], e0, s.w3[kMlpHid + o] * e1) : 0.0f;
        }
        // dL/dz1 = W2^T d2 * [h1 > 0]
        for (int k = 0; k < kMlpHid; ++k) {
            float a = 0.0f;
#pragma unroll 8
            for (int o = 0; o < kMlpHid; ++o) a = fmaf(s.w2[o * kMlpHid + k], T.d2[t][o], a);
            T.d1[t][k] = T.h1[t][k] > 0.0f ? a : 0.0f;
        }
        __syncthreads();
        // ---- tile gradients: parameter p = t + kMlpTile q, a dot product over the tile
#pragma unroll
        for (int q = 0; q < kMlpPerThread; ++q) {
            const int p = t + kMlpTile * q;
            if (p >= kMlpParams) continue;
            float g = 0.0f;
            if (p < kMlpW1) {
                const int o = p / kMlpIn, k = p % kMlpIn;
                for (int r = 0; r < kMlpTile; ++r) g = fmaf(T.d1[r][o], T.x[r][k], g);
            } else if (p < kMlpW1 + kMlpW2) {
                const int o = (p - kMlpW1) / kMlpHid, k = (p - kMlpW1) % kMlpHid;
                for (int r = 0; r < kMlpTile; ++r) g = fmaf(T.d2[r][o], T.h1[r][k], g);
            } else if (p < kMlpWeights) {
                const int c = (p - kMlpW1 - kMlpW2) / kMlpHid, o = (p - kMlpW1 - kMlpW2) % kMlpHid;
                for (int r = 0; r < kMlpTile; ++r) g = fmaf(T.d3[r][c], T.a2[r][o], g);
            } else if (p < kMlpWeights + kMlpHid) {
                const int o = p - kMlpWeights;
                for (int r = 0; r < kMlpTile; ++r) g += T.d1[r][o];
            } else if (p < kMlpWeights + 2 * kMlpHid) {
                const int o = p - kMlpWeights - kMlpHid;
                for (int r = 0; r < kMlpTile; ++r) g += T.d2[r][o];
            } else {
                const int c = p - kMlpWeights - 2 * kMlpHid;
                for (int r = 0; r < kMlpTile; ++r) g += T.d3[r][c];
            }
            acc[q] += g;
        }
        __syncthreads();
    }
#pragma unroll
    for (int q = 0; q < kMlpPerThread; ++q) {
        const int p = t + kMlpTile * q;
        if (p < kMlpParams) part[(long long)blockIdx.x * kMlpParams + p] = acc[q];
    }
    // block loss in a fixed tree order
    __shared__ float lred[kMlpTile];
    lred[t] = loss;
    __syncthreads();
    for (int h = kMlpTile / 2; h > 0; h >>= 1) {
        if (t < h) lred[t] += lred[t + h];
        __syncthreads();
    }
    if (t == 0) loss_part[blockIdx.x] = lred[0];
}

// out[p] = scale * sum over blocks (in block order) of part[block][p]; same for the loss
__global__ void k_mlp_reduce(int blocks, const float* __restrict__ part, const float* __restrict__ loss_part,
                             float scale, float* __restrict__ grad, float* __restrict__ loss) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < kMlpParams) {
        float g = 0.0f;
        for (int k = 0; k < blocks; ++k) g += part[(long long)k * kMlpParams + p];
        grad[p] = scale * g;
    }
    if (p == 0) {
        float l = 0.0f;
        for (int k = 0; k < blocks; ++k) l += loss_part[k];
        *loss = scale * l;
    }
}

// Adam on the FP32 master parameters, then the BF16 weights and FP32 biases in use
__global__ void k_mlp_adam(float* __restrict__ master, float* __restrict__ m1, float* __restrict__ m2,
                           const float* __restrict__ grad, float lr, float beta1, float beta2, float eps,
                           float bc1, float bc2, float decay, __nv_bfloat16* __restrict__ w,
                           float* __restrict__ b) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kMlpParams) return;
    const float g = grad[p];
    const float a = beta1 * m1[p] + (1.0f - beta1) * g;
    const float v = beta2 * m2[p] + (1.0f - beta2) * g * g;
    m1[p] = a;
    m2[p] = v;
    float x = master[p];
    if (p < kMlpWeights) x -= lr * decay * x;  // decoupled weight decay on the weights only
    x -= lr * (a / bc1) / (sqrtf(v / bc2) + eps);
    master[p] = x;
    if (p < kMlpWeights)
        w[p] = __float2bfloat16_rn(x);
    else
        b[p - kMlpWeights] = x;
}

// ---- solver-side features of the candidates -------------------------------------
// feature row c (candidate j = cand[c]):
//   [0] log(theta_j) / 10     [1] log(nnz_j)      [2] log(|a_j|_2)
//   [3] log(max(mu, 1e-300)) / 10                 [4] 1 if j is in the current core
//   [5] log(max(score_c, 1e-300)) / 10            (the spectral rule's score)
__global__ void k_mlp_features(long long ncand, const long long* __restrict__ cand,
                               const int* __restrict__ at_ptr, const double* __restrict__ at_val,
                               const double* __restrict__ theta, const double* __restrict__ score,
                               const unsigned char* __restrict__ core_flags, double mu, float* __restrict__ x) {
    const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= ncand) return;
    const long long j = cand[c];
    const int b = at_ptr[j], e = at_ptr[j + 1];
    double sq = 0.0;
    for (int k = b; k < e; ++k) sq += at_val[k] * at_val[k];
    float* o = x + c * kMlpIn;
    o[0] = (float)(0.1 * log(theta[j]));
    o[1] = (float)log((double)(e - b));
    o[2] = (float)(0.5 * log(fmax(sq, 1e-300)));
    o[3] = (float)(0.1 * log(fmax(mu, 1e-300)));
    o[4] = core_flags ? (float)core_flags[c] : 0.0f;
    o[5] = (float)(0.1 * log(fmax(score[c], 1e-300)));
}

// scores (FP64, candidate order) = out[:, 0]; where allow (may be null) is 0: -inf
__global__ void k_mlp_take_scores(long long ncand, const float* __restrict__ out,
                                  const unsigned char* __restrict__ allow, double* __restrict__ score) {
    const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c < ncand) score[c] = (allow && !allow[c]) ? -INFINITY : (double)out[2 * c];
}

}  // namespace psipm
