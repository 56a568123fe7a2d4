// FP64 vector steps of the PS-IPM inner loop on device-resident vectors.
//
// They restate the O(n) NumPy arithmetic of the reference's prox_eval /
// psipm_solve (psipm_active_pool.py:1947-2271, 2559-2637) as fused passes:
//   P1  Theta, Newton right-hand side r1, dual directions dz/dw
//   P2  fraction-to-the-boundary step lengths (min-reductions), trial mu
//   P3  proximal residuals rd, rp, natural residual, outer KKT measures
// plus the Gondzio corrector targets and the iterate update with the box
// floors (psipm_active_pool.py:1845-1872).  Masks `pos` / `box` are uint8.
//
// Reductions: sums go through a block sum that each block writes to its own
// slot (slot k of a sum at part[k * kIpmPartStride + block]); k_ipm_fold adds
// the slots in block order, so every total is the same on every run.  Minima
// of nonnegative doubles use atomicMin on their bit patterns, which order like
// the values (exact in any order).
#pragma once

#include "common.cuh"

namespace psipm {

constexpr double kPosFloor = 8.0 * 2.220446049250313e-16;  // psipm_active_pool.py:61

constexpr int kIpmPartStride = 4096;  // >= the largest grid of the IPM kernels

__device__ __forceinline__ void block_add(double v, double* out, double* scratch) {
    v = block_sum(v, scratch);
    if (threadIdx.x == 0) out[blockIdx.x] = v;
}

// red[k] = sum over b < kIpmPartStride of part[k * kIpmPartStride + b], in order
__global__ void k_ipm_fold(int nred, const double* __restrict__ part, double* __restrict__ red) {
    const int k = threadIdx.x;
    if (k >= nred) return;
    double s = 0.0;
    for (int b = 0; b < kIpmPartStride; ++b) s += part[(long long)k * kIpmPartStride + b];
    red[k] = s;
}

// minimum of nonnegative values through their (monotone) bit patterns
__device__ __forceinline__ void block_min_nonneg(double v, unsigned long long* out) {
    unsigned long long b = (unsigned long long)__double_as_longlong(v);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long c = __shfl_xor_sync(0xffffffffu, b, o);
        b = c < b ? c : b;
    }
    if ((threadIdx.x & 31) == 0) atomicMin(out, b);
}

// max that keeps a NaN (whose bit pattern orders above +inf)
__device__ __forceinline__ double nan_max(double a, double b) { return (b > a || b != b) ? b : a; }

__device__ __forceinline__ void box_floors(double u, double& xf, double& sf) {
    const double q = 0.25 * u;
    xf = fmin(kPosFloor, q);
    sf = fmin(kPosFloor * fmax(1.0, u), q);
}

// theta = theta_min + pos z/x + box w/s, non-finite -> cap, clipped to [theta_min, cap]
__global__ void k_ipm_theta(long long n, const double* __restrict__ x, const double* __restrict__ z,
                            const double* __restrict__ w, const double* __restrict__ s,
                            const unsigned char* __restrict__ pos, const unsigned char* __restrict__ box,
                            double tmin, double cap, double* __restrict__ theta) {
    long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j >= n) return;
    double t = tmin;
    if (pos[j]) t += z[j] / x[j];
    if (box[j]) t += w[j] / s[j];
    if (!isfinite(t)) t = cap;
    theta[j] = fmin(fmax(t, tmin), cap);
}

// r1 = rd + pos rmz/x - box rmw/s
__global__ void k_ipm_r1(long long n, const double* __restrict__ rd, const double* __restrict__ rmz,
                         const double* __restrict__ rmw, const double* __restrict__ x,
                         const double* __restrict__ s, const unsigned char* __restrict__ pos,
                         const unsigned char* __restrict__ box, double* __restrict__ r1) {
    long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j >= n) return;
    double v = rd ? rd[j] : 0.0;
    if (pos[j]) v += rmz[j] / x[j];
    if (box[j]) v -= rmw[j] / s[j];
    r1[j] = v;
}

// dz = pos (rmz - z dx)/x ; dw = box (rmw + w dx)/s; flag = 1 if dx, dy, dz or dw holds a
// non-finite entry (the grid covers max(n, m))
__global__ void k_ipm_dual_dirs(long long n, long long m, const double* __restrict__ rmz,
                                const double* __restrict__ rmw, const double* __restrict__ x,
                                const double* __restrict__ z, const double* __restrict__ w,
                                const double* __restrict__ s, const double* __restrict__ dx,
                                const double* __restrict__ dy, const unsigned char* __restrict__ pos,
                                const unsigned char* __restrict__ box, double* __restrict__ dz,
                                double* __restrict__ dw, int* __restrict__ flag) {
    long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    bool bad = false;
    if (j < n) {
        const double d = dx[j];
        const double a = pos[j] ? (rmz[j] - z[j] * d) / x[j] : 0.0;
        const double b = box[j] ? (rmw[j] + w[j] * d) / s[j] : 0.0;
        dz[j] = a;
        dw[j] = b;
        bad = !(isfinite(d) && isfinite(a) && isfinite(b));
    }
    if (j < m) bad = bad || !isfinite(dy[j]);
    if (bad) atomicExch(flag, 1);
}

// step lengths for d = d0 + gamma d1 (d1 may be null):
//   out[0] = min(1, min_{pos, dx<0} -x/dx, min_{box, ds<0} -s/ds)   ds = -dx
//   out[1] = min(1, min_{pos, dz<0} -z/dz, min_{box, dw<0} -w/dw)
__global__ void k_ipm_steps(long long n, const double* __restrict__ x, const double* __restrict__ s,
                            const double* __restrict__ z, const double* __restrict__ w,
                            const double* __restrict__ dx, const double* __restrict__ dz,
                            const double* __restrict__ dw, const double* __restrict__ dxc,
                            const double* __restrict__ dzc, const double* __restrict__ dwc, double gamma,
                            const unsigned char* __restrict__ pos, const unsigned char* __restrict__ box,
                            unsigned long long* __restrict__ out) {
    double ap = 1.0, ad = 1.0;
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n;
         j += (long long)gridDim.x * blockDim.x) {
        const double ddx = dx[j] + (dxc ? gamma * dxc[j] : 0.0);
        if (pos[j]) {
            const double ddz = dz[j] + (dzc ? gamma * dzc[j] : 0.0);
            if (ddx < 0.0) ap = fmin(ap, -x[j] / ddx);
            if (ddz < 0.0) ad = fmin(ad, -z[j] / ddz);
        }
        if (box[j]) {
            const double dds = -ddx;
            const double ddw = dw[j] + (dwc ? gamma * dwc[j] : 0.0);
            if (dds < 0.0) ap = fmin(ap, -s[j] / dds);
            if (ddw < 0.0) ad = fmin(ad, -w[j] / ddw);
        }
    }
    block_min_nonneg(ap > 0.0 ? ap : 0.0, out);  // +0 for a zero or negative step
    block_min_nonneg(ad > 0.0 ? ad : 0.0, out + 1);
}

// sum_pos (x + ax dx)(z + az dz) + sum_box (s - ax dx)(w + az dw), d = d0 + gamma d1
__global__ void k_ipm_comp(long long n, const double* __restrict__ x, const double* __restrict__ s,
                           const double* __restrict__ z, const double* __restrict__ w,
                           const double* __restrict__ dx, const double* __restrict__ dz,
                           const double* __restrict__ dw, const double* __restrict__ dxc,
                           const double* __restrict__ dzc, const double* __restrict__ dwc, double gamma,
                           double ax, double az, const unsigned char* __restrict__ pos,
                           const unsigned char* __restrict__ box, double* __restrict__ out) {
    __shared__ double scratch[32];
    double acc = 0.0;
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n;
         j += (long long)gridDim.x * blockDim.x) {
        const double ddx = dx ? dx[j] + (dxc ? gamma * dxc[j] : 0.0) : 0.0;
        if (pos[j]) {
            const double ddz = dz ? dz[j] + (dzc ? gamma * dzc[j] : 0.0) : 0.0;
            acc += (x[j] + ax * ddx) * (z[j] + az * ddz);
        }
        if (box[j]) {
            const double ddw = dw ? dw[j] + (dwc ? gamma * dwc[j] : 0.0) : 0.0;
            acc += (s[j] - ax * ddx) * (w[j] + az * ddw);
        }
    }
    block_add(acc, out, scratch);
}

// predictor / plain targets: rmz = pos (-x z + c0), rmw = box (-s w + c0)
__global__ void k_ipm_targets(long long n, const double* __restrict__ x, const double* __restrict__ s,
                              const double* __restrict__ z, const double* __restrict__ w, double c0,
                              const unsigned char* __restrict__ pos, const unsigned char* __restrict__ box,
                              double* __restrict__ rmz, double* __restrict__ rmw) {
    long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j >= n) return;
    rmz[j] = pos[j] ? -x[j] * z[j] + c0 : 0.0;
    rmw[j] = box[j] ? -s[j] * w[j] + c0 : 0.0;
}

// Mehrotra corrector targets (psipm_active_pool.py:2113-2114):
// rmz = pos (mu_t - dx dz), rmw = box (mu_t - ds dw) with ds = -dx
__global__ void k_ipm_mehrotra(long long n, const double* __restrict__ dx, const double* __restrict__ dz,
                               const double* __restrict__ dw, double mu_t, const unsigned char* __restrict__ pos,
                               const unsigned char* __restrict__ box, double* __restrict__ rmz,
                               double* __restrict__ rmw) {
    long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j >= n) return;
    rmz[j] = pos[j] ? mu_t - dx[j] * dz[j] : 0.0;
    rmw[j] = box[j] ? mu_t - (-dx[j]) * dw[j] : 0.0;
}

// Gondzio corrector targets (psipm_active_pool.py:2180-2197)
__global__ void k_ipm_gondzio(long long n, const double* __restrict__ x, const double* __restrict__ s,
                              const double* __restrict__ z, const double* __restrict__ w,
                              const double* __restrict__ dx, const double* __restrict__ dz,
                              const double* __restrict__ dw, double ta_x, double ta_z, double mu_t,
                              double bmin, double bmax, const unsigned char* __restrict__ pos,
                              const unsigned char* __restrict__ box, double* __restrict__ rmz,
                              double* __restrict__ rmw) {
    long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j >= n) return;
    const double lo = bmin * mu_t, hi = bmax * mu_t;
    if (pos[j]) {
        const double prod = (x[j] + ta_x * dx[j]) * (z[j] + ta_z * dz[j]);
        double corr = fmin(fmax(prod, lo), hi) - prod;
        rmz[j] = fmin(fmax(corr, -hi), 2.0 * hi);
    }
    if (box[j]) {
        const double prod = (s[j] - ta_x * dx[j]) * (w[j] + ta_z * dw[j]);
        double corr = fmin(fmax(prod, lo), hi) - prod;
        rmw[j] = fmin(fmax(corr, -hi), 2.0 * hi);
    }
}

// d += gamma dc for the four directions (dy has m entries)
__global__ void k_ipm_accept(long long n, long long m, double* __restrict__ dx, double* __restrict__ dy,
                             double* __restrict__ dz, double* __restrict__ dw, const double* __restrict__ dxc,
                             const double* __restrict__ dyc, const double* __restrict__ dzc,
                             const double* __restrict__ dwc, double gamma) {
    long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j < n) {
        dx[j] += gamma * dxc[j];
        dz[j] += gamma * dzc[j];
        dw[j] += gamma * dwc[j];
    }
    if (j < m) dy[j] += gamma * dyc[j];
}

// x += ax dx, z += az dz, w += az dw (n); y += az dy (m); then the box floors:
// x = clip(x, x_floor, u - s_floor), s = max(u - x, s_floor) on box
__global__ void k_ipm_update(long long n, long long m, double* __restrict__ x, double* __restrict__ y,
                             double* __restrict__ z, double* __restrict__ w, double* __restrict__ s,
                             const double* __restrict__ u, const unsigned char* __restrict__ box,
                             const double* __restrict__ dx, const double* __restrict__ dy,
                             const double* __restrict__ dz, const double* __restrict__ dw, double ax, double az) {
    long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j < n) {
        double xj = x[j] + ax * dx[j];
        z[j] += az * dz[j];
        w[j] += az * dw[j];
        if (box[j]) {
            double xf, sf;
            box_floors(u[j], xf, sf);
            xj = fmin(fmax(xj, xf), u[j] - sf);
            s[j] = fmax(u[j] - xj, sf);
        }
        x[j] = xj;
    }
    if (j < m) y[j] += az * dy[j];
}

// box floors only (s from x), for a fresh iterate
__global__ void k_ipm_sync_box(long long n, double* __restrict__ x, double* __restrict__ s,
                               const double* __restrict__ u, const unsigned char* __restrict__ box) {
    long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j >= n) return;
    if (box[j]) {
        double xf, sf;
        box_floors(u[j], xf, sf);
        const double xj = fmin(fmax(x[j], xf), u[j] - sf);
        x[j] = xj;
        s[j] = fmax(u[j] - xj, sf);
    } else {
        s[j] = 1.0;
    }
}

// proximal residuals (psipm_active_pool.py:1984-1993), given aty = A'y and ax = A x:
//   rd = -(c - aty - z + w + rho (x - xk)),  rp = -(ax - b + delta (y - yk))
//   g = c - aty + rho (x - xk);  gp = pos ? x - clip(x - g, 0, u) : g
// out[0] += |gp|^2, out[1] += |rp|^2, out[2] += |rd|^2, out[3] += |x - xk|^2, out[4] += |y - yk|^2
__global__ void k_ipm_residual_n(long long n, const double* __restrict__ c, const double* __restrict__ aty,
                                 const double* __restrict__ x, const double* __restrict__ z,
                                 const double* __restrict__ w, const double* __restrict__ xk,
                                 const double* __restrict__ u, const unsigned char* __restrict__ pos,
                                 double rho, double* __restrict__ rd, double* __restrict__ out) {
    __shared__ double scratch[32];
    double a0 = 0.0, a2 = 0.0, a3 = 0.0;
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n;
         j += (long long)gridDim.x * blockDim.x) {
        const double dxk = x[j] - xk[j];
        const double g = c[j] - aty[j] + rho * dxk;
        const double r = -(c[j] - aty[j] - z[j] + w[j] + rho * dxk);
        rd[j] = r;
        const double gp = pos[j] ? x[j] - fmin(fmax(x[j] - g, 0.0), u[j]) : g;
        a0 += gp * gp;
        a2 += r * r;
        a3 += dxk * dxk;
    }
    block_add(a0, out + 0 * kIpmPartStride, scratch);
    block_add(a2, out + 2 * kIpmPartStride, scratch);
    block_add(a3, out + 3 * kIpmPartStride, scratch);
}

__global__ void k_ipm_residual_m(long long m, const double* __restrict__ ax, const double* __restrict__ b,
                                 const double* __restrict__ y, const double* __restrict__ yk, double delta,
                                 double* __restrict__ rp, double* __restrict__ out) {
    __shared__ double scratch[32];
    double a1 = 0.0, a4 = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m;
         i += (long long)gridDim.x * blockDim.x) {
        const double dyk = y[i] - yk[i];
        const double r = -(ax[i] - b[i] + delta * dyk);
        rp[i] = r;
        a1 += r * r;
        a4 += dyk * dyk;
    }
    block_add(a1, out + 1 * kIpmPartStride, scratch);
    block_add(a4, out + 4 * kIpmPartStride, scratch);
}

// outer KKT measures (psipm_active_pool.py:2561-2599), given aty and ax:
//   out_max[0] = max |b - ax|,  out_max[1] = max |c - aty - z + w|   (as bit patterns)
//   out[0] = c.x, out[1] = b.y, out[2] = sum_box w u, out[3] = sum_pos x z + sum_box s w
__global__ void k_ipm_outer_n(long long n, const double* __restrict__ c, const double* __restrict__ aty,
                              const double* __restrict__ x, const double* __restrict__ z,
                              const double* __restrict__ w, const double* __restrict__ s,
                              const double* __restrict__ u, const unsigned char* __restrict__ pos,
                              const unsigned char* __restrict__ box, double* __restrict__ out,
                              unsigned long long* __restrict__ out_max) {
    __shared__ double scratch[32];
    double cx = 0.0, wu = 0.0, comp = 0.0, rdmax = 0.0;
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n;
         j += (long long)gridDim.x * blockDim.x) {
        cx += c[j] * x[j];
        const double rd = c[j] - aty[j] - z[j] + w[j];
        rdmax = nan_max(rdmax, fabs(rd));
        if (pos[j]) comp += x[j] * z[j];
        if (box[j]) {
            wu += w[j] * u[j];
            comp += s[j] * w[j];
        }
    }
    block_add(cx, out + 0 * kIpmPartStride, scratch);
    block_add(wu, out + 2 * kIpmPartStride, scratch);
    block_add(comp, out + 3 * kIpmPartStride, scratch);
    unsigned long long bm = (unsigned long long)__double_as_longlong(rdmax);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long cnd = __shfl_xor_sync(0xffffffffu, bm, o);
        bm = cnd > bm ? cnd : bm;
    }
    if ((threadIdx.x & 31) == 0) atomicMax(out_max + 1, bm);
}

__global__ void k_ipm_outer_m(long long m, const double* __restrict__ ax, const double* __restrict__ b,
                              const double* __restrict__ y, double* __restrict__ out,
                              unsigned long long* __restrict__ out_max) {
    __shared__ double scratch[32];
    double by = 0.0, rpmax = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m;
         i += (long long)gridDim.x * blockDim.x) {
        by += b[i] * y[i];
        rpmax = nan_max(rpmax, fabs(b[i] - ax[i]));
    }
    block_add(by, out + 1 * kIpmPartStride, scratch);
    unsigned long long bm = (unsigned long long)__double_as_longlong(rpmax);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long cnd = __shfl_xor_sync(0xffffffffu, bm, o);
        bm = cnd > bm ? cnd : bm;
    }
    if ((threadIdx.x & 31) == 0) atomicMax(out_max, bm);
}

// y = M v for CSR M (A^T with n rows, or A with m rows), W lanes per row.
// Each warp takes 32/W consecutive rows per trip; the trip base is uniform
// across the warp so every lane reaches the shuffles.
template <int W>
__global__ void k_spmv_rows(long long rows, const int* __restrict__ ptr, const int* __restrict__ idx,
                            const double* __restrict__ val, const double* __restrict__ v,
                            double* __restrict__ y) {
    constexpr int kRowsPerWarp = 32 / W;
    const int lane = threadIdx.x & (W - 1);
    const int sub = (threadIdx.x & 31) / W;
    const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long base = warp * kRowsPerWarp; base < rows; base += nwarps * kRowsPerWarp) {
        const long long i = base + sub;
        double acc = 0.0;
        if (i < rows)
            for (int k = ptr[i] + lane; k < ptr[i + 1]; k += W) acc += val[k] * v[idx[k]];
#pragma unroll
        for (int o = W / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o, W);
        if (lane == 0 && i < rows) y[i] = acc;
    }
}

// reduction scratch: red[0..nred) = 0, redu[0..nu) = uval, *flag = 0
__global__ void k_ipm_reset(double* __restrict__ red, int nred, unsigned long long* __restrict__ redu, int nu,
                            unsigned long long uval, int* __restrict__ flag) {
    const int t = threadIdx.x;
    if (t < nred) red[t] = 0.0;
    if (t < nu) redu[t] = uval;
    if (t == 0 && flag) *flag = 0;
}

// centre <-> iterate copies of (x, z, w) on n and y on m
__global__ void k_ipm_copy(long long n, long long m, const double* __restrict__ x, const double* __restrict__ y,
                           const double* __restrict__ z, const double* __restrict__ w, double* __restrict__ xo,
                           double* __restrict__ yo, double* __restrict__ zo, double* __restrict__ wo) {
    long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j < n) {
        xo[j] = x[j];
        zo[j] = z[j];
        wo[j] = w[j];
    }
    if (j < m) yo[j] = y[j];
}

// lag bound (psipm_spectral_preconditioner.py:396-410): ratio = w / max(w_ref, tiny);
// out[0] = max ratio, out[1] = min ratio (bit patterns), flag = 1 if a ratio is not finite or <= 0
__global__ void k_lag_ratio(long long n, const double* __restrict__ w, const double* __restrict__ wref,
                            unsigned long long* __restrict__ out, int* __restrict__ flag) {
    double mx = 0.0, mn = 1.0e308;
    int bad = 0;
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n;
         j += (long long)gridDim.x * blockDim.x) {
        const double r = w[j] / fmax(wref[j], 2.2250738585072014e-308);
        if (!(isfinite(r) && r > 0.0)) {
            bad = 1;
            continue;
        }
        mx = fmax(mx, r);
        mn = fmin(mn, r);
    }
    unsigned long long bmx = (unsigned long long)__double_as_longlong(mx);
    unsigned long long bmn = (unsigned long long)__double_as_longlong(mn);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long a = __shfl_xor_sync(0xffffffffu, bmx, o);
        unsigned long long b = __shfl_xor_sync(0xffffffffu, bmn, o);
        bmx = a > bmx ? a : bmx;
        bmn = b < bmn ? b : bmn;
        bad |= __shfl_xor_sync(0xffffffffu, bad, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(out, bmx);
        atomicMin(out + 1, bmn);
        if (bad) atomicExch(flag, 1);
    }
}

}  // namespace psipm

namespace psipm {

// ---- starting point (psipm_active_pool.py:4122-4304, legacy projection) -------
// Each kernel writes kStartSlots partial results per block into
// part[slot * gridDim.x + block]; the host folds them in block order, so the
// starting point is the same on every run.
constexpr int kStartSlots = 6;

__device__ __forceinline__ void start_partial_sum(double v, int slot, double* part, double* scratch) {
    v = block_sum(v, scratch);
    if (threadIdx.x == 0) part[slot * gridDim.x + blockIdx.x] = v;
}
__device__ __forceinline__ double block_max(double v, double* scratch) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    __syncthreads();
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    double s = 0.0;
    if (warp == 0) {
        s = lane < nw ? scratch[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s = fmax(s, __shfl_xor_sync(0xffffffffu, s, o));
        if (lane == 0) scratch[0] = s;
    }
    __syncthreads();
    s = scratch[0];
    __syncthreads();
    return s;
}
__device__ __forceinline__ void start_partial_max(double v, int slot, double* part, double* scratch) {
    v = block_max(v, scratch);
    if (threadIdx.x == 0) part[slot * gridDim.x + blockIdx.x] = v;
}

// *flag = 1 if dx (n) or dy (m) holds a non-finite entry
__global__ void k_start_finite(long long n, long long m, const double* __restrict__ dx,
                               const double* __restrict__ dy, int* __restrict__ flag) {
    long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    bool bad = false;
    if (j < n) bad = !isfinite(dx[j]);
    if (j < m) bad = bad || !isfinite(dy[j]);
    if (bad) atomicExch(flag, 1);
}

// x, y from the two projections: part slot 0 = 1 if x holds a non-finite entry,
// slot 3 = 1 if y does; then xl = pos ? x : 0, xu = box ? u - x : 0 and the
// infeasibilities slot 1 = max(0, max_pos -xl), slot 2 = max(0, max_box -xu)   (:4135-4160)
__global__ void k_start_bounds(long long n, long long m, const double* __restrict__ x, const double* __restrict__ y,
                               const double* __restrict__ u, const unsigned char* __restrict__ pos,
                               const unsigned char* __restrict__ box, double* __restrict__ xl,
                               double* __restrict__ xu, double* __restrict__ part) {
    __shared__ double scratch[32];
    double bad = 0.0, ybad = 0.0, il = 0.0, iu = 0.0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n || j < m; j += stride) {
        if (j < m && !isfinite(y[j])) ybad = 1.0;
        if (j >= n) continue;
        const double xj = x[j];
        if (!isfinite(xj)) bad = 1.0;
        const double l = pos[j] ? xj : 0.0;
        const double r = box[j] ? u[j] - xj : 0.0;
        xl[j] = l;
        xu[j] = r;
        if (pos[j]) il = fmax(il, -l);
        if (box[j]) iu = fmax(iu, -r);
    }
    start_partial_max(bad, 0, part, scratch);
    start_partial_max(il, 1, part, scratch);
    start_partial_max(iu, 2, part, scratch);
    start_partial_max(ybad, 3, part, scratch);
}

// zero x and/or y when they held a non-finite entry (the reference's fallback)
__global__ void k_start_zero(long long n, double* __restrict__ v) {
    long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j < n) v[j] = 0.0;
}

// r = c - A^T y (aty given): slot 0 = |c|^2, slot 1 = |r|^2
__global__ void k_start_dual_norms(long long n, const double* __restrict__ c, const double* __restrict__ aty,
                                   double* __restrict__ r, double* __restrict__ part) {
    __shared__ double scratch[32];
    double cc = 0.0, rr = 0.0;
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n;
         j += (long long)gridDim.x * blockDim.x) {
        const double rj = c[j] - aty[j];
        r[j] = rj;
        cc += c[j] * c[j];
        rr += rj * rj;
    }
    start_partial_sum(cc, 0, part, scratch);
    start_partial_sum(rr, 1, part, scratch);
}

__global__ void k_start_scale(long long m, double a, double* __restrict__ y) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < m) y[i] *= a;
}

// xl += xshift1 (pos), xu += xshift1 (box); dual slacks from r (:4166-4199):
// c = 0: z = 1 on pos, w = 1 on box; else z = r on lower-only, z = r/2 and
// w = -r/2 on box; slot 0 = max(0, max_pos -z), slot 1 = max(0, max_box -w)
__global__ void k_start_slacks(long long n, const double* __restrict__ r, double xshift1, int c_zero,
                               const unsigned char* __restrict__ pos, const unsigned char* __restrict__ box,
                               double* __restrict__ xl, double* __restrict__ xu, double* __restrict__ z,
                               double* __restrict__ w, double* __restrict__ part) {
    __shared__ double scratch[32];
    double iz = 0.0, iw = 0.0;
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n;
         j += (long long)gridDim.x * blockDim.x) {
        const bool p = pos[j], b = box[j];
        if (p) xl[j] += xshift1;
        if (b) xu[j] += xshift1;
        double zj = 0.0, wj = 0.0;
        if (c_zero) {
            zj = p ? 1.0 : 0.0;
            wj = b ? 1.0 : 0.0;
        } else {
            if (p && !b) zj = r[j];
            if (b) {
                zj = 0.5 * r[j];
                wj = -0.5 * r[j];
            }
            if (p) iz = fmax(iz, -zj);
            if (b) iw = fmax(iw, -wj);
        }
        z[j] = zj;
        w[j] = wj;
    }
    start_partial_max(iz, 0, part, scratch);
    start_partial_max(iw, 1, part, scratch);
}

// z += zshift1 (pos), w += zshift1 (box) when c != 0, then the sums of :4200-4215:
// slots 0..5 = sum_pos xl, sum_box xu, sum_pos z, sum_box w, sum_pos xl z, sum_box xu w
__global__ void k_start_sums(long long n, double zshift1, const unsigned char* __restrict__ pos,
                             const unsigned char* __restrict__ box, const double* __restrict__ xl,
                             const double* __restrict__ xu, double* __restrict__ z, double* __restrict__ w,
                             double* __restrict__ part) {
    __shared__ double scratch[32];
    double a[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n;
         j += (long long)gridDim.x * blockDim.x) {
        if (pos[j]) {
            const double zj = z[j] + zshift1;
            z[j] = zj;
            a[0] += xl[j];
            a[2] += zj;
            a[4] += xl[j] * zj;
        }
        if (box[j]) {
            const double wj = w[j] + zshift1;
            w[j] = wj;
            a[1] += xu[j];
            a[3] += wj;
            a[5] += xu[j] * wj;
        }
    }
#pragma unroll
    for (int k = 0; k < 6; ++k) start_partial_sum(a[k], k, part, scratch);
}

// final shifts and the primal point (:4216-4240): xl, xu += xshift2; z, w += zshift2;
// x = max(xl, 1e-12) on lower-only columns; x = clip(u xl / (xl + xu), floors) on box
__global__ void k_start_final(long long n, double xshift2, double zshift2, const double* __restrict__ u,
                              const unsigned char* __restrict__ pos, const unsigned char* __restrict__ box,
                              double* __restrict__ xl, double* __restrict__ xu, double* __restrict__ x,
                              double* __restrict__ z, double* __restrict__ w) {
    long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j >= n) return;
    const bool p = pos[j], b = box[j];
    double l = xl[j], r = xu[j];
    if (p) l += xshift2;
    if (b) r += xshift2;
    if (p) z[j] += zshift2;
    if (b) w[j] += zshift2;
    if (p && !b) x[j] = fmax(l, 1e-12);
    if (b) {
        const double d = l + r;
        const double xb = d > 0.0 ? u[j] * l / d : 0.5 * u[j];
        double xf, sf;
        box_floors(u[j], xf, sf);
        x[j] = fmin(fmax(xb, xf), u[j] - sf);
    }
}

}  // namespace psipm
