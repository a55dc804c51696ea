// Krylov-vector kernels for the device GMRES (K6): batched inner products with a fixed-order
// in-kernel final reduction, Gram-Schmidt updates and basis combinations. Every kernel takes
// the right-hand-side index from blockIdx.y so all RHS of a multi-RHS solve share launches.
//
// Basis layout: V[k][r][i] (k = Krylov index, r = RHS, i = element), i.e. each Krylov column
// V[k] is one contiguous [nrhs][n] block, the layout the matvec kernels take as x.
#pragma once

#include <cuda_runtime.h>

namespace kemcu
{

constexpr int kDotThreads = 256;
constexpr int kDotBlocks = 64;  // chunks per vector; partials are summed by the last block

__device__ __forceinline__ double block_sum(double v, double* sh)
{
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0)
        sh[w] = v;
    __syncthreads();
    v = 0.;
    if (threadIdx.x < (blockDim.x >> 5))
        v = sh[threadIdx.x];
    if (w == 0)
        for (int o = 16; o > 0; o >>= 1)
            v += __shfl_down_sync(0xffffffffu, v, o);
    return v;  // valid in thread 0
}

// h[r][k0 + k] = sum_i V[k0 + k][r][i] * w[r][i] for k < nk (nk <= 64 per launch); h row stride hs.
// grid (kDotBlocks, nrhs); partial[r][k][blk]; counter[r] must start at 0 and is reset.
// A CTA covers one slice of the rows i. Its 8 warps take the basis vectors in groups of 8: with
// G = ceil(nk / 8) groups, 8 / G warps share a group and stride over the rows, each lane keeping
// 8 running sums (one w load serves 8 basis entries); warp shuffles then reduce the lanes,
// shared memory the warps of a group, and the last CTA of a right-hand side sums the slices in
// block order, so the result does not depend on scheduling.
__global__ void __launch_bounds__(kDotThreads, 4) multi_dot_kernel(const double* __restrict__ V, const double* __restrict__ w,
                                                                int n, int nrhs, int k0, int nk, double* __restrict__ partial,
                                                                unsigned* __restrict__ counter, double* __restrict__ h, int hs)
{
    static_assert(kDotThreads == 256, "8 warps of 8 basis vectors cover the 64 vectors of a launch");
    __shared__ double s_red[8][8];
    __shared__ double s_part[64 * (kDotBlocks + 1)];  // the last CTA's copy of the slices' sums
    __shared__ bool last;
    const int r = blockIdx.y;
    const int per = (n + gridDim.x - 1) / gridDim.x;
    const int i0 = blockIdx.x * per, i1 = min(n, i0 + per);
    const double* wr = w + (size_t) r * n;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int groups = (nk + 7) >> 3;
    const int wpg = max(1, 8 / groups);  // warps per group of 8 basis vectors
    const int grp = warp / wpg, slice = warp % wpg;
    double acc[8];
#pragma unroll
    for (int q = 0; q < 8; q++)
        acc[q] = 0.;
    if (grp < groups) {
        const int kb = 8 * grp, kn = min(8, nk - kb);
        const size_t vstride = (size_t) nrhs * n;
        const double* vb = V + ((size_t) (k0 + kb) * nrhs + r) * n;
        const int step = 32 * wpg;
        int i = i0 + 32 * slice + lane;
        // two rows per pass: the 18 loads are all issued before the FMAs, which keep the
        // one-row-at-a-time order of each lane's sums
        for (; i + step < i1; i += 2 * step) {
            const double wa = wr[i], wb = wr[i + step];
            double va[8], vc[8];
#pragma unroll
            for (int q = 0; q < 8; q++)
                if (q < kn) {
                    va[q] = vb[q * vstride + i];
                    vc[q] = vb[q * vstride + i + step];
                }
#pragma unroll
            for (int q = 0; q < 8; q++)
                if (q < kn)
                    acc[q] = fma(va[q], wa, acc[q]);
#pragma unroll
            for (int q = 0; q < 8; q++)
                if (q < kn)
                    acc[q] = fma(vc[q], wb, acc[q]);
        }
        if (i < i1) {
            const double wi = wr[i];
#pragma unroll
            for (int q = 0; q < 8; q++)
                if (q < kn)
                    acc[q] = fma(vb[q * vstride + i], wi, acc[q]);
        }
    }
#pragma unroll
    for (int q = 0; q < 8; q++) {
        double v = acc[q];
        for (int o = 16; o > 0; o >>= 1)
            v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0)
            s_red[warp][q] = v;
    }
    __syncthreads();
    if (threadIdx.x < 64) {
        const int g2 = threadIdx.x >> 3, q = threadIdx.x & 7;
        if (g2 < groups && 8 * g2 + q < nk) {
            double v = 0.;
            for (int sl = 0; sl < wpg; sl++)
                v += s_red[g2 * wpg + sl][q];
            partial[((size_t) r * 64 + 8 * g2 + q) * gridDim.x + blockIdx.x] = v;
        }
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0)
        last = atomicAdd(counter + r, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last)
        return;
    __threadfence();
    const int nb = (int) gridDim.x;
    const double* pr = partial + (size_t) r * 64 * nb;  // partial[r][k][b] for k < nk is contiguous
    if (nb <= kDotBlocks) {
        // the slices' sums go to shared memory with parallel loads (rows padded by one against
        // bank conflicts); each thread then sums its k in block order as below
        for (int t = threadIdx.x; t < nk * nb; t += blockDim.x)
            s_part[(t / nb) * (nb + 1) + t % nb] = __ldcg(pr + t);
        __syncthreads();
        for (int k = threadIdx.x; k < nk; k += blockDim.x) {
            double s = 0.;
            for (int b = 0; b < nb; b++)
                s += s_part[k * (nb + 1) + b];
            h[(size_t) r * hs + k0 + k] = s;
        }
    }
    else
        for (int k = threadIdx.x; k < nk; k += blockDim.x) {
            double s = 0.;
            for (int b = 0; b < nb; b++)
                s += __ldcg(pr + (size_t) k * nb + b);
            h[(size_t) r * hs + k0 + k] = s;
        }
    if (threadIdx.x == 0)
        counter[r] = 0u;
}

// w[r][i] -= sum_{k < nk} h[r][k0 + k] V[k0 + k][r][i];   grid (ceil(n/256), nrhs)
__global__ void gs_update_kernel(const double* __restrict__ V, double* __restrict__ w, int n, int nrhs, int k0, int nk,
                                 const double* __restrict__ h, int hs, const int* __restrict__ active)
{
    const int r = blockIdx.y;
    if (active && !active[r])
        return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    double s = 0.;
    for (int k = 0; k < nk; k++)
        s += h[(size_t) r * hs + k0 + k] * V[((size_t) (k0 + k) * nrhs + r) * n + i];
    w[(size_t) r * n + i] -= s;
}

// dst[r][i] = src[r][i] * scale[r] (scale given as 1 / norm); grid (ceil(n/256), nrhs)
__global__ void scale_kernel(const double* __restrict__ src, double* __restrict__ dst, int n, const double* __restrict__ nrm,
                             int nrm_stride, int nrm_index)
{
    const int r = blockIdx.y;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const double v = nrm[(size_t) r * nrm_stride + nrm_index];
    dst[(size_t) r * n + i] = v > 0. ? src[(size_t) r * n + i] * (1. / sqrt(v)) : 0.;
}

// x[r][i] += sum_k y[r][k] V[k][r][i];   grid (ceil(n/256), nrhs)
__global__ void combine_kernel(const double* __restrict__ V, const double* __restrict__ y, int ystride, int n, int nrhs,
                               const int* __restrict__ nk, double* __restrict__ x)
{
    const int r = blockIdx.y;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    double s = 0.;
    for (int k = 0; k < nk[r]; k++)
        s += y[(size_t) r * ystride + k] * V[((size_t) k * nrhs + r) * n + i];
    x[(size_t) r * n + i] += s;
}

// r = b - r (in place on r), used for residuals r = b - A x
__global__ void residual_kernel(const double* __restrict__ b, double* __restrict__ r, size_t n)
{
    const size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        r[i] = b[i] - r[i];
}

__global__ void axpy_kernel(double a, const double* __restrict__ x, double* __restrict__ y, size_t n)
{
    const size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        y[i] += a * x[i];
}

// One Arnoldi step for small systems in a single CTA per right-hand side: w = A v_j is given;
// modified Gram-Schmidt against V[0..j] (as KGeneralizedMinimalResidual.hh:219-231) applied twice,
// h[r][0..j] = sum of both passes' projections,
// beta[r] = |w| written to h[r][hs - 1], and V[j+1] = w / beta. One launch replaces the five of
// the multi-CTA path when n is small enough for one CTA to stream the basis.
constexpr int kArnoldiThreads = 1024;
__global__ void __launch_bounds__(kArnoldiThreads) arnoldi_small_kernel(double* __restrict__ V, double* __restrict__ w,
                                                                       int n, int nrhs, int j, double* __restrict__ h,
                                                                       int hs)
{
    __shared__ double sh[32];
    __shared__ double s_h[2];
    const int r = blockIdx.x;
    double* wr = w + (size_t) r * n;
    for (int k = 0; k <= j; k++)
        if (threadIdx.x == 0)
            h[(size_t) r * hs + k] = 0.;
    for (int pass = 0; pass < 2; pass++) {
        for (int k = 0; k <= j; k++) {
            const double* vk = V + ((size_t) k * nrhs + r) * n;
            double s = 0.;
            for (int i = threadIdx.x; i < n; i += blockDim.x)
                s += vk[i] * wr[i];
            s = block_sum(s, sh);
            if (threadIdx.x == 0) {
                s_h[0] = s;
                h[(size_t) r * hs + k] += s;
            }
            __syncthreads();
            const double hk = s_h[0];
            for (int i = threadIdx.x; i < n; i += blockDim.x)
                wr[i] -= hk * vk[i];
            __syncthreads();
        }
    }
    double s = 0.;
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        s += wr[i] * wr[i];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) {
        s_h[1] = sqrt(s);
        h[(size_t) r * hs + hs - 1] = s_h[1];
    }
    __syncthreads();
    const double beta = s_h[1];
    double* vn = V + ((size_t) (j + 1) * nrhs + r) * n;
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        vn[i] = beta > 0. ? wr[i] * (1. / beta) : 0.;
}

// y[r][i] = d[i] x[r][i], or y[r][i] += d[i] x[r][i] when accumulate (the Jacobi
// preconditioner, KJacobiPreconditioner.hh:40-45, and its use in forming the GMRES solution);
// grid (ceil(n/256), nrhs)
__global__ void diag_scale_kernel(const double* __restrict__ d, const double* __restrict__ x, double* __restrict__ y,
                                  int n, int accumulate)
{
    const int r = blockIdx.y;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const double v = d[i] * x[(size_t) r * n + i];
    y[(size_t) r * n + i] = accumulate ? y[(size_t) r * n + i] + v : v;
}

// d[i] = 1 / d[i]
__global__ void invert_kernel(double* __restrict__ d, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        d[i] = 1. / d[i];
}

// up to three inner products per right-hand side in one launch (BiCGStab's scalars):
// out[r][q] = sum_i a_q[r][i] b_q[r][i] for q < np, out row stride 4. grid (kDotBlocks, nrhs);
// partial[r][q][blk]; counter[r] starts at 0 and is reset. Each CTA sums a slice of the rows,
// the last CTA of a right-hand side sums the slices in block order (scheduling-independent).
struct DotPairs
{
    const double* a[3];
    const double* b[3];
    int np;
};
__global__ void __launch_bounds__(kDotThreads) pair_dot_kernel(DotPairs dp, int n, double* __restrict__ partial,
                                                               unsigned* __restrict__ counter, double* __restrict__ out)
{
    __shared__ double sh[32];
    __shared__ bool last;
    const int r = blockIdx.y;
    const int per = (n + gridDim.x - 1) / gridDim.x;
    const int i0 = blockIdx.x * per, i1 = min(n, i0 + per);
    double acc[3] = {0., 0., 0.};
    for (int i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
        const size_t k = (size_t) r * n + i;
#pragma unroll
        for (int q = 0; q < 3; q++)
            if (q < dp.np)
                acc[q] = fma(dp.a[q][k], dp.b[q][k], acc[q]);
    }
    for (int q = 0; q < dp.np; q++) {
        const double s = block_sum(acc[q], sh);
        if (threadIdx.x == 0)
            partial[((size_t) r * 4 + q) * gridDim.x + blockIdx.x] = s;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0)
        last = atomicAdd(counter + r, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last)
        return;
    __threadfence();
    if (threadIdx.x < dp.np) {
        double s = 0.;
        for (int b = 0; b < (int) gridDim.x; b++)
            s += __ldcg(partial + ((size_t) r * 4 + threadIdx.x) * gridDim.x + b);
        out[(size_t) r * 4 + threadIdx.x] = s;
    }
    if (threadIdx.x == 0)
        counter[r] = 0u;
}

// per-right-hand-side coefficients of a BiCGStab vector update
struct RhsCoef
{
    double a[kMaxRhs], b[kMaxRhs];
};

// p = r + beta (p - omega v)  (a = beta, b = omega; KBiconjugateGradientStabilized.hh:162-164)
__global__ void bicg_direction_kernel(const double* __restrict__ r, const double* __restrict__ v, double* __restrict__ p,
                                      int n, RhsCoef c)
{
    const int q = blockIdx.y;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const size_t k = (size_t) q * n + i;
    p[k] = r[k] + c.a[q] * (p[k] - c.b[q] * v[k]);
}

// s = r - alpha v  (a = alpha; :170-172)
__global__ void bicg_half_kernel(const double* __restrict__ r, const double* __restrict__ v, double* __restrict__ s,
                                 int n, RhsCoef c)
{
    const int q = blockIdx.y;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const size_t k = (size_t) q * n + i;
    s[k] = r[k] - c.a[q] * v[k];
}

// x += alpha y + omega z, r = s - omega t  (a = alpha, b = omega; :178-181)
__global__ void bicg_update_kernel(const double* __restrict__ y, const double* __restrict__ z,
                                   const double* __restrict__ s, const double* __restrict__ t, double* __restrict__ x,
                                   double* __restrict__ r, int n, RhsCoef c)
{
    const int q = blockIdx.y;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const size_t k = (size_t) q * n + i;
    x[k] = x[k] + c.a[q] * y[k] + c.b[q] * z[k];
    r[k] = s[k] - c.b[q] * t[k];
}

// non-finite check: flag[0] |= 1 when any value is NaN or Inf
__global__ void finite_kernel(const double* __restrict__ v, size_t n, int* __restrict__ flag)
{
    const size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && !isfinite(v[i]))
        atomicOr(flag, 1);
}

}  // namespace kemcu
