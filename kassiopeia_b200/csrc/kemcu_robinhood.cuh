// Robin Hood charge-density solve on the device (KRobinHood<double, KRobinHood_SingleThread>,
// KEMField/Source/LinearAlgebra/Solvers/include/KRobinHood.hh:61-104 and
// KRobinHood_SingleThread.hh:59-120).
//
// The method is a sequence of single-element corrections, each depending on the previous one
// through the argmax of the residual, so one CTA runs the whole sequence without returning to
// the host: per sub-iteration every thread updates its rows of b_it (the operator applied to
// the current x) with column k of the operator, forms r_i = b_i - b_it_i exactly as the
// reference's FindResidual does, and the CTA reduces (max |r_i|, first index) to the next k.
// Columns come from the assembled FP64 operator (contiguous in its column-major layout) or are
// computed on the fly from element k's record (the same entry<> as the matvec kernels).
#pragma once

#include "kemcu_kernels.cuh"

namespace kemcu
{

constexpr int kRhThreads = 1024;

// state carried between launches (one per solve)
struct RhState
{
    long long subiterations;  // corrections applied so far
    double rmax;              // max_i |b_i - b_it_i| for the current b_it
    double norm;              // relative residual at the last check (starts at 1, KIterativeSolver.hh:15)
    int k;                    // index of rmax (first on ties); -1 before the first pass
    int sub;                  // sub-iterations since the last check (KRobinHood.hh:78-88)
    int iterations;           // residual checks so far
    int pad;
};

// diagonal A(k, k) of the operator (entry<false>: the plain FP64 form, as the matvec)
__global__ void diag_kernel(const double* __restrict__ rec, const TargetRec* __restrict__ tgt, int n,
                            double* __restrict__ diag)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n)
        return;
    const TargetRec t = tgt[k];
    diag[k] = entry<false>(rec + (size_t) k * rRecSize, t, v3(t.cen[0], t.cen[1], t.cen[2]));
}

// (value, index) maximum over the CTA: larger value wins, the smaller index on equal values
__device__ __forceinline__ void cta_argmax(double& v, int& i, double* s_v, int* s_i)
{
    for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_down_sync(0xffffffffu, v, o);
        const int oi = __shfl_down_sync(0xffffffffu, i, o);
        if (ov > v || (ov == v && oi < i)) {
            v = ov;
            i = oi;
        }
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) {
        s_v[w] = v;
        s_i[w] = i;
    }
    __syncthreads();
    if (w == 0) {
        v = l < (int) (blockDim.x >> 5) ? s_v[l] : -1.;
        i = l < (int) (blockDim.x >> 5) ? s_i[l] : 0x7fffffff;
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_down_sync(0xffffffffu, v, o);
            const int oi = __shfl_down_sync(0xffffffffu, i, o);
            if (ov > v || (ov == v && oi < i)) {
                v = ov;
                i = oi;
            }
        }
        if (l == 0) {
            s_v[0] = v;
            s_i[0] = i;
        }
    }
    __syncthreads();
    v = s_v[0];
    i = s_i[0];
}

// up to `budget` sub-iterations (one CTA of kRhThreads threads); stops early once a residual
// check finds norm <= tol (after completing that sub-iteration, as KRobinHood::Solve does)
template<bool ASSEMBLED>
__global__ void __launch_bounds__(kRhThreads) robin_hood_kernel(const double* __restrict__ rec, const TargetRec* __restrict__ tgt,
                                                                int n, const double* __restrict__ A, size_t ld,
                                                                const double* __restrict__ diag, const double* __restrict__ b,
                                                                double* __restrict__ bit, double* __restrict__ x,
                                                                double binf, double tol, int interval, long long budget,
                                                                RhState* __restrict__ st)
{
    __shared__ double s_rec[rRecSize];
    __shared__ double s_v[32];
    __shared__ int s_i[32];
    const int tid = threadIdx.x;
    RhState S = *st;
    // residual of the current b_it and its largest element
    auto scan = [&](double& rv, int& ri) {
        rv = -1.;
        ri = 0x7fffffff;
        for (int i = tid; i < n; i += blockDim.x) {
            const double r = fabs(b[i] - bit[i]);
            if (r > rv) {
                rv = r;
                ri = i;
            }
        }
        cta_argmax(rv, ri, s_v, s_i);
    };
    if (S.k < 0)
        scan(S.rmax, S.k);
    long long done = 0;
    while (S.norm > tol && done < budget) {
        if (++S.sub % interval == 0) {
            S.sub = 0;
            S.norm = S.rmax / binf;
            S.iterations++;
        }
        const int k = S.k;
        const double c = (b[k] - bit[k]) / diag[k];
        __syncthreads();  // every thread has read bit[k] before it is updated
        if (tid == 0)
            x[k] += c;
        if (!ASSEMBLED) {
            if (tid < rRecSize)
                s_rec[tid] = rec[(size_t) k * rRecSize + tid];
            __syncthreads();
        }
        double rv = -1.;
        int ri = 0x7fffffff;
        for (int i = tid; i < n; i += blockDim.x) {
            double a;
            if (ASSEMBLED)
                a = A[(size_t) k * ld + i];
            else {
                const TargetRec t = tgt[i];
                a = entry<false>(s_rec, t, v3(t.cen[0], t.cen[1], t.cen[2]));
            }
            const double v = __dadd_rn(bit[i], __dmul_rn(a, c));  // reference rounding, no FMA
            bit[i] = v;
            const double r = fabs(b[i] - v);
            if (r > rv) {
                rv = r;
                ri = i;
            }
        }
        cta_argmax(rv, ri, s_v, s_i);  // ends with a CTA barrier: bit[] is visible to all threads
        S.rmax = rv;
        S.k = ri;
        done++;
    }
    if (tid == 0) {
        S.subiterations += done;
        *st = S;
    }
}

}  // namespace kemcu
