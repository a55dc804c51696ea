// Robin Hood charge-density solve on the device (KRobinHood<double, KRobinHood_SingleThread>,
// KEMField/Source/LinearAlgebra/Solvers/include/KRobinHood.hh:61-104 and
// KRobinHood_SingleThread.hh:59-120).
//
// The method is a sequence of single-element corrections, each depending on the previous one
// through the argmax of the residual. One persistent cooperative launch runs a whole stretch of
// them on as many CTAs as the rows can use: every CTA owns a contiguous block of rows of
// b_it (the operator applied to the current x); per correction it updates its rows with
// column k of the operator, forms r_i = b_i - b_it_i exactly as the reference's FindResidual
// does, reduces (max |r_i|, first index, signed r_i) over its rows and publishes the result;
// after one grid-wide barrier every CTA reduces the published results itself (the same
// deterministic reduction everywhere, so all CTAs agree on the next k without a second
// barrier). The correction value c = r_k / A(k, k) comes from the published signed residual,
// so no CTA reads a row of b_it that its owner is about to change. Columns come from the
// assembled FP64 operator (contiguous in its column-major layout) or are computed on the fly
// from element k's record (the same entry<> as the matvec kernels); the OpenCL plugin spreads
// the same column update over the device (kEMField_RobinHood_kernel.cl:219-276).
//
// The grid barrier is a generation counter in global memory; every wait gives up after ~2^31
// cycles (about a second), records KEMCU_ETIMEOUT in the flag word and leaves the loop, so a
// CTA that stops arriving makes every other one return within the limit.
#pragma once

#include <cooperative_groups.h>

#include "kemcu_kernels.cuh"

namespace kemcu
{
namespace cg = cooperative_groups;

constexpr int kRhThreads = 256;

// state carried between launches (one per solve)
struct RhState
{
    long long subiterations;  // corrections applied so far
    double rmax;              // max_i |b_i - b_it_i| for the current b_it
    double rk;                // b_k - b_it_k at the current k (signed)
    double dk;                // A(k, k)
    double norm;              // relative residual at the last check (starts at 1, KIterativeSolver.hh:15)
    int k;                    // index of rmax (first on ties); -1 before the first pass
    int sub;                  // sub-iterations since the last check (KRobinHood.hh:78-88)
    int iterations;           // residual checks so far
    int pad;
};

// one CTA's reduction result, published for the grid-wide reduction
struct RhPart
{
    double v;   // max |r_i| over the CTA's rows
    double r;   // signed r_i at that row
    double d;   // A(i, i) of that row
    int i;      // its row (first on ties)
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

// Near-field list of the operator's columns (compressed by column): the pairs (row i, column
// k) that take the analytic band (band_of == 0, every diagonal entry among them) with their
// FP64 entries, rows increasing within a column. The matrix-free corrections then compute only
// quadrature-band entries on the fly, whose latency is short and uniform, and add the few
// analytic ones from the list. One warp per column.
__global__ void near_count_kernel(const double* __restrict__ rec, const TargetRec* __restrict__ tgt, int n,
                                  int* __restrict__ count)
{
    const int k = (int) ((blockIdx.x * (size_t) blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (k >= n)
        return;
    const double* e = rec + (size_t) k * rRecSize;
    int c = 0;
    for (int i0 = 0; i0 < n; i0 += 32) {
        const int i = i0 + lane;
        bool near = false;
        if (i < n)
            near = band_of(e, v3(tgt[i].cen[0], tgt[i].cen[1], tgt[i].cen[2])) == 0;
        c += __popc(__ballot_sync(0xffffffffu, near));
    }
    if (lane == 0)
        count[k] = c;
}

__global__ void near_fill_kernel(const double* __restrict__ rec, const TargetRec* __restrict__ tgt, int n,
                                 const long long* __restrict__ ptr, int* __restrict__ rows, double* __restrict__ vals)
{
    const int k = (int) ((blockIdx.x * (size_t) blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (k >= n)
        return;
    const double* e = rec + (size_t) k * rRecSize;
    long long pos = ptr[k];
    for (int i0 = 0; i0 < n; i0 += 32) {
        const int i = i0 + lane;
        bool near = false;
        TargetRec t{};
        V3 C = v3(0., 0., 0.);
        if (i < n) {
            t = tgt[i];
            C = v3(t.cen[0], t.cen[1], t.cen[2]);
            near = band_of(e, C) == 0;
        }
        const unsigned m = __ballot_sync(0xffffffffu, near);
        if (near) {
            const long long q = pos + __popc(m & ((1u << lane) - 1u));
            rows[q] = i;
            vals[q] = entry<false>(e, t, C);
        }
        pos += __popc(m);
    }
}

// the larger |r| wins, the smaller index on equal values
__device__ __forceinline__ void rh_better(RhPart& a, const RhPart& b)
{
    if (b.v > a.v || (b.v == a.v && b.i < a.i))
        a = b;
}

__device__ __forceinline__ RhPart rh_shfl_down(const RhPart& a, int o)
{
    RhPart b;
    b.v = __shfl_down_sync(0xffffffffu, a.v, o);
    b.r = __shfl_down_sync(0xffffffffu, a.r, o);
    b.d = __shfl_down_sync(0xffffffffu, a.d, o);
    b.i = __shfl_down_sync(0xffffffffu, a.i, o);
    b.pad = 0;
    return b;
}

__device__ __forceinline__ RhPart rh_warp_best(RhPart a)
{
    for (int o = 16; o > 0; o >>= 1)
        rh_better(a, rh_shfl_down(a, o));
    return a;
}

__device__ __forceinline__ RhPart rh_none()
{
    RhPart p;
    p.v = -1.;
    p.r = 0.;
    p.d = 1.;
    p.i = 0x7fffffff;
    p.pad = 0;
    return p;
}

// best over the CTA, result in s[0] (visible to all threads on return)
__device__ __forceinline__ RhPart rh_cta_best(RhPart a, RhPart* s)
{
    a = rh_warp_best(a);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0)
        s[w] = a;
    __syncthreads();
    if (w == 0) {
        a = l < (int) (blockDim.x >> 5) ? s[l] : rh_none();
        a = rh_warp_best(a);
        if (l == 0)
            s[0] = a;
    }
    __syncthreads();
    return s[0];
}

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// grid-wide barrier over gridDim.x co-resident CTAs: bar[0] counts arrivals, bar[1] is the
// generation. False when the wait gave up (~2^31 cycles).
__device__ __forceinline__ bool grid_barrier(unsigned* bar, unsigned& gen, int* s_ok)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        __threadfence();
        const unsigned arrived = atomicAdd(&bar[0], 1u) + 1u;
        if (arrived == gridDim.x) {
            bar[0] = 0u;
            __threadfence();
            atomicExch(&bar[1], gen + 1u);
        }
        else {
            const long long t0 = clock64();
            while (ld_acquire_u32(&bar[1]) == gen)
                if (clock64() - t0 > (1ll << 31)) {
                    ok = 0;
                    break;
                }
        }
        __threadfence();
        *s_ok = ok;
    }
    gen++;
    __syncthreads();
    return *s_ok != 0;
}

// up to `budget` sub-iterations; stops early once a residual check finds norm <= tol (after
// completing that sub-iteration, as KRobinHood::Solve does). The CTA's rows of b_it, b and the
// diagonal live in shared memory for the launch (dynamic: 3 x rows-per-CTA doubles); b_it is
// written back at the end. Matrix-free columns: quadrature-band entries on the fly, analytic
// ones from the near-field list (near_ptr[k] .. near_ptr[k + 1]). part: 2 x gridDim.x results
// (double-buffered by exchange parity); bar: {arrivals, generation}, zero arrivals on entry
// (every CTA reads the generation before it first arrives, so all start from the same value);
// flag |= 2 when a barrier wait gave up (bar must then be cleared before the next launch).
//
// CLUSTER: the grid is one thread-block cluster (up to 16 CTAs holding all rows of the system);
// the per-correction exchange is each CTA's best row in its shared memory, the hardware cluster
// barrier, and a read of every CTA's result through distributed shared memory (double-buffered by
// parity) instead of `part` and the software grid barrier; it has no wait that could time out.
template<bool ASSEMBLED, bool CLUSTER>
__global__ void __launch_bounds__(kRhThreads) robin_hood_kernel(const double* __restrict__ rec, const TargetRec* __restrict__ tgt,
                                                                int n, const double* __restrict__ A, size_t ld,
                                                                const long long* __restrict__ near_ptr,
                                                                const int* __restrict__ near_row,
                                                                const double* __restrict__ near_val,
                                                                const double* __restrict__ diag, const double* __restrict__ b,
                                                                double* __restrict__ bit, double* __restrict__ x,
                                                                double binf, double tol, int interval, long long budget,
                                                                RhState* __restrict__ st, RhPart* __restrict__ part,
                                                                unsigned* __restrict__ bar, int* __restrict__ flag)
{
    extern __shared__ __align__(16) double s_rows[];  // [3][per]: b_it, b, A(i, i)
    __shared__ double s_rec[rRecSize];
    __shared__ RhPart s_part[32];
    __shared__ RhPart s_best;
    __shared__ RhPart s_slot[2];  // CLUSTER: this CTA's best row, read by the cluster's CTAs
    __shared__ int s_ok;
    const int tid = threadIdx.x, G = (int) gridDim.x;
    const int per = (n + G - 1) / G;
    const int r0 = min(n, (int) blockIdx.x * per), r1 = min(n, r0 + per), nr = r1 - r0;
    double* s_bit = s_rows;
    double* s_b = s_rows + per;
    double* s_dg = s_rows + 2 * per;
    for (int q = tid; q < nr; q += blockDim.x) {
        s_bit[q] = bit[r0 + q];
        s_b[q] = b[r0 + q];
        s_dg[q] = diag[r0 + q];
    }
    RhState S = *st;
    unsigned gen = ld_acquire_u32(&bar[1]);
    int parity = 0;
    __syncthreads();
    // this thread's best row of the CTA's residual r_i = b_i - b_it_i
    auto my_best = [&]() {
        RhPart mine = rh_none();
        for (int q = tid; q < nr; q += blockDim.x) {
            const double r = s_b[q] - s_bit[q];
            RhPart p;
            p.v = fabs(r);
            p.r = r;
            p.d = s_dg[q];
            p.i = r0 + q;
            p.pad = 0;
            rh_better(mine, p);
        }
        return mine;
    };
    // publish this CTA's best, wait for all, reduce the published results (every CTA alike)
    auto exchange = [&](RhPart mine) -> bool {
        mine = rh_cta_best(mine, s_part);
        if (CLUSTER) {
            if (tid == 0)
                s_slot[parity] = mine;
            cg::this_cluster().sync();
            if (tid < 32) {
                RhPart a = rh_none();
                for (int q = tid; q < G; q += 32)
                    rh_better(a, *cg::this_cluster().map_shared_rank(&s_slot[parity], q));
                a = rh_warp_best(a);
                if (tid == 0)
                    s_best = a;
            }
            __syncthreads();
            S.rmax = s_best.v;
            S.k = s_best.i;
            S.rk = s_best.r;
            S.dk = s_best.d;
            parity ^= 1;
            return true;
        }
        if (tid == 0)
            part[parity * G + blockIdx.x] = mine;
        if (G > 1 && !grid_barrier(bar, gen, &s_ok))
            return false;
        if (tid < 32) {
            RhPart a = rh_none();
            if (G == 1) {
                if (tid == 0)
                    a = mine;
            }
            else
                for (int q = tid; q < G; q += 32) {
                    const RhPart* src = part + parity * G + q;
                    RhPart p;
                    p.v = __ldcg(&src->v);
                    p.r = __ldcg(&src->r);
                    p.d = __ldcg(&src->d);
                    p.i = __ldcg(&src->i);
                    p.pad = 0;
                    rh_better(a, p);
                }
            a = rh_warp_best(a);
            if (tid == 0)
                s_best = a;
        }
        __syncthreads();
        S.rmax = s_best.v;
        S.k = s_best.i;
        S.rk = s_best.r;
        S.dk = s_best.d;
        parity ^= 1;
        return true;
    };
    bool ok = true;
    if (S.k < 0)
        ok = exchange(my_best());
    long long done = 0;
    while (ok && S.norm > tol && done < budget) {
        if (++S.sub % interval == 0) {
            S.sub = 0;
            S.norm = S.rmax / binf;
            S.iterations++;
        }
        const int k = S.k;
        const double c = S.rk / S.dk;  // (b_k - b_it_k) / A(k, k), KRobinHood_SingleThread.hh:95-109
        if (blockIdx.x == 0 && tid == 0)
            x[k] += c;
        if (ASSEMBLED) {
            for (int q = tid; q < nr; q += blockDim.x) {
                const double a = A[(size_t) k * ld + r0 + q];
                s_bit[q] = __dadd_rn(s_bit[q], __dmul_rn(a, c));  // reference rounding, no FMA
            }
        }
        else {
            const long long p0 = near_ptr[k], p1 = near_ptr[k + 1];
            if (tid < rRecSize)
                s_rec[tid] = rec[(size_t) k * rRecSize + tid];
            __syncthreads();
            for (int q = tid; q < nr; q += blockDim.x) {
                const TargetRec t = tgt[r0 + q];
                const V3 C = v3(t.cen[0], t.cen[1], t.cen[2]);
                V3 d;
                double r2;
                const int band = band_of(s_rec, C, d, r2);
                if (band != 0)
                    s_bit[q] = __dadd_rn(s_bit[q], __dmul_rn(entry_far<false>(s_rec, t, C, d, r2, band), c));
            }
            // the analytic entries of column k that fall on this CTA's rows (distinct rows)
            for (long long q = p0 + tid; q < p1; q += blockDim.x) {
                const int i = near_row[q];
                if (i >= r0 && i < r1)
                    s_bit[i - r0] = __dadd_rn(s_bit[i - r0], __dmul_rn(near_val[q], c));
            }
        }
        __syncthreads();
        ok = exchange(my_best());  // its CTA barriers also free s_rec for the next column
        done++;
    }
    __syncthreads();
    for (int q = tid; q < nr; q += blockDim.x)
        bit[r0 + q] = s_bit[q];
    if (CLUSTER)
        cg::this_cluster().sync();  // no CTA leaves while another may still read its slots
    if (!ok && tid == 0)
        atomicOr(flag, 2);
    if (blockIdx.x == 0 && tid == 0) {
        S.subiterations += done;
        *st = S;
    }
}

}  // namespace kemcu
