// Direct-summation kernels: field evaluation at many points (K1), the matrix-free
// boundary-integral matvec (K2), operator assembly and the dense (assembled) matvec.
//
// Layout: one thread owns one evaluation point (a field point, or a target centroid for the
// matvec); a CTA of kThreads points streams its slice of the element records (256 B each)
// through a ring of shared-memory stages filled by bulk copies (ElementRing), and every
// thread sums the contributions with Kahan compensation, as the reference's
// KIntegratingFieldSolver does (KElectrostaticIntegratingFieldSolver.hh:261-339); the direct
// sum adds the 32 contributions of a tile in plain FP64 first and compensates across tiles
// (16 fewer FP64 operations per element, differences at the 1e-15 level). When there
// are too few points to fill the GPU the element list is split over gridDim.y; each split
// writes a partial sum to scratch and reduce_splits adds the splits in a fixed order, so the
// result does not depend on scheduling.
#pragma once

#include "kemcu_device.cuh"

namespace kemcu
{

constexpr int kThreads = 128;
// resident CTAs per SM the direct-sum kernels are compiled for (bounds their registers)
#ifndef KEMCU_MIN_BLOCKS
#define KEMCU_MIN_BLOCKS 5
#endif
constexpr int kMinBlocks = KEMCU_MIN_BLOCKS;

// Leading dimension of the assembled operator: rows padded to a multiple of 4 so that every
// column starts on a 16-byte boundary in both the FP64 and the FP32 copy.
__host__ __device__ __forceinline__ size_t op_ld(size_t n)
{
    return (n + 3) / 4 * 4;
}

struct Kahan
{
    double s = 0., c = 0.;
    __device__ __forceinline__ void add(double v)
    {
        const double y = v - c;
        const double t = s + y;
        c = (t - s) - y;
        s = t;
    }
};

// cooperative copy of `count` element records (256 B each) into shared memory (tracker)
__device__ __forceinline__ void load_tile(double* sm, const double* __restrict__ rec, int first, int count)
{
    const double2* src = reinterpret_cast<const double2*>(rec + (size_t) first * rRecSize);
    double2* dst = reinterpret_cast<double2*>(sm);
    const int n2 = count * (rRecSize / 2);
    for (int i = threadIdx.x; i < n2; i += blockDim.x)
        dst[i] = __ldg(src + i);
}

// ------------------------------------------------------------------------- element pipeline
// K1 streams element records through a ring of kPipe shared-memory stages of kFieldTile
// records each. A stage is filled by one bulk copy (cp.async.bulk, completion counted on the
// stage's mbarrier together with the 32 arrivals of the filling warp, whose lanes also store
// the tile's charge densities). Warps consume stages at their own pace; each warp counts its
// release of a stage in a shared counter, and the warp that releases it last refills it with
// the tile kPipe ahead. A warp therefore waits only for data, never for the other warps
// (which a __syncthreads per tile would impose), so warps that meet near-field elements and
// warps that meet far-field ones drift apart by up to kPipe - 1 tiles.
#ifndef KEMCU_FIELD_TILE
#define KEMCU_FIELD_TILE 32
#endif
#ifndef KEMCU_PIPE
#define KEMCU_PIPE 4
#endif
constexpr int kFieldTile = KEMCU_FIELD_TILE;
constexpr int kPipe = KEMCU_PIPE;
static_assert(kFieldTile <= 32 && kFieldTile % 2 == 0, "one lane of the filling warp per element");

__device__ __forceinline__ unsigned smem_u32(const void* p)
{
    return (unsigned) __cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned long long* bar)
{
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(unsigned long long* bar, unsigned bytes)
{
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity)
{
    unsigned ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(smem_u32(bar)), "r"(parity)
                 : "memory");
    return ok != 0u;
}
// bounded wait for the completion of the phase with the given parity: false after ~2^31
// cycles (about a second), which only a defect can cause
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity)
{
    if (mbar_try_wait(bar, parity))
        return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > (1ll << 31))
            return false;
    return true;
}
// same wait with a caller-chosen cycle limit (the failure-path self-test)
__device__ __forceinline__ bool mbar_wait_limit(unsigned long long* bar, unsigned parity, long long limit)
{
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > limit)
            return false;
    return true;
}

// Self-test of the timeout path: one warp waits on an mbarrier phase that completes only when
// `complete` is set (one arrival of the expected one); otherwise the wait gives up after
// `limit` cycles and the kernel reports it in flag (|= 2), as the element ring does.
__global__ void wait_timeout_selftest_kernel(int* __restrict__ flag, long long limit, int complete)
{
    __shared__ __align__(8) unsigned long long bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        mbar_init_fence();
    }
    __syncthreads();
    if (complete && threadIdx.x == 0)
        mbar_arrive(&bar);
    const bool ok = mbar_wait_limit(&bar, 0u, limit);
    if (!ok && threadIdx.x == 0)
        atomicOr(flag, 2);
}

__device__ __forceinline__ void fence_proxy_async()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// global -> shared bulk copy; addresses 16 B aligned, bytes a multiple of 16
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// element slice [e0, e1) of [first, last) for split blockIdx.y, in whole tiles
__device__ __forceinline__ void split_range(int first, int last, int& e0, int& e1)
{
    const int span = last - first;
    const int per = ((span + (int) gridDim.y - 1) / (int) gridDim.y + kFieldTile - 1) / kFieldTile * kFieldTile;
    e0 = min(last, first + (int) blockIdx.y * per);
    e1 = min(last, e0 + per);
}

// The ring: NP stages (kPipe by default) of kFieldTile element records plus SIDE doubles of
// per-element side data (charge densities, matvec operands) per element, stored by the filling
// warp's lanes. RingStorage lives in shared memory; ElementRing (registers) holds the CTA's
// element slice and a reference to it. A CYCLIC ring passes over the slice again and again
// (the tracker's stage evaluations) and keeps prefetching until finish().
template<int SIDE, int NP = kPipe> struct RingStorage
{
    double rec[NP][kFieldTile * rRecSize];
    double side[NP][SIDE > 0 ? SIDE : 1][kFieldTile];
    unsigned long long full[NP];
    unsigned rel[NP], used[NP];
};

template<int SIDE, int NP = kPipe, bool CYCLIC = false> struct ElementRing
{
    RingStorage<SIDE, NP>& S;
    int e0, e1;  // this CTA's element slice

    __device__ __forceinline__ ElementRing(RingStorage<SIDE, NP>& storage, int first, int last) : S(storage)
    {
        split_range(first, last, e0, e1);
        if (threadIdx.x < NP) {
            mbar_init(&S.full[threadIdx.x], 32);
            S.rel[threadIdx.x] = 0u;
            S.used[threadIdx.x] = 0u;
            mbar_init_fence();
        }
        __syncthreads();
    }
    __device__ __forceinline__ int tiles() const
    {
        return (e1 - e0 + kFieldTile - 1) / kFieldTile;
    }
    // first element of tile i of the sequence (CYCLIC: the slice is passed over repeatedly)
    __device__ __forceinline__ int first(int i) const
    {
        return e0 + (CYCLIC ? i % tiles() : i) * kFieldTile;
    }
    __device__ __forceinline__ int count(int i) const
    {
        return min(kFieldTile, e1 - first(i));
    }
    __device__ __forceinline__ const double* element(int i, int j) const
    {
        return S.rec[i % NP] + j * rRecSize;
    }
    __device__ __forceinline__ double side(int i, int k, int j) const
    {
        return S.side[i % NP][k][j];
    }
    // fill stage i % NP with tile i: called by all 32 lanes of one warp;
    // side_fn(double (*side)[kFieldTile], int t0, int cnt, int lane) stores the side data
    template<class F> __device__ __forceinline__ void fill(const double* __restrict__ src, int i, F side_fn)
    {
        const int s = i % NP, t0 = first(i), cnt = count(i), lane = threadIdx.x & 31;
        side_fn(S.side[s], t0, cnt, lane);
        if (lane == 0) {
            S.used[s]++;
            fence_proxy_async();
            const unsigned bytes = (unsigned) (cnt * rRecSize * sizeof(double));
            mbar_arrive_tx(&S.full[s], bytes);
            bulk_g2s(S.rec[s], src + (size_t) t0 * rRecSize, bytes, &S.full[s]);
        }
        else
            mbar_arrive(&S.full[s]);
    }
    template<class F> __device__ __forceinline__ void prologue(const double* __restrict__ src, F side_fn)
    {
        if (threadIdx.x < 32)
            for (int i = 0; i < (CYCLIC ? NP : min(NP, tiles())); i++)
                fill(src, i, side_fn);
    }
    __device__ __forceinline__ bool wait(int i)
    {
        return mbar_wait(&S.full[i % NP], (unsigned) (i / NP) & 1u);
    }
    // whole warp: release tile i; the warp that releases a stage last refills it
    template<class F> __device__ __forceinline__ void release(const double* __restrict__ src, int i, F side_fn)
    {
        const int s = i % NP;
        __syncwarp();
        unsigned last = 0u;
        if ((threadIdx.x & 31) == 0) {
            __threadfence_block();
            last = atomicAdd(&S.rel[s], 1u) % (blockDim.x >> 5) == (blockDim.x >> 5) - 1u;
        }
        last = __shfl_sync(0xffffffffu, last, 0);
        if (last && (CYCLIC || i + NP < tiles())) {
            __threadfence_block();
            fill(src, i + NP, side_fn);
        }
    }
    // after the tile loop (all threads): report a timed-out wait in flag (|= 2) and wait,
    // bounded, for copies still in flight
    __device__ __forceinline__ void finish(bool ok, int* flag)
    {
        if (!ok && (threadIdx.x & 31) == 0)
            atomicOr(flag, 2);
        __syncthreads();
        if (threadIdx.x < NP && S.used[threadIdx.x] > 0u)
            mbar_wait(&S.full[threadIdx.x], (S.used[threadIdx.x] - 1u) & 1u);
    }
};

// A warp's points in a bounding sphere, and whether a tile of the element ring holds an element
// within its analytic band of any of them: the element's centre distance from the sphere's
// centre, less the radius and a 1e-12 rounding allowance, squared, must exceed the band-0 cut with
// a 1e-6 margin for the tile to be far (then the fast band comparison of band_of decides band >= 1
// for every pair, as the exact one would). Called by all 32 lanes.
__device__ __forceinline__ void warp_sphere(bool active, V3 P, V3& wc, double& wr)
{
    double lo[3] = {active ? P.x : 1e300, active ? P.y : 1e300, active ? P.z : 1e300};
    double hi[3] = {active ? P.x : -1e300, active ? P.y : -1e300, active ? P.z : -1e300};
    for (int o = 16; o > 0; o >>= 1)
        for (int c = 0; c < 3; c++) {
            lo[c] = fmin(lo[c], __shfl_xor_sync(0xffffffffu, lo[c], o));
            hi[c] = fmax(hi[c], __shfl_xor_sync(0xffffffffu, hi[c], o));
        }
    wc = v3(0.5 * (lo[0] + hi[0]), 0.5 * (lo[1] + hi[1]), 0.5 * (lo[2] + hi[2]));
    wr = 0.5 * sqrt((hi[0] - lo[0]) * (hi[0] - lo[0]) + (hi[1] - lo[1]) * (hi[1] - lo[1]) +
                    (hi[2] - lo[2]) * (hi[2] - lo[2]));
}
template<class Ring> __device__ __forceinline__ bool tile_near(const Ring& R, int i, int cnt, V3 wc, double wr)
{
    bool near = false;
    for (int j = (int) (threadIdx.x & 31); j < cnt; j += 32) {
        const double* e = R.element(i, j);
        const double dx = e[rCen] - wc.x, dy = e[rCen + 1] - wc.y, dz = e[rCen + 2] - wc.z;
        const double dist = sqrt(dx * dx + dy * dy + dz * dz);
        const double dm = dist - wr - 1e-12 * (dist + wr);
        near = near || !(dm > 0. && dm * dm > e[rCut] * (1. + 1e-6));
    }
    return __any_sync(0xffffffffu, near);
}

// K1: field and/or potential at points. out layout per point: (Ex, Ey, Ez, phi).
// The analytic near-field pairs (band 0: RWG triangles and rectangles, analytic wires) are
// evaluated in place through a non-inlined call: a design with a call-free quadrature kernel and
// a second kernel for the analytic pairs was built and measured slower (the near pass ran alone,
// latency-bound, where here its latency hides behind other warps' quadrature work).
// nsplit == gridDim.y; partial != nullptr when nsplit > 1 (then out is untouched).
// flag |= 2 if a pipeline wait timed out (the outputs are then incomplete).
// MINB (resident CTAs per SM the registers are bounded for) and NP (ring stages) are the shapes
// the autotuner chooses between (field_variants); neither changes an operation or its order, so
// every variant gives the same result bit for bit. F32: the FP32 far-field form of the cubature
// bands (precision KEMCU_FP32), the tile and Kahan sums staying FP64.
template<bool MIXED, bool POT, bool FIELD, int MINB = kMinBlocks, int NP = kPipe, bool F32 = false>
__global__ void __launch_bounds__(kThreads, MINB) field_kernel(const double* __restrict__ rec, const double* __restrict__ sigma,
                                                               int n_elem, const double* __restrict__ pts, int n_pts,
                                                               double* __restrict__ out, double* __restrict__ partial,
                                                               int* __restrict__ flag)
{
    __shared__ __align__(128) RingStorage<1, NP> S;
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = p < n_pts;
    V3 P = v3(0., 0., 0.);
    if (active)
        P = v3(pts[3 * p], pts[3 * p + 1], pts[3 * p + 2]);
    ElementRing<1, NP> R(S, 0, n_elem);
    auto side = [&](double (*sd)[kFieldTile], int t0, int cnt, int lane) {
        if (lane < cnt)
            sd[0][lane] = sigma[t0 + lane];
    };
    R.prologue(rec, side);
    const int ntiles = R.tiles();
    // the warp's points in a bounding sphere (no sphere without active lanes, and then every
    // tile takes the general path)
    V3 wc;
    double wr;
    warp_sphere(active, P, wc, wr);
    const bool warp_active = __any_sync(0xffffffffu, active);
    Kahan kx, ky, kz, kp;
    bool ok = true;
    for (int i = 0; i < ntiles; i++) {
        if (!R.wait(i)) {
            ok = false;
            break;
        }
        const int cnt = R.count(i);
        // far tile: every element of the tile is beyond its analytic band for every point of the
        // warp, so the pair loop needs no analytic call
        const bool near = !warp_active || tile_near(R, i, cnt, wc, wr);
        if (active) {
            double tx = 0., ty = 0., tz = 0., tp = 0.;
            if (!near) {
                for (int j = 0; j < cnt; j++) {
                    const Out4 r = epi_beyond_near<MIXED, POT, FIELD, F32>(R.element(i, j), P);
                    const double sg = R.side(i, 0, j);
                    if (FIELD) {
                        tx = fma(r.ex, sg, tx);
                        ty = fma(r.ey, sg, ty);
                        tz = fma(r.ez, sg, tz);
                    }
                    if (POT)
                        tp = fma(r.phi, sg, tp);
                }
            }
            else
                for (int j = 0; j < cnt; j++) {
                    const Out4 r = epi<MIXED, POT, FIELD, F32>(R.element(i, j), P);
                    const double sg = R.side(i, 0, j);
                    if (FIELD) {
                        tx = fma(r.ex, sg, tx);
                        ty = fma(r.ey, sg, ty);
                        tz = fma(r.ez, sg, tz);
                    }
                    if (POT)
                        tp = fma(r.phi, sg, tp);
                }
            if (FIELD) {
                kx.add(tx);
                ky.add(ty);
                kz.add(tz);
            }
            if (POT)
                kp.add(tp);
        }
        R.release(rec, i, side);
    }
    R.finish(ok, flag);
    if (!active)
        return;
    double* o = partial ? partial + ((size_t) blockIdx.y * n_pts + p) * 4 : out + (size_t) p * 4;
    o[0] = kx.s;
    o[1] = ky.s;
    o[2] = kz.s;
    o[3] = kp.s;
}

// fixed-order sum of gridDim.y partial results: out[i] = sum_s partial[s][i]
__global__ void reduce_splits(const double* __restrict__ partial, int nsplit, size_t n, double* __restrict__ out)
{
    const size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    Kahan k;
    for (int s = 0; s < nsplit; s++)
        k.add(partial[(size_t) s * n + i]);
    out[i] = k.s;
}

// Target description for matrix rows: centroid, boundary kind, outward normal and the
// Neumann self-term value (KElectrostaticBoundaryIntegrator.hh:260-280)
struct TargetRec
{
    double cen[3];
    double normal[3];
    double diag;      // (1 + eps_r) / (1 - eps_r) / (2 eps0) for Neumann rows
    double neumann;   // 0 Dirichlet, 1 Neumann
};

// one matrix entry A(i, j) with source record e and target t (F32: the FP32 far-field form of
// the cubature bands)
template<bool MIXED, bool F32 = false> __device__ __forceinline__ double entry(const double* e, const TargetRec& t, V3 C)
{
    if (t.neumann == 0.) {
        return epi<MIXED, true, false, F32>(e, C).phi;
    }
    const V3 cs = ld3(e + rCen2);
    const double dist = norm(cs - C);
    if (dist >= 1e-12) {
        const Out4 r = epi<MIXED, false, true, F32>(e, C);
        return r.ex * t.normal[0] + r.ey * t.normal[1] + r.ez * t.normal[2];
    }
    return t.diag;
}

// an entry whose pair is in a quadrature band (band_of returned band >= 1 with d, r2): the same
// value as entry<MIXED>, without the analytic near-field code (a Neumann self term is band 0)
template<bool MIXED>
__device__ __forceinline__ double entry_far(const double* e, const TargetRec& t, V3 C, V3 d, double r2, int band)
{
    if (t.neumann == 0.)
        return epi_far<MIXED, true, false>(e, C, d, r2, band).phi;
    const Out4 r = epi_far<MIXED, false, true>(e, C, d, r2, band);
    return r.ex * t.normal[0] + r.ey * t.normal[1] + r.ez * t.normal[2];
}

// one entry A(i, j) (kemcu_matrix_element), the FP64 form the matvec uses
__global__ void entry_kernel(const double* __restrict__ rec, const TargetRec* __restrict__ tgt, int i, int j,
                             double* __restrict__ a)
{
    const TargetRec t = tgt[i];
    *a = entry<false>(rec + (size_t) j * rRecSize, t, v3(t.cen[0], t.cen[1], t.cen[2]));
}

// K2: y[r][i] = sum_j A(i, j) x[r][j] for r < nrhs (nrhs <= NR <= kMaxRhs), entries
// recomputed on the fly (KMatrix::Multiply over KBoundaryIntegralMatrix::operator(),
// KMatrix.hh:92-99, KBoundaryIntegralMatrix.hh:31-55). Same element ring as K1, with the
// operand values of the tile as side data.
constexpr int kMaxRhs = 8;
template<bool MIXED, int NR, bool F32 = false>
__global__ void __launch_bounds__(kThreads, kMinBlocks) matvec_kernel(const double* __restrict__ rec, const TargetRec* __restrict__ tgt,
                                                          int n, const double* __restrict__ x, int nrhs,
                                                          double* __restrict__ y, double* __restrict__ partial,
                                                          int* __restrict__ flag)
{
    __shared__ __align__(128) RingStorage<NR> S;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = i < n;
    TargetRec t{};
    V3 C = v3(0., 0., 0.);
    if (active) {
        t = tgt[i];
        C = v3(t.cen[0], t.cen[1], t.cen[2]);
    }
    ElementRing<NR> R(S, 0, n);
    auto side = [&](double (*sd)[kFieldTile], int t0, int cnt, int lane) {
        if (lane < cnt)
            for (int r = 0; r < nrhs; r++)
                sd[r][lane] = x[(size_t) r * n + t0 + lane];
    };
    R.prologue(rec, side);
    const int ntiles = R.tiles();
    // (the far-tile split of K1 was built here too and measured slower: the second pair loop
    // costs this kernel's register allocation more than the call it saves)
    Kahan acc[NR];
    bool ok = true;
    for (int q = 0; q < ntiles; q++) {
        if (!R.wait(q)) {
            ok = false;
            break;
        }
        if (active) {
            const int cnt = R.count(q);
            for (int j = 0; j < cnt; j++) {
                const double a = entry<MIXED, F32>(R.element(q, j), t, C);
#pragma unroll
                for (int r = 0; r < NR; r++)
                    if (r < nrhs)
                        acc[r].add(a * R.side(q, r, j));
            }
        }
        R.release(rec, q, side);
    }
    R.finish(ok, flag);
    if (!active)
        return;
#pragma unroll
    for (int r = 0; r < NR; r++) {
        if (r >= nrhs)
            break;
        if (partial)
            partial[((size_t) blockIdx.y * nrhs + r) * n + i] = acc[r].s;
        else
            y[(size_t) r * n + i] = acc[r].s;
    }
}

// operator assembly: column-major dense A (A[j * op_ld(n) + i] = A(i, j)) for columns
// [j0, j1), written in FP64 and, when a32 != nullptr, also rounded to FP32
template<bool MIXED>
__global__ void __launch_bounds__(kThreads, kMinBlocks) assemble_kernel(const double* __restrict__ rec, const TargetRec* __restrict__ tgt,
                                                            int n, int j0, int j1, double* __restrict__ a64,
                                                            float* __restrict__ a32, int* __restrict__ flag)
{
    __shared__ __align__(128) RingStorage<0> S;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = i < n;
    TargetRec t{};
    V3 C = v3(0., 0., 0.);
    if (active) {
        t = tgt[i];
        C = v3(t.cen[0], t.cen[1], t.cen[2]);
    }
    ElementRing<0> R(S, j0, j1);
    auto side = [](double (*)[kFieldTile], int, int, int) {};
    R.prologue(rec, side);
    const int ntiles = R.tiles();
    bool ok = true;
    for (int q = 0; q < ntiles; q++) {
        if (!R.wait(q)) {
            ok = false;
            break;
        }
        if (active) {
            const int t0 = R.first(q), cnt = R.count(q);
            for (int j = 0; j < cnt; j++) {
                const double a = entry<MIXED>(R.element(q, j), t, C);
                const size_t idx = (size_t) (t0 + j - j0) * op_ld(n) + i;
                if (a64)
                    a64[idx] = a;
                if (a32)
                    a32[idx] = (float) a;
            }
        }
        R.release(rec, q, side);
    }
    R.finish(ok, flag);
}

// dense matvec on the assembled column-major operator (leading dimension ld):
// y[r][i] = sum_j A[j*ld+i] x[r][j] for r < nrhs <= NR. A thread owns V consecutive rows
// (dense_rows<T, NR>: one 16-byte load per column), entries are streamed past L1/L2 with
// evict-first loads; the column range is split over gridDim.y. HBM-bound for one right-hand
// side (8 or 4 B per entry per call); several right-hand sides go to dense_mma_kernel, whose
// x operand needs no broadcast through shared memory.
template<typename T, int NR> __host__ __device__ constexpr int dense_rows()
{
    return (NR == 1 ? 16 : 8) / (int) sizeof(T);
}

template<typename T, int V> __device__ __forceinline__ void load_rows(const T* p, double* o)
{
    if constexpr (sizeof(T) == 4 && V == 4) {
        const float4 w = __ldcs(reinterpret_cast<const float4*>(p));
        o[0] = w.x;
        o[1] = w.y;
        o[2] = w.z;
        o[3] = w.w;
    }
    else if constexpr (sizeof(T) == 4 && V == 2) {
        const float2 w = __ldcs(reinterpret_cast<const float2*>(p));
        o[0] = w.x;
        o[1] = w.y;
    }
    else if constexpr (V == 2) {
        const double2 w = __ldcs(reinterpret_cast<const double2*>(p));
        o[0] = w.x;
        o[1] = w.y;
    }
    else
        o[0] = __ldcs(p);
}

template<typename T, int NR>
__global__ void __launch_bounds__(256) dense_matvec_kernel(const T* __restrict__ A, int n, size_t ld,
                                                           const double* __restrict__ x, int nrhs,
                                                           double* __restrict__ y, double* __restrict__ partial)
{
    constexpr int V = dense_rows<T, NR>();
    constexpr int kCols = 256;
    __shared__ __align__(16) double s_x[kCols][NR];  // the operand values of one column side by side
    const int row0 = (blockIdx.x * blockDim.x + threadIdx.x) * V;
    const int per = (n + gridDim.y - 1) / gridDim.y;
    const int e0 = blockIdx.y * per;
    const int e1 = min(n, e0 + per);
    double acc[NR][V];
#pragma unroll
    for (int r = 0; r < NR; r++)
#pragma unroll
        for (int q = 0; q < V; q++)
            acc[r][q] = 0.;
    for (int t0 = e0; t0 < e1; t0 += kCols) {
        const int cnt = min(kCols, e1 - t0);
        __syncthreads();
        for (int q = threadIdx.x; q < cnt * NR; q += blockDim.x) {
            const int j = q / NR, r = q % NR;
            s_x[j][r] = r < nrhs ? x[(size_t) r * n + t0 + j] : 0.;
        }
        __syncthreads();
        if (row0 < n) {
            const T* col = A + (size_t) t0 * ld + row0;
#pragma unroll 8
            for (int j = 0; j < cnt; j++) {
                double v[V];
                load_rows<T, V>(col + (size_t) j * ld, v);
#pragma unroll
                for (int r = 0; r < NR; r++) {
                    const double xr = s_x[j][r];
#pragma unroll
                    for (int q = 0; q < V; q++)
                        acc[r][q] = fma(v[q], xr, acc[r][q]);
                }
            }
        }
    }
    // unrolled over NR with a guard, so acc stays in registers (a runtime index would put it
    // in local memory)
#pragma unroll
    for (int r = 0; r < NR; r++) {
        if (r >= nrhs)
            break;
#pragma unroll
        for (int q = 0; q < V; q++) {
            const int i = row0 + q;
            if (i >= n)
                break;
            if (partial)
                partial[((size_t) blockIdx.y * nrhs + r) * n + i] = acc[r][q];
            else
                y[(size_t) r * n + i] = acc[r][q];
        }
    }
}

// dense matvec for several right-hand sides on the FP64 tensor cores: y[r] = A x[r] for
// r < nrhs <= 8 as a skinny GEMM, one mma.sync m8n8k4 (FP64 in, FP64 accumulate) per 8 rows x
// 4 columns x 8 right-hand sides. The 8 right-hand sides are the n = 8 of the MMA, so each lane
// takes its x operand straight from global memory (x is L2-resident) and no broadcast of x
// through shared memory is needed, which is what limits the FMA form at 8 right-hand sides.
// The MMA accumulates its k = 4 products in order, so the sums are those of a per-row FMA
// chain over the columns.
// Lane (g, t) = (lane / 4, lane % 4) reads column c0 + t in 16-byte loads of kPer = 16 / sizeof(T)
// rows; load h starts at row rowbase + 8 kPer h + kPer g for FP64 entries, so the 8 lanes of one
// column read 128 contiguous bytes per load, and at rowbase + 8 g + kPer h for FP32 entries, the
// lane's 8 rows side by side (measured faster for FP32, slower for FP64). Entry rt
// (h = rt / kPer, j = rt % kPer) is the A fragment of row tile rt, whose rows are those of
// entry rt over the 8 lane groups g; the accumulator pair of tile rt holds that row for
// right-hand sides 2t and 2t + 1.
// A warp covers 64 rows; the column range is split over gridDim.y as in dense_matvec_kernel.
// Entries are streamed with evict-first loads.
__device__ __forceinline__ void mma_884(double& d0, double& d1, double a, double b)
{
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
        : "+d"(d0), "+d"(d1)
        : "d"(a), "d"(b));
}

constexpr int kMmaRowsPerCta = 512;  // 8 warps x 64 rows

// (256, 1): ptxas then keeps more loads in flight (2 CTAs per SM for FP32 and FP64 entries);
// its default register heuristic gave fewer registers and ran 5 % / 25 % slower
template<typename T>
__global__ void __launch_bounds__(256, 1)
    dense_mma_kernel(const T* __restrict__ A, int n, size_t ld, const double* __restrict__ x, int nrhs,
                     double* __restrict__ y, double* __restrict__ partial)
{
    // 2 chunks of 4 columns per stage; FP32 entries run two register stages (loads of the next
    // stage in flight during the MMAs of this one: 8.46 -> 6.93 ms on a 100,000^2 operator with
    // 8 right-hand sides), FP64 entries one (already at 1.07x the HBM time; two stages ran 3 %
    // slower at 142 registers)
    constexpr int kU = 2;
    constexpr bool kPipelined = sizeof(T) == 4;
    constexpr int kPer = 16 / (int) sizeof(T);     // rows per 16-byte load
    constexpr int kLoads = 8 / kPer;
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int rowbase = blockIdx.x * kMmaRowsPerCta + (threadIdx.x >> 5) * 64;
    const int per = (n + gridDim.y - 1) / gridDim.y;
    const int e0 = blockIdx.y * per;
    const int e1 = min(n, e0 + per);
    const double* xg = x + (size_t) min(g, nrhs - 1) * n;
    const bool rhs_ok = g < nrhs;
    // load h starts at row r0 + step h (step a compile-time constant); a load is issued when its
    // first row is inside the matrix: ld is a multiple of 4 and that row one of kPer, so a
    // started group of kPer rows ends below ld
    constexpr int kStep = sizeof(T) == 4 ? kPer : 8 * kPer;
    const int r0 = sizeof(T) == 4 ? rowbase + 8 * g : rowbase + kPer * g;
    double acc[8][2];
#pragma unroll
    for (int rt = 0; rt < 8; rt++)
        acc[rt][0] = acc[rt][1] = 0.;
    // kU chunks of 4 columns starting at column cb: entries into a, x values into b (zeros
    // outside the row and column ranges, with no memory access there)
    auto load = [&](T (&a)[kU][8], double (&b)[kU], int cb) {
#pragma unroll
        for (int u = 0; u < kU; u++) {
            const int c = cb + 4 * u + t;
            const bool col_ok = c < e1;
            const T* p = A + (size_t) (col_ok ? c : e0) * ld + (r0 < n ? r0 : 0);
#pragma unroll
            for (int h = 0; h < kLoads; h++) {
                const bool ok = col_ok && r0 + kStep * h < n;
                if constexpr (sizeof(T) == 4) {
                    float4 w = make_float4(0.f, 0.f, 0.f, 0.f);
                    if (ok)
                        w = __ldcs(reinterpret_cast<const float4*>(p + kStep * h));
                    a[u][4 * h] = w.x, a[u][4 * h + 1] = w.y, a[u][4 * h + 2] = w.z, a[u][4 * h + 3] = w.w;
                }
                else {
                    double2 w = make_double2(0., 0.);
                    if (ok)
                        w = __ldcs(reinterpret_cast<const double2*>(p + kStep * h));
                    a[u][2 * h] = w.x, a[u][2 * h + 1] = w.y;
                }
            }
            b[u] = (col_ok && rhs_ok) ? __ldg(xg + c) : 0.;
        }
    };
    auto mma = [&](const T (&a)[kU][8], const double (&b)[kU]) {
#pragma unroll
        for (int u = 0; u < kU; u++)
#pragma unroll
            for (int rt = 0; rt < 8; rt++)
                mma_884(acc[rt][0], acc[rt][1], (double) a[u][rt], b[u]);
    };
    if (rowbase < n) {
        if constexpr (kPipelined) {
            // two register stages (a stage past e1 loads zeros and adds nothing)
            T a0[kU][8], a1[kU][8];
            double b0[kU], b1[kU];
            load(a0, b0, e0);
            for (int c0 = e0; c0 < e1; c0 += 8 * kU) {
                load(a1, b1, c0 + 4 * kU);
                mma(a0, b0);
                load(a0, b0, c0 + 8 * kU);
                mma(a1, b1);
            }
        }
        else {
            for (int c0 = e0; c0 < e1; c0 += 4 * kU) {
                T a[kU][8];
                double b[kU];
                load(a, b, c0);
                mma(a, b);
            }
        }
    }
#pragma unroll
    for (int rt = 0; rt < 8; rt++) {
        const int i = r0 + kStep * (rt / kPer) + rt % kPer;  // increasing in rt
        if (i >= n)
            break;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int r = 2 * t + h;
            if (r < nrhs) {
                if (partial)
                    partial[((size_t) blockIdx.y * nrhs + r) * n + i] = acc[rt][h];
                else
                    y[(size_t) r * n + i] = acc[rt][h];
            }
        }
    }
}

}  // namespace kemcu

namespace kemcu
{
// ------------------------------------------------------------------------- point ordering
// Points are evaluated in Morton (Z-curve) order so that the 32 points of a warp are close
// together and take the same quadrature band for almost every element: the band branch is
// then warp-uniform. The permutation is applied on the device and undone on the results.

__device__ __forceinline__ unsigned long long spread3(unsigned v)
{
    unsigned long long x = v & 0x1fffffu;
    x = (x | x << 32) & 0x1f00000000ffffULL;
    x = (x | x << 16) & 0x1f0000ff0000ffULL;
    x = (x | x << 8) & 0x100f00f00f00f00fULL;
    x = (x | x << 4) & 0x10c30c30c30c30c3ULL;
    x = (x | x << 2) & 0x1249249249249249ULL;
    return x;
}

// bounding box: box[0..2] = min, box[3..5] = max; partial[gridDim.x][6]; last block reduces
__global__ void bbox_kernel(const double* __restrict__ P, int n, double* __restrict__ partial,
                            unsigned* __restrict__ counter, double* __restrict__ box)
{
    __shared__ double sh[6][256];
    __shared__ bool last;
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (int c = 0; c < 3; c++) {
            const double v = P[3 * i + c];
            lo[c] = fmin(lo[c], v);
            hi[c] = fmax(hi[c], v);
        }
    for (int c = 0; c < 3; c++) {
        sh[c][threadIdx.x] = lo[c];
        sh[3 + c][threadIdx.x] = hi[c];
    }
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s)
            for (int c = 0; c < 3; c++) {
                sh[c][threadIdx.x] = fmin(sh[c][threadIdx.x], sh[c][threadIdx.x + s]);
                sh[3 + c][threadIdx.x] = fmax(sh[3 + c][threadIdx.x], sh[3 + c][threadIdx.x + s]);
            }
        __syncthreads();
    }
    if (threadIdx.x < 6)
        partial[blockIdx.x * 6 + threadIdx.x] = sh[threadIdx.x][0];
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0)
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last)
        return;
    __threadfence();
    if (threadIdx.x < 6) {
        double v = threadIdx.x < 3 ? 1e300 : -1e300;
        for (int b = 0; b < (int) gridDim.x; b++) {
            const double q = __ldcg(partial + b * 6 + threadIdx.x);
            v = threadIdx.x < 3 ? fmin(v, q) : fmax(v, q);
        }
        box[threadIdx.x] = v;
    }
    if (threadIdx.x == 0)
        *counter = 0u;
}

__global__ void morton_kernel(const double* __restrict__ P, int n, const double* __restrict__ box,
                              unsigned long long* __restrict__ key, int* __restrict__ idx)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    unsigned q[3];
    for (int c = 0; c < 3; c++) {
        const double ext = box[3 + c] - box[c];
        const double t = ext > 0. ? (P[3 * i + c] - box[c]) / ext : 0.;
        q[c] = (unsigned) fmin(fmax(t * 2097151.0, 0.), 2097151.0);
    }
    key[i] = spread3(q[0]) | (spread3(q[1]) << 1) | (spread3(q[2]) << 2);
    idx[i] = i;
}

// Morton keys in the meridian plane (r, z) for axisymmetric models: the work of a point depends
// on its (r, z) only, so points of one warp that are close in (r, z) run the same ring
// evaluations. r is scaled over [0, r_max] with r_max the corner of the bounding box's x-y
// rectangle farthest from the axis.
__device__ __forceinline__ unsigned long long spread2(unsigned v)
{
    unsigned long long x = v;
    x = (x | x << 16) & 0x0000ffff0000ffffULL;
    x = (x | x << 8) & 0x00ff00ff00ff00ffULL;
    x = (x | x << 4) & 0x0f0f0f0f0f0f0f0fULL;
    x = (x | x << 2) & 0x3333333333333333ULL;
    x = (x | x << 1) & 0x5555555555555555ULL;
    return x;
}

__global__ void morton_rz_kernel(const double* __restrict__ P, int n, const double* __restrict__ box,
                                 unsigned long long* __restrict__ key, int* __restrict__ idx)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const double xm = fmax(fabs(box[0]), fabs(box[3])), ym = fmax(fabs(box[1]), fabs(box[4]));
    const double rmax = sqrt(xm * xm + ym * ym), zext = box[5] - box[2];
    const double r = sqrt(P[3 * i] * P[3 * i] + P[3 * i + 1] * P[3 * i + 1]);
    const double tr = rmax > 0. ? r / rmax : 0., tz = zext > 0. ? (P[3 * i + 2] - box[2]) / zext : 0.;
    const unsigned qr = (unsigned) fmin(fmax(tr * 2147483647.0, 0.), 2147483647.0);
    const unsigned qz = (unsigned) fmin(fmax(tz * 2147483647.0, 0.), 2147483647.0);
    key[i] = spread2(qr) | (spread2(qz) << 1);
    idx[i] = i;
}

__global__ void gather_points_kernel(const double* __restrict__ P, const int* __restrict__ perm, int n,
                                     double* __restrict__ Q)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const int j = perm[i];
    Q[3 * i] = P[3 * j];
    Q[3 * i + 1] = P[3 * j + 1];
    Q[3 * i + 2] = P[3 * j + 2];
}

__global__ void scatter_out_kernel(const double* __restrict__ src, const int* __restrict__ perm, int n,
                                   double* __restrict__ dst)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const int j = perm[i];
    // scalar stores: dst may be a caller's device pointer with only 8-byte alignment
    dst[4 * (size_t) j] = src[4 * (size_t) i];
    dst[4 * (size_t) j + 1] = src[4 * (size_t) i + 1];
    dst[4 * (size_t) j + 2] = src[4 * (size_t) i + 2];
    dst[4 * (size_t) j + 3] = src[4 * (size_t) i + 3];
}
}  // namespace kemcu

namespace kemcu
{
// ------------------------------------------------------------------------- diagnostics
// band histogram over all (element, point) pairs: counts[shape * 4 + band]
__global__ void band_histogram_kernel(const double* __restrict__ rec, int n_elem, const double* __restrict__ pts,
                                      int n_pts, unsigned long long* __restrict__ counts)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned c[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (p < n_pts) {
        const V3 P = v3(pts[3 * p], pts[3 * p + 1], pts[3 * p + 2]);
        for (int j = 0; j < n_elem; j++) {
            const double* e = rec + (size_t) j * rRecSize;
            c[(int) e[rType] * 4 + band_of(e, P)]++;
        }
    }
    for (int k = 0; k < 12; k++) {
        unsigned v = c[k];
        for (int o = 16; o > 0; o >>= 1)
            v += __shfl_down_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0 && v)
            atomicAdd(counts + k, (unsigned long long) v);
    }
}

// FMA throughput probe: kProbeChains independent dependent chains per thread
constexpr int kProbeChains = 8;
template<typename T> __global__ void fma_probe_kernel(T* __restrict__ sink, int iters)
{
    T a[kProbeChains];
    const T x = (T) 0.999999, y = (T) 1e-7;
#pragma unroll
    for (int k = 0; k < kProbeChains; k++)
        a[k] = (T) (threadIdx.x + k);
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < kProbeChains; k++)
            a[k] = fma(a[k], x, y);
    }
    T s = 0;
#pragma unroll
    for (int k = 0; k < kProbeChains; k++)
        s += a[k];
    if (s == (T) -1)  // never true; keeps the chains alive
        sink[threadIdx.x] = s;
}
}  // namespace kemcu
