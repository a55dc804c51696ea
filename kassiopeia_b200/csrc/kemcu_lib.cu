// libkemcu: host side of the C ABI declared in include/kemcu.h.
//
// One translation unit so the __constant__ rule tables are shared by every kernel without
// relocatable device code. Host code here is C++17; nothing crosses the ABI but plain types.

#include "kemcu.h"
#include "kemcu_device.cuh"
#include "kemcu_kernels.cuh"
#include "kemcu_axisym.cuh"
#include "kemcu_solver.cuh"
#include "kemcu_tables.cuh"
#include "kemcu_track.cuh"
#include "kemcu_adjoint.cuh"
#include "kemcu_robinhood.cuh"
#include "kemcu_fftm.cuh"

#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

using namespace kemcu;

// Scratch of kemcu_field_dev_noalloc: a fixed device array instead of cudaMalloc'd memory. In
// host code this name is only a host-side stand-in; the device address is obtained with
// cudaGetSymbolAddress in kemcu_create (kemcu_ctx::noalloc_scratch).
static __device__ __align__(256) double g_noalloc_scratch[KEMCU_NOALLOC_SCRATCH_BYTES / sizeof(double)];

// ------------------------------------------------------------------------------- context
struct DevBuf
{
    void* p = nullptr;
    size_t bytes = 0;
};

struct FmState;  // fast multipole tree and buffers (kemcu_fftm_host.inc)

struct kemcu_ctx
{
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int num_sms = 0;
    Constants k{};
    size_t assembled_budget = 0;
    std::string err;
    double last_ms = 0.;
    // geometry
    size_t n = 0;
    std::vector<double> h_rec;         // n x 32 element records
    std::vector<TargetRec> h_tgt;      // n matrix-row targets
    std::vector<double> h_rhs;         // boundary values
    std::vector<int32_t> h_shape;
    double* d_rec = nullptr;
    TargetRec* d_tgt = nullptr;
    double* d_sigma = nullptr;
    bool have_sigma = false;
    // all elements axisymmetric (conic sections, rings): records in the AxRec layout
    bool axisym = false;
    // assembled operator (column-major)
    double* d_a64 = nullptr;
    float* d_a32 = nullptr;
    // near-field list of the operator's columns (matrix-free Robin Hood), built on first use
    long long* d_near_ptr = nullptr;
    int* d_near_row = nullptr;
    double* d_near_val = nullptr;
    // grow-only scratch
    DevBuf scratch[16];
    unsigned* d_counter = nullptr;
    int* d_flag = nullptr;
    double* noalloc_scratch = nullptr;  // device address of g_noalloc_scratch on this context's device
    kemcu_iteration_callback cb = nullptr;
    void* cb_user = nullptr;
    unsigned long long launches = 0;
    // autotuner of the direct sum (field_variants): per (precision, size class) the chosen
    // variant, or the K1 times of the variants tried so far; a call that times a variant
    // leaves its key and variant pending until its result is back
    bool autotune = true;
    std::map<int, int> tuned;
    std::map<int, std::vector<float>> explored;
    int force_variant = -1;
    bool time_k1 = false;  // time the K1 launch of forced variants (kemcu_tune_field)
    int pending_key = -1, pending_variant = -1;
    cudaEvent_t tv0 = nullptr, tv1 = nullptr;
    FmState* fm = nullptr;  // the fast multipole tree of the current geometry (kemcu_fftm_configure)
    FmState* fm_pre = nullptr;  // the preconditioner's tree (kemcu_fftm_configure_preconditioner)
};

void fm_release(kemcu_ctx* ctx);
int fm_apply(kemcu_ctx* ctx, FmState* S, const double* d_x, double* d_y, int nrhs);

namespace
{
enum Scratch
{
    sPts = 0,
    sOut,
    sPartial,
    sVec0,
    sVec1,
    sVec2,
    sBasis,
    sMisc,
    sSort,  // Morton-ordering workspace of kemcu_field_dev (never aliases a caller's staging slot)
    sZ,     // preconditioned Krylov basis (flexible GMRES) or the Jacobi-scaled vector
    sKry,   // BiCGStab vectors
    sInBasis, sInW, sInMisc, sInK,  // the inner GMRES of the implicit Krylov preconditioner
    kNumScratch
};
static_assert(kNumScratch <= 16, "kemcu_ctx::scratch holds 16 slots");

int fail(kemcu_ctx* c, int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (c)
        c->err = buf;
    return code;
}

#define KC(call)                                                                                        \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess)                                                                          \
            return fail(ctx, KEMCU_ECUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
                        __LINE__);                                                                      \
    } while (0)

// every launch of this library's own kernels is followed by KCHECK_LAUNCH, which also counts it
#define KCHECK_LAUNCH()      \
    do {                     \
        ctx->launches++;     \
        KC(cudaGetLastError()); \
    } while (0)

int ensure(kemcu_ctx* ctx, int slot, size_t bytes, void** out)
{
    DevBuf& b = ctx->scratch[slot];
    if (b.bytes < bytes) {
        if (b.p)
            KC(cudaFree(b.p));
        b.p = nullptr;
        b.bytes = 0;
        const size_t want = std::max(bytes, (size_t) 256);
        if (cudaMalloc(&b.p, want) != cudaSuccess) {
            cudaGetLastError();
            return fail(ctx, KEMCU_ENOMEM, "device allocation of %zu bytes failed", want);
        }
        b.bytes = want;
    }
    *out = b.p;
    return KEMCU_OK;
}

// element record and matrix-row target of one element, in the reference's FP64 operation
// order (no FMA: the host compiler targets baseline x86-64)
// axisymmetric element record (AxRec). Caller layout: conic section geom = (r0, z0, r1, z1),
// ring geom = (r, z) (KConicSection.hh: P0 = (r0, 0, z0), P1 = (r1, 0, z1); KRing.hh: P = (r, 0, z)).
// Prefactors and the centroid as KElectrostaticAnalyticConicSectionIntegrator.cc:91,
// KElectrostaticAnalyticRingIntegrator.cc:36 and KConicSection.hh:29-32 / KRing.hh:29-32 form them.
static_assert((int) aRecUsed <= (int) rRecSize, "the axisymmetric record must fit the element record slot");

void build_axisym_record(const double* g, int shape, double value, const Constants& K, double* r, double& rhs)
{
    if (shape == KEMCU_RING) {
        r[aType] = kAxRing;
        r[aZa] = r[aZb] = g[1];
        r[aRa] = r[aRb] = g[0];
        r[aLen] = 1.;
        r[aPre] = 1. / (g[0] * 2. * K.pi * K.pi * K.eps0);
        r[aCx] = g[0];
        r[aCz] = g[1];
    }
    else {
        r[aType] = kAxConic;
        r[aZa] = g[1];
        r[aRa] = g[0];
        r[aZb] = g[3];
        r[aRb] = g[2];
        const double dx = g[0] - g[2], dz = g[1] - g[3];
        r[aLen] = sqrt(dx * dx + 0. * 0. + dz * dz);
        r[aPre] = 1. / (K.pi * K.eps0);
        r[aCx] = (g[0] + g[2]) * .5;
        r[aCz] = (g[1] + g[3]) * .5;
    }
    r[aCy] = 0.;
    rhs = value;
}

void build_record(const double* g, int shape, int boundary, double value, const Constants& K, double* r,
                  TargetRec& t, double& rhs)
{
    for (int i = 0; i < rRecSize; i++)
        r[i] = 0.;
    r[rType] = (double) shape;
    if (shape == kLineSegment) {
        const double d0 = g[3] - g[0], d1 = g[4] - g[1], d2 = g[5] - g[2];
        const double len = std::sqrt((d0 * d0) + (d1 * d1) + (d2 * d2));
        r[rA] = len;
        r[rB] = g[6];
        for (int c = 0; c < 3; c++) {
            r[rP0 + c] = g[c];
            r[rN1 + c] = g[3 + c];
            r[rEa + c] = g[3 + c] - g[c];
            r[rCen + c] = (g[c] + g[3 + c]) * 0.5;
            r[rCen2 + c] = r[rCen + c];
        }
        r[rInvSize] = 1. / len;
        r[rPrefac] = g[6] / (4. * K.eps0);
        // KLineSegment::Normal() (KLineSegment.cc:27-33)
        double nx, ny, nz;
        if (d0 > 1.e-10) {  // d x (1,0,0)
            nx = 0.;
            ny = d2;
            nz = -d1;
        }
        else {  // d x (0,1,0)
            nx = -d2;
            ny = 0.;
            nz = d0;
        }
        const double m = std::sqrt(nx * nx + ny * ny + nz * nz);
        t.normal[0] = nx / m;
        t.normal[1] = ny / m;
        t.normal[2] = nz / m;
    }
    else {
        const double A = g[0], B = g[1];
        for (int i = 0; i < 11; i++)
            r[i] = g[i];
        for (int c = 0; c < 3; c++) {
            r[rEa + c] = A * g[5 + c];
            r[rEb + c] = B * g[8 + c];
        }
        const double cx = g[6] * g[10] - g[7] * g[9], cy = g[7] * g[8] - g[5] * g[10], cz = g[5] * g[9] - g[6] * g[8];
        const double cm = std::sqrt((cx * cx) + (cy * cy) + (cz * cz));
        const double n3[3] = {cx * (1. / cm), cy * (1. / cm), cz * (1. / cm)};
        // quadratic-form coefficients of the squared node distances
        r[rAA] = r[rEa] * r[rEa] + r[rEa + 1] * r[rEa + 1] + r[rEa + 2] * r[rEa + 2];
        r[rAB2] = 2. * (r[rEa] * r[rEb] + r[rEa + 1] * r[rEb + 1] + r[rEa + 2] * r[rEb + 2]);
        r[rBB] = r[rEb] * r[rEb] + r[rEb + 1] * r[rEb + 1] + r[rEb + 2] * r[rEb + 2];
        if (shape == kTriangle) {
            double p1[3], p2[3];
            for (int c = 0; c < 3; c++) {
                p1[c] = g[2 + c] + (A * g[5 + c]);
                p2[c] = g[2 + c] + (B * g[8 + c]);
                r[rCen + c] = g[2 + c] + (A * g[5 + c] + B * g[8 + c]) / 3.;
                r[rCen2 + c] = r[rCen + c];
            }
            const double l12 = std::sqrt(((p2[0] - p1[0]) * (p2[0] - p1[0])) + ((p2[1] - p1[1]) * (p2[1] - p1[1])) +
                                         ((p2[2] - p1[2]) * (p2[2] - p1[2])));
            const double size = (A + B + l12) / 3.;
            r[rInvSize] = 1. / size;
            r[rPrefac] = 0.5 * A * B * cm * K.one_over_four_pi_eps0;
            for (int c = 0; c < 3; c++)
                t.normal[c] = n3[c];
        }
        else {
            for (int c = 0; c < 3; c++) {
                r[rCen + c] = g[2 + c] + 0.5 * (A * g[5 + c] + B * g[8 + c]);
                r[rCen2 + c] = (g[2 + c] + A * g[5 + c] * .5) + B * g[8 + c] * .5;
            }
            const double size = 0.5 * (A + B);
            r[rInvSize] = 1. / size;
            r[rPrefac] = A * B * K.one_over_four_pi_eps0;
            // KRectangle::Normal() returns N1 x N2 unnormalised (KRectangle.cc:7-16)
            t.normal[0] = cx;
            t.normal[1] = cy;
            t.normal[2] = cz;
        }
    }
    // squared band cut distances (ratio = |P - c| / size); ambiguous cases are resolved
    // on the device with the reference's exact expression
    const double tri_cut[3] = {3.42, 30.4, 131.4}, rect_cut[3] = {4.6, 44.6, 196.2}, line_cut[3] = {2., 27.7, 1e300};
    const double* cut = shape == kTriangle ? tri_cut : shape == kRectangle ? rect_cut : line_cut;
    for (int k = 0; k < 3; k++) {
        const double dcut = cut[k] / r[rInvSize];
        r[rCut + k] = cut[k] > 1e299 ? 1e300 : dcut * dcut;
    }
    for (int c = 0; c < 3; c++)
        t.cen[c] = r[rCen2 + c];
    t.neumann = boundary == KEMCU_NEUMANN ? 1. : 0.;
    t.diag = boundary == KEMCU_NEUMANN ? ((1. + value) / (1. - value)) / (2. * K.eps0) : 0.;
    rhs = boundary == KEMCU_NEUMANN ? 0. : value;
}

// the direct-sum kernels OR 2 into d_flag[1] when an element-pipeline wait times out; a
// public call clears the word before its first such launch and reads it when it is done
int clear_pipe_flag(kemcu_ctx* ctx)
{
    KC(cudaMemsetAsync(ctx->d_flag + 1, 0, sizeof(int), ctx->stream));
    return KEMCU_OK;
}

int pipe_status(kemcu_ctx* ctx, const char* what)
{
    int f = 0;
    KC(cudaMemcpyAsync(&f, ctx->d_flag + 1, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    KC(cudaStreamSynchronize(ctx->stream));
    if (f)
        return fail(ctx, KEMCU_ETIMEOUT, "element pipeline wait timed out while computing the %s", what);
    return KEMCU_OK;
}

int grid_split(const kemcu_ctx* ctx, size_t n_pts, size_t n_elem)
{
    // enough CTAs for four waves of the resident CTAs per SM, each split keeping >= 32 elements
    const size_t blocks = (n_pts + kThreads - 1) / kThreads;
    const size_t want = (size_t) ctx->num_sms * kMinBlocks * 4;
    size_t split = blocks >= want ? 1 : (want + blocks - 1) / blocks;
    split = std::min(split, std::max((size_t) 1, n_elem / 32));
    split = std::min(split, (size_t) 65535);
    return (int) std::max((size_t) 1, split);
}

// axisymmetric elements: FP64 element integrals whatever the precision argument. The element
// range is split over gridDim.y (axisym_split), partial sums in `scratch` (n x 4 x split
// doubles, capped at `scratch_cap` doubles; null: grow-only scratch of the context)
int launch_axisym_field(kemcu_ctx* ctx, const double* d_pts, size_t n, double* d_out, int what,
                        double* scratch = nullptr, size_t scratch_cap = 0)
{
    const int ne = (int) ctx->n, np = (int) n;
    int split = axisym_split(ctx->num_sms, n, ctx->n);
    double* partial = nullptr;
    if (scratch)
        split = (int) std::min((size_t) split, std::max((size_t) 1, scratch_cap / (4 * n)));
    if (split > 1) {
        if (scratch)
            partial = scratch;
        else {
            void* p;
            if (int rc = ensure(ctx, sPartial, (size_t) split * n * 4 * sizeof(double), &p))
                return rc;
            partial = (double*) p;
        }
    }
    const dim3 grid((unsigned) ((n + kAxThreads - 1) / kAxThreads), (unsigned) split);
    if (what == KEMCU_POTENTIAL)
        axisym_field_kernel<true, false><<<grid, kAxThreads, 0, ctx->stream>>>(ctx->d_rec, rRecSize, ctx->d_sigma, ne,
                                                                               d_pts, np, d_out, partial);
    else if (what == KEMCU_FIELD)
        axisym_field_kernel<false, true><<<grid, kAxThreads, 0, ctx->stream>>>(ctx->d_rec, rRecSize, ctx->d_sigma, ne,
                                                                               d_pts, np, d_out, partial);
    else
        axisym_field_kernel<true, true><<<grid, kAxThreads, 0, ctx->stream>>>(ctx->d_rec, rRecSize, ctx->d_sigma, ne,
                                                                              d_pts, np, d_out, partial);
    KCHECK_LAUNCH();
    if (split > 1) {
        const size_t m = n * 4;
        reduce_splits<<<(unsigned) ((m + 255) / 256), 256, 0, ctx->stream>>>(partial, split, m, d_out);
        KCHECK_LAUNCH();
    }
    return KEMCU_OK;
}

// Launch shapes of K1 the autotuner chooses between: (resident CTAs per SM the registers are
// bounded for, ring stages), the build default first. They change no operation and no order of
// summation, so every variant returns the same bits; only the field-and-potential kernels (the
// path of field evaluation and tracking at scale) are instantiated in every shape.
struct FieldVariant
{
    int min_blocks, ring_stages;
};
constexpr FieldVariant kFieldVariants[] = {{kMinBlocks, kPipe}, {4, 4}, {5, 3}, {4, 3}};
constexpr int kNumFieldVariants = (int) (sizeof(kFieldVariants) / sizeof(kFieldVariants[0]));

template<bool MIXED, bool POT, bool FIELD>
void launch_k1(int variant, dim3 grid, cudaStream_t st, const double* rec, const double* sg, int ne, const double* pts,
               int np, double* out, double* part, int* fl)
{
    if constexpr (POT && FIELD) {
        switch (variant) {
        case 1:
            field_kernel<MIXED, POT, FIELD, 4, 4><<<grid, kThreads, 0, st>>>(rec, sg, ne, pts, np, out, part, fl);
            return;
        case 2:
            field_kernel<MIXED, POT, FIELD, 5, 3><<<grid, kThreads, 0, st>>>(rec, sg, ne, pts, np, out, part, fl);
            return;
        case 3:
            field_kernel<MIXED, POT, FIELD, 4, 3><<<grid, kThreads, 0, st>>>(rec, sg, ne, pts, np, out, part, fl);
            return;
        default:
            break;
        }
    }
    field_kernel<MIXED, POT, FIELD><<<grid, kThreads, 0, st>>>(rec, sg, ne, pts, np, out, part, fl);
}

// tuning key: precision and the size class (bit length of the point count)
int tune_key(int precision, size_t n)
{
    int c = 0;
    while ((n >> c) > 1)
        c++;
    return precision * 64 + c;
}

// the K1 variant of a planar field-and-potential call of n points; marks the call for timing
// when the autotuner still explores this size class
int choose_variant(kemcu_ctx* ctx, size_t n, int precision, int what)
{
    ctx->pending_key = -1;
    if (what != KEMCU_FIELD_AND_POTENTIAL || precision == KEMCU_FP32)
        return 0;  // one launch shape outside the field-and-potential kernels of FP64 and MIXED
    if (ctx->force_variant >= 0)
        return ctx->force_variant;
    const int key = tune_key(precision, n);
    auto it = ctx->tuned.find(key);
    if (it != ctx->tuned.end())
        return it->second;
    if (!ctx->autotune)
        return 0;
    ctx->pending_key = key;
    ctx->pending_variant = (int) ctx->explored[key].size();
    return ctx->pending_variant;
}

// after a timed call's result is complete: record its K1 time; once every variant has run for
// the size class, keep the fastest
void finish_variant(kemcu_ctx* ctx)
{
    if (ctx->pending_key < 0)
        return;
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, ctx->tv0, ctx->tv1) == cudaSuccess) {
        auto& t = ctx->explored[ctx->pending_key];
        if ((int) t.size() == ctx->pending_variant)
            t.push_back(ms);
        if ((int) t.size() == kNumFieldVariants)
            ctx->tuned[ctx->pending_key] = (int) (std::min_element(t.begin(), t.end()) - t.begin());
    }
    else
        cudaGetLastError();
    ctx->pending_key = -1;
}

// the planar direct sum at device points (d_out n x 4): K1, split `split` ways over the element
// list (partial sums in `partial`, then reduced in split order)
int launch_planar_field(kemcu_ctx* ctx, const double* d_pts, size_t n, double* d_out, int precision, int what,
                        int split, double* partial)
{
    dim3 grid((unsigned) ((n + kThreads - 1) / kThreads), (unsigned) split);
    if (int rc = clear_pipe_flag(ctx))
        return rc;
    const bool mixed = precision == KEMCU_MIXED;
    const double* sg = ctx->d_sigma;
    const int ne = (int) ctx->n, np = (int) n;
    double* part = split > 1 ? partial : nullptr;
    int* fl = ctx->d_flag + 1;
    const int v = choose_variant(ctx, n, precision, what);
    cudaStream_t st = ctx->stream;
    const bool timed = ctx->pending_key >= 0 || ctx->time_k1;
    if (timed)
        KC(cudaEventRecord(ctx->tv0, st));
    if (precision == KEMCU_FP32) {
        const double* r = ctx->d_rec;
        if (what == KEMCU_POTENTIAL)
            field_kernel<false, true, false, kMinBlocks, kPipe, true><<<grid, kThreads, 0, st>>>(r, sg, ne, d_pts, np, d_out, part, fl);
        else if (what == KEMCU_FIELD)
            field_kernel<false, false, true, kMinBlocks, kPipe, true><<<grid, kThreads, 0, st>>>(r, sg, ne, d_pts, np, d_out, part, fl);
        else
            field_kernel<false, true, true, kMinBlocks, kPipe, true><<<grid, kThreads, 0, st>>>(r, sg, ne, d_pts, np, d_out, part, fl);
    }
    else if (what == KEMCU_POTENTIAL) {
        if (mixed)
            launch_k1<true, true, false>(v, grid, st, ctx->d_rec, sg, ne, d_pts, np, d_out, part, fl);
        else
            launch_k1<false, true, false>(v, grid, st, ctx->d_rec, sg, ne, d_pts, np, d_out, part, fl);
    }
    else if (what == KEMCU_FIELD) {
        if (mixed)
            launch_k1<true, false, true>(v, grid, st, ctx->d_rec, sg, ne, d_pts, np, d_out, part, fl);
        else
            launch_k1<false, false, true>(v, grid, st, ctx->d_rec, sg, ne, d_pts, np, d_out, part, fl);
    }
    else {
        if (mixed)
            launch_k1<true, true, true>(v, grid, st, ctx->d_rec, sg, ne, d_pts, np, d_out, part, fl);
        else
            launch_k1<false, true, true>(v, grid, st, ctx->d_rec, sg, ne, d_pts, np, d_out, part, fl);
    }
    KCHECK_LAUNCH();
    if (timed)
        KC(cudaEventRecord(ctx->tv1, st));
    if (split > 1) {
        const size_t m = n * 4;
        reduce_splits<<<(unsigned) ((m + 255) / 256), 256, 0, ctx->stream>>>(part, split, m, d_out);
        KCHECK_LAUNCH();
    }
    return KEMCU_OK;
}

// field at device points; d_out n x 4
int launch_field(kemcu_ctx* ctx, const double* d_pts, size_t n, double* d_out, int precision, int what)
{
    if (ctx->axisym)
        return launch_axisym_field(ctx, d_pts, n, d_out, what);
    const int split = grid_split(ctx, n, ctx->n);
    double* partial = nullptr;
    if (split > 1) {
        void* p;
        int rc = ensure(ctx, sPartial, (size_t) split * n * 4 * sizeof(double), &p);
        if (rc)
            return rc;
        partial = (double*) p;
    }
    return launch_planar_field(ctx, d_pts, n, d_out, precision, what, split, partial);
}

constexpr size_t kSortMin = 4096;  // below this the point set is evaluated in caller order

size_t cub_sort_bytes(size_t n)
{
    size_t b = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, b, (const unsigned long long*) nullptr, (unsigned long long*) nullptr,
                                    (const int*) nullptr, (int*) nullptr, (int) n, 0, 63);
    return b;
}

int check_finite(kemcu_ctx* ctx, const double* d, size_t m, const char* what)
{
    KC(cudaMemsetAsync(ctx->d_flag, 0, sizeof(int), ctx->stream));
    finite_kernel<<<(unsigned) ((m + 255) / 256), 256, 0, ctx->stream>>>(d, m, ctx->d_flag);
    KCHECK_LAUNCH();
    int flag[2] = {0, 0};
    KC(cudaMemcpyAsync(flag, ctx->d_flag, 2 * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    KC(cudaStreamSynchronize(ctx->stream));
    if (flag[1])
        return fail(ctx, KEMCU_ETIMEOUT, "element pipeline wait timed out while computing the %s", what);
    if (flag[0])
        return fail(ctx, KEMCU_ENONFINITE, "%s contains NaN or Inf", what);
    return KEMCU_OK;
}

int check_ready(kemcu_ctx* ctx, bool need_sigma)
{
    if (!ctx)
        return KEMCU_EINVAL;
    if (ctx->n == 0)
        return fail(ctx, KEMCU_ESTATE, "no geometry set");
    if (need_sigma && !ctx->have_sigma)
        return fail(ctx, KEMCU_ESTATE, "no charge densities set (kemcu_set_sigma or kemcu_gmres first)");
    return KEMCU_OK;
}

// entry points whose kernels take planar elements only (triangles, rectangles, wires)
int planar_only(kemcu_ctx* ctx, const char* what)
{
    if (ctx->axisym)
        return fail(ctx, KEMCU_EINVAL, "%s is not available for axisymmetric elements (conic sections, rings)", what);
    return KEMCU_OK;
}

struct Timer
{
    kemcu_ctx* ctx;
    explicit Timer(kemcu_ctx* c) : ctx(c)
    {
        cudaEventRecord(ctx->ev0, ctx->stream);
    }
    void stop()
    {
        cudaEventRecord(ctx->ev1, ctx->stream);
        cudaEventSynchronize(ctx->ev1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
        ctx->last_ms = ms;
    }
};

// ------------------------------------------------------------------------------- operators
enum OpKind
{
    kFree64 = 0,
    kFreeMixed,
    kDense64,
    kDense32,
    kFree32,  // matrix-free with the FP32 far-field form
    kFftm,    // the fast multipole operator (kemcu_fftm_configure)
    kFftmPre  // the preconditioner's fast multipole operator (kemcu_fftm_configure_preconditioner)
};

int apply_op(kemcu_ctx* ctx, int op, const double* d_x, double* d_y, int nrhs)
{
    const int n = (int) ctx->n;
    if (op == kFftm || op == kFftmPre)
        return fm_apply(ctx, op == kFftm ? ctx->fm : ctx->fm_pre, d_x, d_y, nrhs);
    if ((op == kFree64 || op == kFreeMixed || op == kFree32) && ctx->axisym) {
        const int split = axisym_split(ctx->num_sms, n, n);
        double* partial = nullptr;
        if (split > 1) {
            void* p;
            if (int rc = ensure(ctx, sPartial, (size_t) split * nrhs * n * sizeof(double), &p))
                return rc;
            partial = (double*) p;
        }
        const dim3 grid((unsigned) ((n + kAxThreads - 1) / kAxThreads), (unsigned) split);
        if (nrhs == 1)
            axisym_matvec_kernel<1><<<grid, kAxThreads, 0, ctx->stream>>>(ctx->d_rec, rRecSize, n, d_x, nrhs, d_y,
                                                                          partial);
        else
            axisym_matvec_kernel<kMaxRhs><<<grid, kAxThreads, 0, ctx->stream>>>(ctx->d_rec, rRecSize, n, d_x, nrhs,
                                                                                d_y, partial);
        KCHECK_LAUNCH();
        if (split > 1) {
            const size_t m = (size_t) nrhs * n;
            reduce_splits<<<(unsigned) ((m + 255) / 256), 256, 0, ctx->stream>>>(partial, split, m, d_y);
            KCHECK_LAUNCH();
        }
        return KEMCU_OK;
    }
    if (op == kFree64 || op == kFreeMixed || op == kFree32) {
        const int split = grid_split(ctx, n, n);
        double* partial = nullptr;
        if (split > 1) {
            void* p;
            int rc = ensure(ctx, sPartial, (size_t) split * nrhs * n * sizeof(double), &p);
            if (rc)
                return rc;
            partial = (double*) p;
        }
        dim3 grid((n + kThreads - 1) / kThreads, split);
        int* fl = ctx->d_flag + 1;
        if (op == kFree32) {
            if (nrhs == 1)
                matvec_kernel<false, 1, true><<<grid, kThreads, 0, ctx->stream>>>(ctx->d_rec, ctx->d_tgt, n, d_x, nrhs, d_y,
                                                                                partial, fl);
            else
                matvec_kernel<false, kMaxRhs, true><<<grid, kThreads, 0, ctx->stream>>>(ctx->d_rec, ctx->d_tgt, n, d_x, nrhs,
                                                                                      d_y, partial, fl);
        }
        else if (op == kFree64) {
            if (nrhs == 1)
                matvec_kernel<false, 1><<<grid, kThreads, 0, ctx->stream>>>(ctx->d_rec, ctx->d_tgt, n, d_x, nrhs, d_y, partial, fl);
            else
                matvec_kernel<false, kMaxRhs><<<grid, kThreads, 0, ctx->stream>>>(ctx->d_rec, ctx->d_tgt, n, d_x, nrhs, d_y,
                                                                                  partial, fl);
        }
        else {
            if (nrhs == 1)
                matvec_kernel<true, 1><<<grid, kThreads, 0, ctx->stream>>>(ctx->d_rec, ctx->d_tgt, n, d_x, nrhs, d_y, partial, fl);
            else
                matvec_kernel<true, kMaxRhs><<<grid, kThreads, 0, ctx->stream>>>(ctx->d_rec, ctx->d_tgt, n, d_x, nrhs, d_y,
                                                                                 partial, fl);
        }
        KCHECK_LAUNCH();
        if (split > 1) {
            const size_t m = (size_t) nrhs * n;
            reduce_splits<<<(unsigned) ((m + 255) / 256), 256, 0, ctx->stream>>>(partial, split, m, d_y);
            KCHECK_LAUNCH();
        }
        return KEMCU_OK;
    }
    // dense operator: 256 V rows per CTA; the column range is split S ways. Every CTA does the
    // same work, so the time goes as waves / S with waves = ceil(rows_blocks S / resident CTAs):
    // S is the smallest split that minimises it (up to 128 ways), which fills the GPU whether the
    // row blocks are fewer or more than one wave
    auto launch = [&](auto kernel, const auto* A, int V) -> int {
        const size_t rows_blocks = (n + 256 * (size_t) V - 1) / (256 * (size_t) V);
        int per_sm = 0;
        KC(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 256, 0));
        const size_t resident = (size_t) ctx->num_sms * std::max(1, per_sm);
        const size_t max_split = std::min((size_t) 128, (size_t) std::max(1, n / 256));
        size_t split = 1;
        double best = 1e300;
        for (size_t s = 1; s <= max_split; s++) {
            const double cost = (double) ((rows_blocks * s + resident - 1) / resident) / (double) s;
            if (cost < best * (1. - 1e-9)) {
                best = cost;
                split = s;
            }
        }
        double* partial = nullptr;
        if (split > 1) {
            void* p;
            int rc = ensure(ctx, sPartial, split * nrhs * n * sizeof(double), &p);
            if (rc)
                return rc;
            partial = (double*) p;
        }
        dim3 grid((unsigned) rows_blocks, (unsigned) split);
        kernel<<<grid, 256, 0, ctx->stream>>>(A, n, op_ld(n), d_x, nrhs, d_y, partial);
        KCHECK_LAUNCH();
        if (split > 1) {
            const size_t m = (size_t) nrhs * n;
            reduce_splits<<<(unsigned) ((m + 255) / 256), 256, 0, ctx->stream>>>(partial, (int) split, m, d_y);
            KCHECK_LAUNCH();
        }
        return KEMCU_OK;
    };
    // one right-hand side: FMA kernel, HBM-bound; several: the FP64 tensor-core kernel
    static_assert(kMaxRhs <= 8, "dense_mma_kernel takes at most 8 right-hand sides");
    if (op == kDense64)
        return nrhs == 1 ? launch(dense_matvec_kernel<double, 1>, ctx->d_a64, dense_rows<double, 1>())
                         : launch(dense_mma_kernel<double>, ctx->d_a64, kMmaRowsPerCta / 256);
    return nrhs == 1 ? launch(dense_matvec_kernel<float, 1>, ctx->d_a32, dense_rows<float, 1>())
                     : launch(dense_mma_kernel<float>, ctx->d_a32, kMmaRowsPerCta / 256);
}

int assemble(kemcu_ctx* ctx, bool want32)
{
    const size_t n = ctx->n;
    if (ctx->d_a64 && (!want32 || ctx->d_a32))
        return KEMCU_OK;
    const size_t ld = op_ld(n);
    const size_t bytes64 = ld * n * sizeof(double), bytes32 = want32 ? ld * n * sizeof(float) : 0;
    size_t budget = ctx->assembled_budget;
    if (budget == 0) {
        size_t fr = 0, tot = 0;
        KC(cudaMemGetInfo(&fr, &tot));
        budget = (size_t) (0.7 * (double) fr) + (ctx->d_a64 ? bytes64 : 0);
    }
    if (bytes64 + bytes32 > budget)
        return fail(ctx, KEMCU_ENOMEM, "assembled operator needs %zu bytes, budget %zu", bytes64 + bytes32, budget);
    if (!ctx->d_a64 && cudaMalloc(&ctx->d_a64, bytes64) != cudaSuccess) {
        cudaGetLastError();
        ctx->d_a64 = nullptr;
        return fail(ctx, KEMCU_ENOMEM, "allocation of the assembled operator failed");
    }
    const bool fill32 = want32 && !ctx->d_a32;
    if (fill32 && cudaMalloc(&ctx->d_a32, bytes32) != cudaSuccess) {
        cudaGetLastError();
        ctx->d_a32 = nullptr;
        return fail(ctx, KEMCU_ENOMEM, "allocation of the FP32 operator copy failed");
    }
    if (ctx->axisym) {
        const dim3 grid((unsigned) ((n + kAxThreads - 1) / kAxThreads), (unsigned) axisym_split(ctx->num_sms, n, n));
        axisym_assemble_kernel<<<grid, kAxThreads, 0, ctx->stream>>>(ctx->d_rec, rRecSize, (int) n, ld, ctx->d_a64,
                                                                     fill32 ? ctx->d_a32 : nullptr);
        KCHECK_LAUNCH();
        return KEMCU_OK;
    }
    const int split = grid_split(ctx, n, n);
    dim3 grid((unsigned) ((n + kThreads - 1) / kThreads), (unsigned) split);
    assemble_kernel<false><<<grid, kThreads, 0, ctx->stream>>>(ctx->d_rec, ctx->d_tgt, (int) n, 0, (int) n, ctx->d_a64,
                                                              fill32 ? ctx->d_a32 : nullptr, ctx->d_flag + 1);
    KCHECK_LAUNCH();
    return KEMCU_OK;
}

// ------------------------------------------------------------------------------- GMRES
// GMRES from x0 = 0, as KGeneralizedMinimalResidual (x = V y, residual estimate |p_{j+1}|
// relative to |b|), with the restarts of KIterativeKrylovRestartCondition (every `restart`
// iterations: x += V y, r = b - A x, a new Krylov space from r; 0 = never) and the right
// preconditioning of KPreconditionedGeneralizedMinimalResidual (w = A P v_j; x += P V y for a
// stationary P, x += Z y with the kept Z_j = P v_j otherwise). The reference forms x from the
// last cycle's basis alone (KGeneralizedMinimalResidual.hh UpdateSolution clears x), which after
// a restart drops the earlier cycles' part; here every cycle adds its correction, so a restarted
// solve converges to the same solution as an unrestarted one. Orthogonalisation is classical
// Gram-Schmidt applied twice (CGS2), which is as accurate as the reference's modified
// Gram-Schmidt and reads the basis with two batched passes instead of j sequential ones. The
// j x j triangular solve uses back-substitution (KGeneralizedMinimalResidual::UseBackSubstitution).
// basis entries (n x (j+1)) up to which one CTA per RHS orthogonalises (arnoldi_small_kernel)
constexpr size_t kArnoldiSmall = (size_t) 1 << 16;

// Right preconditioner of a Krylov solve (KPreconditioner, KEMField/Source/LinearAlgebra/
// Preconditioners): Jacobi scales by the inverse diagonal (KJacobiPreconditioner.hh,
// stationary); the implicit Krylov form runs an inner GMRES from zero on its own operator to a
// relative tolerance (KImplicitKrylovPreconditioner.hh:50-54, not stationary).
struct Precond
{
    int kind = KEMCU_PRECON_NONE;
    const double* dinv = nullptr;  // Jacobi: 1 / A(i, i), n values
    int op = kFree64;              // implicit Krylov: the inner operator, tolerance and iterations
    double tol = 0.01;
    int max_iter = 30;
    int inner_iters = 0;           // accumulated over the applications
    int inner_matvecs = 0;
};

// workspace slots of one GMRES: the outer solve's, or those of the implicit Krylov
// preconditioner's inner solve (which runs inside an outer iteration)
struct KrylovSlots
{
    int basis, w, misc, k;
};
constexpr KrylovSlots kOuterSlots{sBasis, sVec2, sMisc, sVec1};
constexpr KrylovSlots kInnerSlots{sInBasis, sInW, sInMisc, sInK};

int apply_precond(kemcu_ctx* ctx, Precond& pc, const double* d_in, double* d_out, int nrhs);

int gmres_core(kemcu_ctx* ctx, int op, const double* d_b, double* d_x, int nrhs, double tol, int max_iter,
               int& iters, double& est, int& matvecs, int restart = 0, Precond* pc = nullptr,
               const KrylovSlots& sl = kOuterSlots)
{
    const int n = (int) ctx->n;
    const int m = std::max(1, restart > 0 ? std::min(restart, max_iter) : max_iter);  // iterations per cycle
    const int hs = m + 2;
    const bool flexible = pc && pc->kind == KEMCU_PRECON_IMPLICIT_KRYLOV;
    const bool jacobi = pc && pc->kind == KEMCU_PRECON_JACOBI;
    const bool outer = sl.basis == sBasis;
    void *pV, *pW, *pH, *pZ = nullptr;
    int rc;
    if ((rc = ensure(ctx, sl.basis, (size_t) (m + 1) * nrhs * n * sizeof(double), &pV)))
        return rc;
    if ((rc = ensure(ctx, sl.w, (size_t) nrhs * n * sizeof(double), &pW)))
        return rc;
    if ((rc = ensure(ctx, sl.misc, (size_t) nrhs * hs * 3 * sizeof(double) + 64 * (size_t) nrhs * kDotBlocks * sizeof(double), &pH)))
        return rc;
    // the preconditioned basis (flexible), or one vector for the Jacobi-scaled v_j and P V y
    if ((flexible || jacobi) && (rc = ensure(ctx, sZ, (size_t) (flexible ? m : 1) * nrhs * n * sizeof(double), &pZ)))
        return rc;
    double* V = (double*) pV;
    double* w = (double*) pW;
    double* Z = (double*) pZ;
    double* h = (double*) pH;             // [nrhs][hs] first projection
    double* h2 = h + (size_t) nrhs * hs;  // [nrhs][hs] second projection / norms
    double* yv = h2 + (size_t) nrhs * hs; // [nrhs][hs] solution coefficients
    double* part = yv + (size_t) nrhs * hs;
    void* pk;
    if ((rc = ensure(ctx, sl.k, (size_t) nrhs * sizeof(int) + 256, &pk)))
        return rc;
    int* d_k = (int*) pk;
    const dim3 vg((n + 255) / 256, nrhs);
    const size_t vec = (size_t) nrhs * n;
    // x0 = 0, r0 = b
    KC(cudaMemsetAsync(d_x, 0, vec * sizeof(double), ctx->stream));
    KC(cudaMemcpyAsync(V, d_b, vec * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    std::vector<double> hb((size_t) nrhs * hs);
    std::vector<double> bnorm(nrhs, 0.), p((size_t) nrhs * hs, 0.), cs((size_t) nrhs * hs), sn((size_t) nrhs * hs);
    std::vector<std::vector<double>> H(nrhs);  // column-major R, one column of hs added per iteration
    std::vector<int> kfin(nrhs, 0);
    std::vector<char> done(nrhs, 0);
    std::vector<double> hcol((size_t) nrhs * hs), hcol2((size_t) nrhs * hs), b2((size_t) nrhs * hs);
    std::vector<double> y((size_t) nrhs * hs);
    iters = 0;
    est = 0.;
    bool stop = false;
    for (int cycle = 0;; cycle++) {
        // |r| and v0 = r / |r|
        multi_dot_kernel<<<dim3(kDotBlocks, nrhs), kDotThreads, 0, ctx->stream>>>(V, V, n, nrhs, 0, 1, part, ctx->d_counter, h2, hs);
        KCHECK_LAUNCH();
        scale_kernel<<<vg, 256, 0, ctx->stream>>>(V, V, n, h2, hs, 0);
        KCHECK_LAUNCH();
        KC(cudaMemcpyAsync(hb.data(), h2, (size_t) nrhs * hs * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        KC(cudaStreamSynchronize(ctx->stream));
        std::fill(p.begin(), p.end(), 0.);
        double worst0 = 0.;
        for (int r = 0; r < nrhs; r++) {
            const double rn = std::sqrt(hb[(size_t) r * hs]);
            if (cycle == 0)
                bnorm[r] = rn;
            p[(size_t) r * hs] = rn;
            kfin[r] = 0;
            H[r].clear();
            if (cycle > 0 && !done[r] && bnorm[r] > 0.)
                worst0 = std::max(worst0, rn / bnorm[r]);
            if (!(bnorm[r] > 0.) || (cycle > 0 && rn <= tol * bnorm[r]))
                done[r] = 1;
        }
        if (cycle > 0)
            est = worst0;  // the restarted residual, until the new cycle's first estimate
        for (int j = 0; j < m && iters < max_iter; j++) {
            bool all = true;
            for (int r = 0; r < nrhs; r++)
                all = all && done[r];
            if (all)
                break;
            double* vj = V + (size_t) j * vec;
            double* vn = V + (size_t) (j + 1) * vec;
            const double* src = vj;
            if (jacobi) {
                diag_scale_kernel<<<vg, 256, 0, ctx->stream>>>(pc->dinv, vj, Z, n, 0);
                KCHECK_LAUNCH();
                src = Z;
            }
            else if (flexible) {
                double* zj = Z + (size_t) j * vec;
                if ((rc = apply_precond(ctx, *pc, vj, zj, nrhs)))
                    return rc;
                src = zj;
            }
            if ((rc = apply_op(ctx, op, src, w, nrhs)))
                return rc;
            matvecs++;
            if ((size_t) n * (size_t) (j + 1) <= kArnoldiSmall) {
                // one CTA per RHS: both Gram-Schmidt passes, the norm and the new basis vector
                arnoldi_small_kernel<<<nrhs, kArnoldiThreads, 0, ctx->stream>>>(V, w, n, nrhs, j, h, hs);
                KCHECK_LAUNCH();
                KC(cudaMemcpyAsync(hcol.data(), h, (size_t) nrhs * hs * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
                KC(cudaStreamSynchronize(ctx->stream));
                for (int r = 0; r < nrhs; r++) {
                    const double beta = hcol[(size_t) r * hs + hs - 1];
                    b2[(size_t) r * hs] = beta * beta;
                    for (int k = 0; k <= j; k++)
                        hcol2[(size_t) r * hs + k] = 0.;
                }
            }
            else {
                for (int pass = 0; pass < 2; pass++) {
                    double* hh = pass == 0 ? h : h2;
                    for (int k0 = 0; k0 <= j; k0 += 64) {
                        const int nk = std::min(64, j + 1 - k0);
                        multi_dot_kernel<<<dim3(kDotBlocks, nrhs), kDotThreads, 0, ctx->stream>>>(V, w, n, nrhs, k0, nk,
                                                                                                 part, ctx->d_counter, hh, hs);
                        KCHECK_LAUNCH();
                    }
                    for (int k0 = 0; k0 <= j; k0 += 64) {
                        const int nk = std::min(64, j + 1 - k0);
                        gs_update_kernel<<<vg, 256, 0, ctx->stream>>>(V, w, n, nrhs, k0, nk, hh, hs, nullptr);
                        KCHECK_LAUNCH();
                    }
                }
                // beta^2 into yv[r][0]
                multi_dot_kernel<<<dim3(kDotBlocks, nrhs), kDotThreads, 0, ctx->stream>>>(w, w, n, nrhs, 0, 1, part,
                                                                                         ctx->d_counter, yv, hs);
                KCHECK_LAUNCH();
                scale_kernel<<<vg, 256, 0, ctx->stream>>>(w, vn, n, yv, hs, 0);
                KCHECK_LAUNCH();
                KC(cudaMemcpyAsync(hcol.data(), h, (size_t) nrhs * hs * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
                KC(cudaMemcpyAsync(hcol2.data(), h2, (size_t) nrhs * hs * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
                KC(cudaMemcpyAsync(b2.data(), yv, (size_t) nrhs * hs * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
                KC(cudaStreamSynchronize(ctx->stream));
            }
            iters++;
            double worst = 0.;
            for (int r = 0; r < nrhs; r++) {
                if (done[r])
                    continue;
                H[r].resize((size_t) (j + 1) * hs, 0.);
                double* col = H[r].data() + (size_t) j * hs;
                for (int k = 0; k <= j; k++)
                    col[k] = hcol[(size_t) r * hs + k] + hcol2[(size_t) r * hs + k];
                const double beta = std::sqrt(b2[(size_t) r * hs]);
                // apply previous Givens rotations (KGeneralizedMinimalResidual.hh:240-246)
                for (int k = 0; k < j; k++) {
                    const double a = col[k], b = col[k + 1];
                    col[k] = cs[(size_t) r * hs + k] * a + sn[(size_t) r * hs + k] * b;
                    col[k + 1] = -sn[(size_t) r * hs + k] * a + cs[(size_t) r * hs + k] * b;
                }
                const double gam = std::sqrt(col[j] * col[j] + beta * beta);
                cs[(size_t) r * hs + j] = col[j] / gam;
                sn[(size_t) r * hs + j] = beta / gam;
                col[j] = gam;
                p[(size_t) r * hs + j + 1] = -sn[(size_t) r * hs + j] * p[(size_t) r * hs + j];
                p[(size_t) r * hs + j] = cs[(size_t) r * hs + j] * p[(size_t) r * hs + j];
                const double rel = std::fabs(p[(size_t) r * hs + j + 1]) / bnorm[r];
                kfin[r] = j + 1;
                if (rel <= tol || !(beta > 0.))
                    done[r] = 1;
                worst = std::max(worst, rel);
            }
            est = worst;
            if (outer && ctx->cb && ctx->cb(ctx->cb_user, iters, worst)) {
                stop = true;
                break;
            }
        }
        // y = R^-1 p; x += V y (P V y for Jacobi, Z y for the flexible form)
        std::fill(y.begin(), y.end(), 0.);
        for (int r = 0; r < nrhs; r++) {
            const int k = kfin[r];
            for (int i = k - 1; i >= 0; i--) {
                double s = p[(size_t) r * hs + i];
                for (int c = i + 1; c < k; c++)
                    s -= H[r][(size_t) c * hs + i] * y[(size_t) r * hs + c];
                y[(size_t) r * hs + i] = s / H[r][(size_t) i * hs + i];
            }
        }
        KC(cudaMemcpyAsync(yv, y.data(), (size_t) nrhs * hs * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
        KC(cudaMemcpyAsync(d_k, kfin.data(), (size_t) nrhs * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
        if (flexible) {
            combine_kernel<<<vg, 256, 0, ctx->stream>>>(Z, yv, hs, n, nrhs, d_k, d_x);
            KCHECK_LAUNCH();
        }
        else if (jacobi) {
            KC(cudaMemsetAsync(Z, 0, vec * sizeof(double), ctx->stream));
            combine_kernel<<<vg, 256, 0, ctx->stream>>>(V, yv, hs, n, nrhs, d_k, Z);
            KCHECK_LAUNCH();
            diag_scale_kernel<<<vg, 256, 0, ctx->stream>>>(pc->dinv, Z, d_x, n, 1);
            KCHECK_LAUNCH();
        }
        else {
            combine_kernel<<<vg, 256, 0, ctx->stream>>>(V, yv, hs, n, nrhs, d_k, d_x);
            KCHECK_LAUNCH();
        }
        bool all = true;
        for (int r = 0; r < nrhs; r++)
            all = all && done[r];
        if (all || stop || iters >= max_iter || restart <= 0)
            break;
        // restart from the current solution: r = b - A x into V[0]
        if ((rc = apply_op(ctx, op, d_x, V, nrhs)))
            return rc;
        matvecs++;
        residual_kernel<<<(unsigned) ((vec + 255) / 256), 256, 0, ctx->stream>>>(d_b, V, vec);
        KCHECK_LAUNCH();
    }
    KC(cudaStreamSynchronize(ctx->stream));
    return KEMCU_OK;
}

// z = P v: Jacobi scaling, or the implicit Krylov preconditioner's inner GMRES from zero
int apply_precond(kemcu_ctx* ctx, Precond& pc, const double* d_in, double* d_out, int nrhs)
{
    const int n = (int) ctx->n;
    if (pc.kind == KEMCU_PRECON_JACOBI) {
        diag_scale_kernel<<<dim3((n + 255) / 256, nrhs), 256, 0, ctx->stream>>>(pc.dinv, d_in, d_out, n, 0);
        KCHECK_LAUNCH();
        return KEMCU_OK;
    }
    if (pc.kind == KEMCU_PRECON_IMPLICIT_KRYLOV) {
        int it = 0, mv = 0;
        double e = 0.;
        int rc = gmres_core(ctx, pc.op, d_in, d_out, nrhs, pc.tol, pc.max_iter, it, e, mv, 0, nullptr, kInnerSlots);
        pc.inner_iters += it;
        pc.inner_matvecs += mv;
        return rc;
    }
    KC(cudaMemcpyAsync(d_out, d_in, (size_t) nrhs * n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    return KEMCU_OK;
}

double inner_tolerance()
{
    const char* s = getenv("KEMCU_INNER_TOL");
    return s ? atof(s) : 1e-6;
}

// Iterative refinement (solve modes KEMCU_SOLVE_MIXED, _ASSEMBLED and _FP32): x from 0, then
// repeatedly a correction d from an inner solve of A_low d = r (inner(r, d, tol, iterations,
// estimate, products)) and the residual r = b - A x with the FP64 operator hi_op, until the
// worst right-hand side's |r| / |b| is at most rel_tol (or an inner solve makes no progress,
// or 20 steps). The inner solve only has to bring the worst right-hand side to a tenth of the
// target: from relative residual rel, a reduction by 0.1 rel_tol / rel suffices (the first
// step, rel = 1, runs to the inner tolerance).
template<class Inner>
int refine_solve(kemcu_ctx* ctx, int hi_op, const double* d_b, double* d_x, double* d_r, double* d_d, int n_rhs,
                 double rel_tol, Inner inner, int& iters, double& est, double& rel, int& steps, int& fp64, int& low)
{
    const int n = (int) ctx->n;
    const size_t m = (size_t) n_rhs * n;
    int rc;
    const double tin = std::max(rel_tol, inner_tolerance());
    KC(cudaMemsetAsync(d_x, 0, m * sizeof(double), ctx->stream));
    KC(cudaMemcpyAsync(d_r, d_b, m * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    std::vector<double> hb(m);
    KC(cudaMemcpyAsync(hb.data(), d_b, m * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    KC(cudaStreamSynchronize(ctx->stream));
    std::vector<double> bn(n_rhs, 0.);
    for (int r = 0; r < n_rhs; r++) {
        for (int i = 0; i < n; i++)
            bn[r] += hb[(size_t) r * n + i] * hb[(size_t) r * n + i];
        bn[r] = std::sqrt(bn[r]);
    }
    rel = 1.;
    for (int outer = 0; outer < 20; outer++) {
        int it = 0;
        const double tin_k = std::min(0.5, std::max(tin, 0.1 * rel_tol / rel));
        if ((rc = inner(d_r, d_d, tin_k, it, est, low)))
            return rc;
        iters += it;
        axpy_kernel<<<(unsigned) ((m + 255) / 256), 256, 0, ctx->stream>>>(1., d_d, d_x, m);
        KCHECK_LAUNCH();
        if ((rc = apply_op(ctx, hi_op, d_x, d_r, n_rhs)))
            return rc;
        fp64++;
        residual_kernel<<<(unsigned) ((m + 255) / 256), 256, 0, ctx->stream>>>(d_b, d_r, m);
        KCHECK_LAUNCH();
        KC(cudaMemcpyAsync(hb.data(), d_r, m * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        KC(cudaStreamSynchronize(ctx->stream));
        rel = 0.;
        for (int r = 0; r < n_rhs; r++) {
            double s = 0.;
            for (int i = 0; i < n; i++)
                s += hb[(size_t) r * n + i] * hb[(size_t) r * n + i];
            rel = std::max(rel, bn[r] > 0. ? std::sqrt(s) / bn[r] : 0.);
        }
        steps = outer + 1;
        if (rel <= rel_tol || it == 0)
            break;
    }
    return KEMCU_OK;
}
}  // namespace

// ------------------------------------------------------------------------------- C ABI
extern "C" {

void kemcu_default_config(kemcu_config* cfg)
{
    if (!cfg)
        return;
    cfg->device = 0;
    cfg->one_over_four_pi_eps0 = 1. / (4. * 3.141592653589793238462643383279502884 * 8.8541878128e-12);
    cfg->eps0 = 8.8541878128e-12;
    cfg->assembled_budget_bytes = 0;
    cfg->autotune = 1;
}

int kemcu_create(kemcu_ctx** out, const kemcu_config* cfg)
{
    if (!out)
        return KEMCU_EINVAL;
    *out = nullptr;
    kemcu_config def;
    kemcu_default_config(&def);
    if (!cfg)
        cfg = &def;
    auto* ctx = new kemcu_ctx();
    ctx->device = cfg->device;
    ctx->k.one_over_four_pi_eps0 = cfg->one_over_four_pi_eps0;
    ctx->k.eps0 = cfg->eps0;
    ctx->k.pi = 3.141592653589793238462643383279502884;
    ctx->assembled_budget = cfg->assembled_budget_bytes;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev <= cfg->device || cfg->device < 0) {
        cudaGetLastError();
        *out = ctx;
        return fail(ctx, KEMCU_ECUDA, "no usable CUDA device %d (%s)", cfg->device,
                    e == cudaSuccess ? "ordinal out of range" : cudaGetErrorString(e));
    }
    *out = ctx;
    KC(cudaSetDevice(ctx->device));
    cudaDeviceProp prop;
    KC(cudaGetDeviceProperties(&prop, ctx->device));
    if (prop.major < 10)
        return fail(ctx, KEMCU_ECUDA, "device %s is sm_%d%d; this library is built for sm_100a", prop.name, prop.major,
                    prop.minor);
    ctx->num_sms = prop.multiProcessorCount;
    KC(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    KC(cudaEventCreate(&ctx->ev0));
    KC(cudaEventCreate(&ctx->ev1));
    KC(cudaEventCreate(&ctx->tv0));
    KC(cudaEventCreate(&ctx->tv1));
    ctx->autotune = cfg->autotune != 0;
    KC(cudaMalloc(&ctx->d_counter, 64 * sizeof(unsigned)));
    KC(cudaMemset(ctx->d_counter, 0, 64 * sizeof(unsigned)));
    // [0]: non-finite values seen; [1]: a direct-sum pipeline wait timed out
    KC(cudaMalloc(&ctx->d_flag, 2 * sizeof(int)));
    KC(cudaMemset(ctx->d_flag, 0, 2 * sizeof(int)));
    // set-up of kemcu_field_dev_noalloc: the static scratch array's device address on this
    // device (host code may not use the symbol itself as a device pointer)
    KC(cudaGetSymbolAddress((void**) &ctx->noalloc_scratch, g_noalloc_scratch));
    // rule tables
    std::vector<double> rules(kNumNodes * 3), gl(20), q(kNumNodes * kQ);
    tables::build(rules.data(), gl.data());
    for (int k = 0; k < kNumNodes; k++) {
        const double sc = k < kRect7 ? 1. / 3. : 0.5;  // rule centroid
        const double s = rules[3 * k] - sc, t = rules[3 * k + 1] - sc, w = rules[3 * k + 2];
        const double v[kQ] = {-2. * s, -2. * t, s * s, s * t, t * t, w, w * s, w * t};
        for (int c = 0; c < kQ; c++)
            q[kQ * k + c] = v[c];
    }
    KC(cudaMemcpyToSymbol(c_q, q.data(), q.size() * sizeof(double)));
    std::vector<double> qa(kNumNodes * kQA);
    for (int k = 0; k < kNumNodes; k++) {
        const double sc = k < kRect7 ? 1. / 3. : 0.5;
        const double s = rules[3 * k] - sc, t = rules[3 * k + 1] - sc, w = rules[3 * k + 2];
        const double v[kQA] = {w, w * s, w * t, w * s * s, w * s * t, w * t * t};
        for (int c = 0; c < kQA; c++)
            qa[kQA * k + c] = v[c];
    }
    KC(cudaMemcpyToSymbol(c_qa, qa.data(), qa.size() * sizeof(double)));
    // pair form of the centrally symmetric rectangle rules
    std::vector<double> qp(kNumPairs * kQ, 0.);
    double qc[2] = {0., 0.};
    const int rule_first[3] = {kRect7, kRect12, kRect33}, rule_n[3] = {7, 12, 33};
    const int pair_first[3] = {kPair7, kPair12, kPair33}, pair_n[3] = {3, 6, 16}, center[3] = {0, -1, 1};
    for (int r = 0; r < 3; r++) {
        std::vector<bool> used(rule_n[r], false);
        int np = 0, nc = 0;
        for (int i = 0; i < rule_n[r]; i++) {
            if (used[i])
                continue;
            const double* a = &q[kQ * (rule_first[r] + i)];
            used[i] = true;
            if (std::fabs(a[0]) < 1e-14 && std::fabs(a[1]) < 1e-14) {
                if (center[r] < 0 || nc++)
                    return fail(ctx, KEMCU_ECUDA, "rectangle rule %d: unexpected centroid node", rule_n[r]);
                qc[center[r]] = a[5];
                continue;
            }
            int j = i + 1;
            for (; j < rule_n[r]; j++) {
                const double* b = &q[kQ * (rule_first[r] + j)];
                if (!used[j] && std::fabs(a[0] + b[0]) < 1e-13 && std::fabs(a[1] + b[1]) < 1e-13 && std::fabs(a[5] - b[5]) <= 1e-13 * std::fabs(a[5]))
                    break;
            }
            if (j == rule_n[r] || np == pair_n[r])
                return fail(ctx, KEMCU_ECUDA, "rectangle rule %d is not centrally symmetric", rule_n[r]);
            used[j] = true;
            for (int c = 0; c < kQ; c++)
                qp[kQ * (pair_first[r] + np) + c] = a[c];
            np++;
        }
        if (np != pair_n[r] || nc != (center[r] >= 0 ? 1 : 0))
            return fail(ctx, KEMCU_ECUDA, "rectangle rule %d: unexpected node pairing", rule_n[r]);
    }
    KC(cudaMemcpyToSymbol(c_qp, qp.data(), qp.size() * sizeof(double)));
    KC(cudaMemcpyToSymbol(c_qc, qc, sizeof qc));
    {
        std::vector<float> q32(q.begin(), q.end()), qp32(qp.begin(), qp.end());
        const float qc32[2] = {(float) qc[0], (float) qc[1]};
        KC(cudaMemcpyToSymbol(c_q32, q32.data(), q32.size() * sizeof(float)));
        KC(cudaMemcpyToSymbol(c_qp32, qp32.data(), qp32.size() * sizeof(float)));
        KC(cudaMemcpyToSymbol(c_qc32, qc32, sizeof qc32));
    }
    KC(cudaMemcpyToSymbol(c_gl, gl.data(), gl.size() * sizeof(double)));
    KC(cudaMemcpyToSymbol(c_k, &ctx->k, sizeof(Constants)));
    double rk[kStages][kStages];
    rk8_table(rk);
    KC(cudaMemcpyToSymbol(c_rk8, rk, sizeof rk));
    return KEMCU_OK;
}

int kemcu_destroy(kemcu_ctx* ctx)
{
    if (!ctx)
        return KEMCU_OK;
    if (ctx->stream) {
        cudaSetDevice(ctx->device);
        cudaStreamSynchronize(ctx->stream);
        for (auto& b : ctx->scratch)
            if (b.p)
                cudaFree(b.p);
        cudaFree(ctx->d_rec);
        cudaFree(ctx->d_tgt);
        cudaFree(ctx->d_sigma);
        cudaFree(ctx->d_a64);
        cudaFree(ctx->d_a32);
        cudaFree(ctx->d_near_ptr);
        cudaFree(ctx->d_near_row);
        cudaFree(ctx->d_near_val);
        cudaFree(ctx->d_counter);
        cudaFree(ctx->d_flag);
        fm_release(ctx);
        cudaEventDestroy(ctx->ev0);
        cudaEventDestroy(ctx->ev1);
        cudaEventDestroy(ctx->tv0);
        cudaEventDestroy(ctx->tv1);
        cudaStreamDestroy(ctx->stream);
    }
    delete ctx;
    return KEMCU_OK;
}

const char* kemcu_last_error(const kemcu_ctx* ctx)
{
    return ctx ? ctx->err.c_str() : "null context";
}

double kemcu_last_kernel_ms(const kemcu_ctx* ctx)
{
    return ctx ? ctx->last_ms : 0.;
}

size_t kemcu_num_elements(const kemcu_ctx* ctx)
{
    return ctx ? ctx->n : 0;
}

int kemcu_set_geometry(kemcu_ctx* ctx, size_t n, const int32_t* shape, const int32_t* boundary, const double* geom11,
                       const double* value)
{
    if (!ctx || !ctx->stream)
        return ctx ? fail(ctx, KEMCU_ESTATE, "context has no device") : KEMCU_EINVAL;
    if (n == 0 || n > (size_t) 0x7fffffff || !shape || !boundary || !geom11 || !value)
        return fail(ctx, KEMCU_EINVAL, "invalid geometry arguments (n = %zu)", n);
    KC(cudaSetDevice(ctx->device));
    size_t n_axisym = 0;
    for (size_t i = 0; i < n; i++) {
        if (shape[i] < 0 || shape[i] > KEMCU_RING || (boundary[i] != 0 && boundary[i] != 1))
            return fail(ctx, KEMCU_EINVAL, "element %zu: shape %d / boundary %d not supported", i, shape[i], boundary[i]);
        for (int c = 0; c < 11; c++)
            if (!std::isfinite(geom11[11 * i + c]))
                return fail(ctx, KEMCU_EINVAL, "element %zu: non-finite geometry", i);
        const double* g = geom11 + 11 * i;
        if (shape[i] == KEMCU_CONIC_SECTION || shape[i] == KEMCU_RING) {
            n_axisym++;
            if (boundary[i] != KEMCU_DIRICHLET)
                return fail(ctx, KEMCU_EINVAL, "element %zu: axisymmetric elements take Dirichlet boundaries only", i);
            if (shape[i] == KEMCU_RING ? !(g[0] > 0.)
                                       : !(g[0] >= 0. && g[2] >= 0. && (g[0] != g[2] || g[1] != g[3])))
                return fail(ctx, KEMCU_EINVAL, "element %zu: radii must be non-negative (a ring's positive) and a "
                                               "conic section's end points distinct", i);
        }
        else if (shape[i] != kLineSegment && !(g[0] > 0. && g[1] > 0.))
            return fail(ctx, KEMCU_EINVAL, "element %zu: side lengths must be positive", i);
    }
    if (n_axisym != 0 && n_axisym != n)
        return fail(ctx, KEMCU_EINVAL, "axisymmetric elements (conic sections, rings) cannot share a context with "
                                       "triangles, rectangles or line segments");
    // release everything that depends on the old geometry
    fm_release(ctx);
    cudaFree(ctx->d_rec);
    cudaFree(ctx->d_tgt);
    cudaFree(ctx->d_sigma);
    cudaFree(ctx->d_a64);
    cudaFree(ctx->d_a32);
    cudaFree(ctx->d_near_ptr);
    cudaFree(ctx->d_near_row);
    cudaFree(ctx->d_near_val);
    ctx->d_rec = nullptr;
    ctx->d_tgt = nullptr;
    ctx->d_sigma = nullptr;
    ctx->d_a64 = nullptr;
    ctx->d_a32 = nullptr;
    ctx->d_near_ptr = nullptr;
    ctx->d_near_row = nullptr;
    ctx->d_near_val = nullptr;
    ctx->have_sigma = false;
    ctx->n = 0;
    ctx->h_rec.assign(n * rRecSize, 0.);
    ctx->h_tgt.assign(n, TargetRec{});
    ctx->h_rhs.assign(n, 0.);
    ctx->h_shape.assign(shape, shape + n);
    ctx->axisym = n_axisym != 0;
    for (size_t i = 0; i < n; i++) {
        if (ctx->axisym)
            build_axisym_record(geom11 + 11 * i, shape[i], value[i], ctx->k, ctx->h_rec.data() + i * rRecSize,
                                ctx->h_rhs[i]);
        else
            build_record(geom11 + 11 * i, shape[i], boundary[i], value[i], ctx->k, ctx->h_rec.data() + i * rRecSize,
                         ctx->h_tgt[i], ctx->h_rhs[i]);
    }
    KC(cudaMalloc(&ctx->d_rec, n * rRecSize * sizeof(double)));
    KC(cudaMalloc(&ctx->d_tgt, n * sizeof(TargetRec)));
    KC(cudaMalloc(&ctx->d_sigma, n * sizeof(double)));
    KC(cudaMemcpy(ctx->d_rec, ctx->h_rec.data(), n * rRecSize * sizeof(double), cudaMemcpyHostToDevice));
    KC(cudaMemcpy(ctx->d_tgt, ctx->h_tgt.data(), n * sizeof(TargetRec), cudaMemcpyHostToDevice));
    KC(cudaMemset(ctx->d_sigma, 0, n * sizeof(double)));
    ctx->n = n;
    return KEMCU_OK;
}

int kemcu_set_sigma(kemcu_ctx* ctx, const double* sigma)
{
    int rc = check_ready(ctx, false);
    if (rc)
        return rc;
    if (!sigma)
        return fail(ctx, KEMCU_EINVAL, "null sigma");
    KC(cudaMemcpy(ctx->d_sigma, sigma, ctx->n * sizeof(double), cudaMemcpyHostToDevice));
    ctx->have_sigma = true;
    return KEMCU_OK;
}

int kemcu_get_sigma(kemcu_ctx* ctx, double* sigma)
{
    int rc = check_ready(ctx, true);
    if (rc)
        return rc;
    KC(cudaMemcpy(sigma, ctx->d_sigma, ctx->n * sizeof(double), cudaMemcpyDeviceToHost));
    return KEMCU_OK;
}

int kemcu_rhs(kemcu_ctx* ctx, double* b)
{
    int rc = check_ready(ctx, false);
    if (rc)
        return rc;
    std::memcpy(b, ctx->h_rhs.data(), ctx->n * sizeof(double));
    return KEMCU_OK;
}

int kemcu_field_dev(kemcu_ctx* ctx, const double* dP, size_t n, double* dout4, int precision, int what)
{
    int rc = check_ready(ctx, true);
    if (rc)
        return rc;
    if (n == 0)
        return KEMCU_OK;
    if (!dP || !dout4 || n > (size_t) 0x7fffffff || precision < KEMCU_FP64 || precision > KEMCU_FP32 || what < 0 ||
        what > 2)
        return fail(ctx, KEMCU_EINVAL, "invalid field arguments");
    KC(cudaSetDevice(ctx->device));
    Timer t(ctx);
    if (n < kSortMin) {
        if ((rc = launch_field(ctx, dP, n, dout4, precision, what)))
            return rc;
    }
    else {
        // Morton order (meridian plane for axisymmetric models): bbox -> keys -> radix sort -> gather ->
        // evaluate -> scatter back
        const size_t cub_bytes = cub_sort_bytes(n);
        const size_t need = n * (2 * sizeof(unsigned long long) + 2 * sizeof(int) + 7 * sizeof(double)) + cub_bytes +
                            1024 + 128 * 6 * sizeof(double);
        void* base;
        if ((rc = ensure(ctx, sSort, need, &base)))
            return rc;
        char* q = (char*) base;
        auto take = [&q](size_t b) {
            char* r = q;
            q += (b + 255) & ~(size_t) 255;
            return r;
        };
        auto* k0 = (unsigned long long*) take(n * 8);
        auto* k1 = (unsigned long long*) take(n * 8);
        auto* i0 = (int*) take(n * 4);
        auto* i1 = (int*) take(n * 4);
        auto* ps = (double*) take(n * 24);
        auto* os = (double*) take(n * 32);
        auto* box = (double*) take(6 * sizeof(double));
        auto* part = (double*) take(128 * 6 * sizeof(double));
        void* tmp = take(cub_bytes);
        bbox_kernel<<<128, 256, 0, ctx->stream>>>(dP, (int) n, part, ctx->d_counter + 32, box);
        KCHECK_LAUNCH();
        if (ctx->axisym)
            morton_rz_kernel<<<(unsigned) ((n + 255) / 256), 256, 0, ctx->stream>>>(dP, (int) n, box, k0, i0);
        else
            morton_kernel<<<(unsigned) ((n + 255) / 256), 256, 0, ctx->stream>>>(dP, (int) n, box, k0, i0);
        KCHECK_LAUNCH();
        size_t tb = cub_bytes;
        KC(cub::DeviceRadixSort::SortPairs(tmp, tb, k0, k1, i0, i1, (int) n, 0, 63, ctx->stream));
        gather_points_kernel<<<(unsigned) ((n + 255) / 256), 256, 0, ctx->stream>>>(dP, i1, (int) n, ps);
        KCHECK_LAUNCH();
        if ((rc = launch_field(ctx, ps, n, os, precision, what)))
            return rc;
        scatter_out_kernel<<<(unsigned) ((n + 255) / 256), 256, 0, ctx->stream>>>(os, i1, (int) n, dout4);
        KCHECK_LAUNCH();
    }
    t.stop();
    rc = check_finite(ctx, dout4, n * 4, "field result");
    if (rc == KEMCU_OK)
        finish_variant(ctx);
    ctx->pending_key = -1;
    return rc;
}

// Allocation-free direct sum (declared in kemcu.h): the element-split partial sums go to the
// file-scope g_noalloc_scratch instead of a grow-only cudaMalloc'd buffer. Every split writes
// its whole slice before reduce_splits reads it, so nothing needs clearing between calls.
int kemcu_field_dev_noalloc(kemcu_ctx* ctx, const double* dP, size_t n, double* dout4, int precision, int what)
{
    int rc = check_ready(ctx, true);
    if (rc)
        return rc;
    if (n == 0)
        return KEMCU_OK;
    if (!dP || !dout4 || precision < KEMCU_FP64 || precision > KEMCU_FP32 || what < 0 || what > 2)
        return fail(ctx, KEMCU_EINVAL, "invalid field arguments");
    if (n > (size_t) KEMCU_NOALLOC_MAX_POINTS)
        return fail(ctx, KEMCU_EINVAL, "kemcu_field_dev_noalloc takes at most %u points (got %zu): its scratch is "
                                       "a fixed %u-byte device array", (unsigned) KEMCU_NOALLOC_MAX_POINTS, n,
                    (unsigned) KEMCU_NOALLOC_SCRATCH_BYTES);
    if (!ctx->noalloc_scratch)
        return fail(ctx, KEMCU_ESTATE, "no-allocation scratch not set up");
    KC(cudaSetDevice(ctx->device));
    Timer t(ctx);
    if (ctx->axisym) {
        if ((rc = launch_axisym_field(ctx, dP, n, dout4, what, ctx->noalloc_scratch,
                                      KEMCU_NOALLOC_SCRATCH_BYTES / sizeof(double))))
            return rc;
        t.stop();
        return check_finite(ctx, dout4, n * 4, "field result");
    }
    const size_t cap = KEMCU_NOALLOC_SCRATCH_BYTES / sizeof(double);
    const int split = (int) std::min((size_t) grid_split(ctx, n, ctx->n), std::max((size_t) 1, cap / (4 * n)));
    if ((rc = launch_planar_field(ctx, dP, n, dout4, precision, what, split, ctx->noalloc_scratch)))
        return rc;
    t.stop();
    rc = check_finite(ctx, dout4, n * 4, "field result");
    if (rc == KEMCU_OK)
        finish_variant(ctx);
    ctx->pending_key = -1;
    return rc;
}

int kemcu_field(kemcu_ctx* ctx, const double* P, size_t n, double* out4, int precision, int what)
{
    int rc = check_ready(ctx, true);
    if (rc)
        return rc;
    if (n == 0)
        return KEMCU_OK;
    if (!P || !out4)
        return fail(ctx, KEMCU_EINVAL, "null point or output buffer");
    KC(cudaSetDevice(ctx->device));
    void *dp, *dout;
    if ((rc = ensure(ctx, sPts, n * 3 * sizeof(double), &dp)) || (rc = ensure(ctx, sOut, n * 4 * sizeof(double), &dout)))
        return rc;
    KC(cudaMemcpyAsync(dp, P, n * 3 * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    if ((rc = kemcu_field_dev(ctx, (const double*) dp, n, (double*) dout, precision, what)))
        return rc;
    KC(cudaMemcpyAsync(out4, dout, n * 4 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    KC(cudaStreamSynchronize(ctx->stream));
    return KEMCU_OK;
}

int kemcu_tune_field(kemcu_ctx* ctx, const double* dP, size_t n, double* dout4, int precision, int* variant,
                     float* ms)
{
    int rc = check_ready(ctx, true);
    if (rc || (rc = planar_only(ctx, "the field autotuner")))
        return rc;
    if (!dP || !dout4 || n == 0 || (precision != KEMCU_FP64 && precision != KEMCU_MIXED))
        return fail(ctx, KEMCU_EINVAL, "invalid tuning arguments");
    // every variant runs the whole evaluation twice (the first warms it up); the K1 launch of the
    // second run is timed
    std::vector<float> t(kNumFieldVariants, 0.f);
    ctx->time_k1 = true;
    for (int v = 0; v < kNumFieldVariants && rc == KEMCU_OK; v++) {
        ctx->force_variant = v;
        for (int rep = 0; rep < 2 && rc == KEMCU_OK; rep++)
            rc = kemcu_field_dev(ctx, dP, n, dout4, precision, KEMCU_FIELD_AND_POTENTIAL);
        if (rc == KEMCU_OK && cudaEventElapsedTime(&t[v], ctx->tv0, ctx->tv1) != cudaSuccess)
            rc = fail(ctx, KEMCU_ECUDA, "tuning timer failed: %s", cudaGetErrorString(cudaGetLastError()));
    }
    ctx->time_k1 = false;
    ctx->force_variant = -1;
    if (rc)
        return rc;
    const int key = tune_key(precision, n);
    const int best = (int) (std::min_element(t.begin(), t.end()) - t.begin());
    ctx->explored[key] = t;
    ctx->tuned[key] = best;
    if (variant)
        *variant = best;
    if (ms)
        std::copy(t.begin(), t.end(), ms);
    return KEMCU_OK;
}

int kemcu_field_variant(const kemcu_ctx* ctx, size_t n, int precision, int* variant)
{
    if (!ctx || !variant)
        return KEMCU_EINVAL;
    auto it = ctx->tuned.find(tune_key(precision, n));
    *variant = it == ctx->tuned.end() ? -1 : it->second;
    return KEMCU_OK;
}

int kemcu_field_variant_info(int variant, int* min_blocks, int* ring_stages)
{
    if (variant < 0 || variant >= kNumFieldVariants)
        return KEMCU_EINVAL;
    if (min_blocks)
        *min_blocks = kFieldVariants[variant].min_blocks;
    if (ring_stages)
        *ring_stages = kFieldVariants[variant].ring_stages;
    return KEMCU_OK;
}

int kemcu_field_variant_count(void)
{
    return kNumFieldVariants;
}

int kemcu_matrix_element(kemcu_ctx* ctx, size_t i, size_t j, double* a)
{
    int rc = check_ready(ctx, false);
    if (rc)
        return rc;
    if (i >= ctx->n || j >= ctx->n || !a)
        return fail(ctx, KEMCU_EINVAL, "matrix index out of range");
    KC(cudaSetDevice(ctx->device));
    // one thread computes the entry, in the FP64 form of the matvec
    void* d;
    if ((rc = ensure(ctx, sVec1, sizeof(double), &d)))
        return rc;
    if (ctx->axisym)
        axisym_entry_kernel<<<1, 1, 0, ctx->stream>>>(ctx->d_rec, rRecSize, (int) i, (int) j, (double*) d);
    else
        entry_kernel<<<1, 1, 0, ctx->stream>>>(ctx->d_rec, ctx->d_tgt, (int) i, (int) j, (double*) d);
    KCHECK_LAUNCH();
    KC(cudaMemcpyAsync(a, d, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    KC(cudaStreamSynchronize(ctx->stream));
    return KEMCU_OK;
}

int kemcu_matvec(kemcu_ctx* ctx, const double* x, double* y, int n_rhs, int precision, int assembled)
{
    int rc = check_ready(ctx, false);
    if (rc)
        return rc;
    if (!x || !y || n_rhs < 1 || n_rhs > kMaxRhs)
        return fail(ctx, KEMCU_EINVAL, "invalid matvec arguments (n_rhs must be 1..%d)", kMaxRhs);
    KC(cudaSetDevice(ctx->device));
    const size_t m = (size_t) n_rhs * ctx->n;
    void *dx, *dy;
    if ((rc = ensure(ctx, sVec0, m * sizeof(double), &dx)) || (rc = ensure(ctx, sVec1, m * sizeof(double), &dy)))
        return rc;
    KC(cudaMemcpyAsync(dx, x, m * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    if ((rc = clear_pipe_flag(ctx)))
        return rc;
    Timer t(ctx);
    if (precision < KEMCU_FP64 || precision > KEMCU_FP32)
        return fail(ctx, KEMCU_EINVAL, "invalid matvec precision %d", precision);
    // matrix-free: the entries in the requested form; assembled: the FP64 operator, or its FP32
    // copy for the reduced forms
    int op = precision == KEMCU_MIXED ? kFreeMixed : precision == KEMCU_FP32 ? kFree32 : kFree64;
    if (assembled) {
        const bool low = precision != KEMCU_FP64;
        if ((rc = assemble(ctx, low)))
            return rc;
        op = low ? kDense32 : kDense64;
    }
    if ((rc = apply_op(ctx, op, (const double*) dx, (double*) dy, n_rhs)))
        return rc;
    t.stop();
    KC(cudaMemcpyAsync(y, dy, m * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    return pipe_status(ctx, "matvec");
}

void kemcu_set_iteration_callback(kemcu_ctx* ctx, kemcu_iteration_callback cb, void* user)
{
    if (!ctx)
        return;
    ctx->cb = cb;
    ctx->cb_user = user;
}

int kemcu_gmres(kemcu_ctx* ctx, const double* b, double* x, int n_rhs, double rel_tol, int max_iter, int mode,
                kemcu_solve_stats* stats)
{
    int rc = check_ready(ctx, false);
    if (rc)
        return rc;
    if (!x || n_rhs < 1 || n_rhs > kMaxRhs || (b == nullptr && n_rhs != 1) || !(rel_tol > 0.) || max_iter < 1 ||
        mode < 0 || mode > KEMCU_SOLVE_FFTM)
        return fail(ctx, KEMCU_EINVAL, "invalid gmres arguments");
    if (mode == KEMCU_SOLVE_FFTM && !ctx->fm)
        return fail(ctx, KEMCU_ESTATE, "KEMCU_SOLVE_FFTM needs kemcu_fftm_configure first");
    KC(cudaSetDevice(ctx->device));
    if ((rc = clear_pipe_flag(ctx)))
        return rc;
    const int n = (int) ctx->n;
    const size_t m = (size_t) n_rhs * n;
    // device vectors: b, x, residual/correction
    double *d_b, *d_x, *d_r, *d_d;
    size_t need = 4 * m * sizeof(double);
    void* p;
    if ((rc = ensure(ctx, sVec0, need, &p)))
        return rc;
    d_b = (double*) p;
    d_x = d_b + m;
    d_r = d_x + m;
    d_d = d_r + m;
    if (b)
        KC(cudaMemcpyAsync(d_b, b, m * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    else
        KC(cudaMemcpyAsync(d_b, ctx->h_rhs.data(), m * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    kemcu_solve_stats st{};
    Timer t(ctx);
    auto t0 = std::chrono::steady_clock::now();
    int iters = 0, fp64 = 0, low = 0;
    double est = 0., rel = 0.;
    if (mode == KEMCU_SOLVE_PLAIN || mode == KEMCU_SOLVE_ASSEMBLED_FP64 || mode == KEMCU_SOLVE_FFTM) {
        int op = mode == KEMCU_SOLVE_FFTM ? kFftm : kFree64;
        if (mode == KEMCU_SOLVE_ASSEMBLED_FP64) {
            if ((rc = assemble(ctx, false)))
                return rc;
            op = kDense64;
        }
        if ((rc = gmres_core(ctx, op, d_b, d_x, n_rhs, rel_tol, max_iter, iters, est, fp64)))
            return rc;
        st.outer = 1;
        rel = est;
    }
    else {
        int low_op = mode == KEMCU_SOLVE_FP32 ? kFree32 : kFreeMixed, hi_op = kFree64;
        if (mode == KEMCU_SOLVE_ASSEMBLED) {
            if ((rc = assemble(ctx, true)))
                return rc;
            low_op = kDense32;
            hi_op = kDense64;
        }
        auto inner = [&](const double* r, double* d, double tol, int& it, double& e, int& mv) {
            return gmres_core(ctx, low_op, r, d, n_rhs, tol, max_iter, it, e, mv);
        };
        if ((rc = refine_solve(ctx, hi_op, d_b, d_x, d_r, d_d, n_rhs, rel_tol, inner, iters, est, rel, st.outer, fp64,
                               low)))
            return rc;
    }
    t.stop();
    st.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    st.iterations = iters;
    st.fp64_matvecs = fp64;
    st.low_matvecs = low;
    st.rel_residual = rel;
    st.rel_residual_estimate = est;
    if (stats)
        *stats = st;
    if ((rc = check_finite(ctx, d_x, m, "solution")))
        return rc;
    KC(cudaMemcpyAsync(x, d_x, m * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    if (n_rhs == 1) {
        KC(cudaMemcpyAsync(ctx->d_sigma, d_x, (size_t) n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
        ctx->have_sigma = true;
    }
    KC(cudaStreamSynchronize(ctx->stream));
    if (rel > rel_tol)
        return fail(ctx, KEMCU_ENOTCONVERGED, "GMRES stopped at relative residual %.3e > %.3e after %d iterations", rel,
                    rel_tol, iters);
    return KEMCU_OK;
}

unsigned long long kemcu_launch_count(const kemcu_ctx* ctx)
{
    return ctx ? ctx->launches : 0ULL;
}

int kemcu_band_histogram(kemcu_ctx* ctx, const double* P, size_t n, long long* counts)
{
    int rc = check_ready(ctx, false);
    if (rc || (rc = planar_only(ctx, "the band histogram")))
        return rc;
    if (!P || !counts || n == 0 || n > (size_t) 0x7fffffff)
        return fail(ctx, KEMCU_EINVAL, "invalid histogram arguments");
    KC(cudaSetDevice(ctx->device));
    void *dp, *dc;
    if ((rc = ensure(ctx, sPts, n * 3 * sizeof(double), &dp)) || (rc = ensure(ctx, sOut, 12 * sizeof(long long), &dc)))
        return rc;
    KC(cudaMemcpyAsync(dp, P, n * 3 * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    KC(cudaMemsetAsync(dc, 0, 12 * sizeof(long long), ctx->stream));
    band_histogram_kernel<<<(unsigned) ((n + 127) / 128), 128, 0, ctx->stream>>>(ctx->d_rec, (int) ctx->n,
                                                                               (const double*) dp, (int) n,
                                                                               (unsigned long long*) dc);
    KCHECK_LAUNCH();
    KC(cudaMemcpyAsync(counts, dc, 12 * sizeof(long long), cudaMemcpyDeviceToHost, ctx->stream));
    KC(cudaStreamSynchronize(ctx->stream));
    return KEMCU_OK;
}

int kemcu_selftest_timeout(kemcu_ctx* ctx, int complete)
{
    if (!ctx)
        return KEMCU_EINVAL;
    KC(cudaSetDevice(ctx->device));
    int rc = clear_pipe_flag(ctx);
    if (rc)
        return rc;
    wait_timeout_selftest_kernel<<<1, 32, 0, ctx->stream>>>(ctx->d_flag + 1, 2000000LL, complete ? 1 : 0);
    KCHECK_LAUNCH();
    return pipe_status(ctx, "self-test wait");
}

int kemcu_fma_peak(kemcu_ctx* ctx, double* fp64_tflops, double* fp32_tflops)
{
    if (!ctx || !ctx->stream)
        return ctx ? fail(ctx, KEMCU_ESTATE, "context has no device") : KEMCU_EINVAL;
    KC(cudaSetDevice(ctx->device));
    void* d;
    int rc;
    if ((rc = ensure(ctx, sMisc, 1 << 22, &d)))
        return rc;
    const int blocks = ctx->num_sms * 8, threads = 256, iters = 4096;
    for (int pass = 0; pass < 2; pass++) {
        for (int rep = 0; rep < 2; rep++) {  // first repetition warms up
            cudaEventRecord(ctx->ev0, ctx->stream);
            if (pass == 0)
                fma_probe_kernel<double><<<blocks, threads, 0, ctx->stream>>>((double*) d, iters);
            else
                fma_probe_kernel<float><<<blocks, threads, 0, ctx->stream>>>((float*) d, iters);
            KCHECK_LAUNCH();
            cudaEventRecord(ctx->ev1, ctx->stream);
            KC(cudaEventSynchronize(ctx->ev1));
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
        const double flops = 2.0 * kProbeChains * (double) iters * blocks * threads;
        const double tf = flops / (ms * 1e-3) / 1e12;
        if (pass == 0 && fp64_tflops)
            *fp64_tflops = tf;
        if (pass == 1 && fp32_tflops)
            *fp32_tflops = tf;
    }
    return KEMCU_OK;
}

int kemcu_rule_nodes(int which, double* out)
{
    if (which < 0 || which > 7 || !out)
        return KEMCU_EINVAL;
    std::vector<double> rules(kNumNodes * 3), gl(20);
    tables::build(rules.data(), gl.data());
    if (which >= 6) {
        const int off = which == 6 ? 0 : 2, half = which == 6 ? 2 : 8;
        for (int i = 0; i < half; i++) {
            out[3 * i] = gl[2 * (off + i)];
            out[3 * i + 1] = gl[2 * (off + i) + 1];
            out[3 * i + 2] = 0.;
        }
        return half;
    }
    const int offs[7] = {kTri7, kTri12, kTri33, kRect7, kRect12, kRect33, kNumNodes};
    const int n = offs[which + 1] - offs[which];
    std::memcpy(out, rules.data() + 3 * offs[which], (size_t) n * 3 * sizeof(double));
    return n;
}

}  // extern "C"

#include "kemcu_track_host.inc"
#include "kemcu_adjoint_host.inc"
#include "kemcu_robinhood_host.inc"
#include "kemcu_fftm_host.inc"
#include "kemcu_krylov_host.inc"
