// Fast multipole method (FFTM) for the direct sum: the device side.
//
// Conventions are the reference's (KFMMath.cc:219-330, 1056-1123): the regular and irregular
// solid harmonics R_n^m(x) = r^n P~_n^|m|(cos t) e^{i m phi}, I_n^m = r^-(n+1) P~_n^|m| e^{i m phi},
// P~_n^m = (-1)^m sqrt((n-m)!/(n+m)!) P_n^m (Schmidt semi-normalised with the Condon-Shortley
// phase), R_n^-m = conj(R_n^m); the multipole moments of a charge q at y about o are
// q conj(R_n^m(y - o)) (KFMElectrostaticMultipoleCalculatorAnalytic.cc:169-190) and the local
// coefficients L about c give phi(x) = sum L_n^m R_n^m(x - c)
// (KFMElectrostaticLocalCoefficientFieldCalculator.cc:285-310); moments of an element are those
// of its charge spread uniformly over it. The translation operators are the reference's
// response functions (Greengard & Rokhlin; KFMResponseKernel_3DLaplaceM2M.cc, ...M2L.cc,
// ...L2L.cc), formed on the host as real matrices.
//
// Storage. Sources have real charges, so M_n^-m = conj(M_n^m) and L_n^-m = conj(L_n^m): an
// expansion of degree p is kept as K = (p + 1)^2 reals, per n the real part of m = 0, then the
// real and imaginary parts of m = 1..n (fm_re / fm_im). Expansions are stored scaled by the side
// L of their cell: M^_n = M_n / L^(n+1), L^_n = L_n L^n, so that M2M, L2L and M2L are the same
// matrices at every level (they depend only on the offset in cell units and on the division
// ratio). The moments carry 1 / (4 pi eps0), so L2P gives the potential in volts.
#pragma once

namespace kemcu
{
constexpr int kFmMaxDegree = 15;  // P2M runs one lane per order m on half a warp
constexpr int kFmMaxQ = 9;        // Gauss-Legendre points per direction: exact to degree 17

__host__ __device__ __forceinline__ int fm_re(int n, int m)
{
    return m == 0 ? n * n : n * n + 2 * m - 1;
}
__host__ __device__ __forceinline__ int fm_im(int n, int m)
{
    return n * n + 2 * m;
}

// Gauss-Legendre rule on [0, 1] with q points (exact for polynomials of degree 2q - 1)
struct FmGl
{
    double x[kFmMaxQ], w[kFmMaxQ];
    int q;
};

// ------------------------------------------------------------------------- P2M
// Moments of every element about the centre of the cell that owns it, scaled by that cell's
// side: one element per half warp, lane m accumulating the orders m of degrees m..p over the
// nodes of an exact cubature (the moments are polynomials of degree <= p over the element):
// triangles on the collapsed square (Duffy map, Jacobian 1 - a), rectangles on the tensor
// square, wires on the segment. em[k][K] in the order `order` lists the elements; os[k] =
// (centre, 1 / side) of the owner cell.
__global__ void fm_p2m_kernel(const double* __restrict__ rec, const double* __restrict__ src,
                              const int* __restrict__ order, const double4* __restrict__ os, int n, int p, FmGl gl,
                              double* __restrict__ em)
{
    const int k = (int) ((blockIdx.x * (size_t) blockDim.x + threadIdx.x) >> 4);
    const int m = threadIdx.x & 15;
    if (k >= n || m > p)
        return;
    const int e = order[k];
    const double* r = rec + (size_t) e * rRecSize;
    const int type = (int) r[rType];
    const double4 o = os[k];
    const int K = (p + 1) * (p + 1);
    double are[kFmMaxDegree + 1], aim[kFmMaxDegree + 1];
    for (int j = 0; j <= kFmMaxDegree; j++)
        are[j] = aim[j] = 0.;
    const V3 p0 = v3(r[rP0], r[rP0 + 1], r[rP0 + 2]);
    const V3 ea = v3(r[rEa], r[rEa + 1], r[rEa + 2]);
    const V3 eb = v3(r[rEb], r[rEb + 1], r[rEb + 2]);
    const int na = gl.q, nb = type == kLineSegment ? 1 : gl.q;
    for (int ia = 0; ia < na; ia++)
        for (int ib = 0; ib < nb; ib++) {
            double wt;
            V3 y;
            if (type == kTriangle) {
                const double a = gl.x[ia], b = gl.x[ib] * (1. - a);
                wt = 2. * gl.w[ia] * gl.w[ib] * (1. - a);
                y = p0 + a * ea + b * eb;
            }
            else if (type == kRectangle) {
                wt = gl.w[ia] * gl.w[ib];
                y = p0 + gl.x[ia] * ea + gl.x[ib] * eb;
            }
            else {
                wt = gl.w[ia];
                y = p0 + gl.x[ia] * ea;  // rEa of a wire is P1 - P0
            }
            const double ux = (y.x - o.x) * o.w, uy = (y.y - o.y) * o.w, uz = (y.z - o.z) * o.w;
            const double r2 = ux * ux + uy * uy + uz * uz;
            // sectoral R_m^m = prod_k (-sqrt((2k-1)/(2k))) (x + i y)
            double sr = 1., si = 0.;
            for (int q = 1; q <= m; q++) {
                const double c = -sqrt((2. * q - 1.) / (2. * q));
                const double tr = c * (ux * sr - uy * si), ti = c * (ux * si + uy * sr);
                sr = tr;
                si = ti;
            }
            // vertical recurrence in n at fixed m
            double r1r = sr, r1i = si, r0r = 0., r0i = 0.;
            are[m] += wt * r1r;
            aim[m] -= wt * r1i;
            for (int nn = m + 1; nn <= p; nn++) {
                double nr, ni;
                if (nn == m + 1) {
                    const double c = sqrt(2. * m + 1.) * uz;
                    nr = c * r1r;
                    ni = c * r1i;
                }
                else {
                    const double inv = 1. / sqrt((double) (nn - m) * (nn + m));
                    const double c1 = (2. * nn - 1.) * uz * inv;
                    const double c2 = sqrt((double) (nn + m - 1) * (nn - m - 1)) * r2 * inv;
                    nr = c1 * r1r - c2 * r0r;
                    ni = c1 * r1i - c2 * r0i;
                }
                r0r = r1r;
                r0i = r1i;
                r1r = nr;
                r1i = ni;
                are[nn] += wt * nr;
                aim[nn] -= wt * ni;
            }
        }
    // charge of the element: sigma * area (wires: sigma * pi d L), with 1 / (4 pi eps0): the
    // record's prefactor (planar: area / (4 pi eps0); wire: pi d / (4 pi eps0), times its length)
    double q = src[e] * r[rPrefac] * o.w;
    if (type == kLineSegment)
        q *= r[rA];
    double* out = em + (size_t) k * K;
    for (int nn = m; nn <= p; nn++) {
        out[fm_re(nn, m)] = q * are[nn];
        if (m > 0)
            out[fm_im(nn, m)] = q * aim[nn];
    }
}

// Moments of every occupied owner cell for the sources src: the sum over its elements, in
// element order, of src times the element's unit-density moments (em, from fm_p2m_kernel with
// unit sources, kept from the tree's construction: the geometry fixes them). One warp per cell,
// lanes over the K coefficients; run[c] = (first, count) of owner cell key[c] in em / order.
template<int NR>
__global__ void fm_cell_sum_kernel(const double* __restrict__ em, const double* __restrict__ src,
                                   const int* __restrict__ order, const int* __restrict__ key,
                                   const int2* __restrict__ run, int ncells, int K, double* __restrict__ M,
                                   int nrhs, size_t n, size_t mstride)
{
    const int c = (int) ((blockIdx.x * (size_t) blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (c >= ncells)
        return;
    const int2 rg = run[c];
    for (int i = lane; i < K; i += 32) {
        // every cached moment read serves all right-hand sides
        double s[NR];
#pragma unroll
        for (int r = 0; r < NR; r++)
            s[r] = 0.;
        for (int j = 0; j < rg.y; j++) {
            const int e = order[rg.x + j];
            const double m = em[(size_t) (rg.x + j) * K + i];
#pragma unroll
            for (int r = 0; r < NR; r++)
                if (NR == 1 || r < nrhs)
                    s[r] += src[r * n + e] * m;
        }
#pragma unroll
        for (int r = 0; r < NR; r++)
            if (NR == 1 || r < nrhs)
                M[r * mstride + (size_t) key[c] * K + i] = s[r];
    }
}

__global__ void fm_fill_kernel(double* __restrict__ x, int n, double v)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        x[i] = v;
}

// ------------------------------------------------------------------------- translations
// y += sum over sources: op (K x K, column-major: op[col * K + row]) times x. One CTA per
// target; threads over the K rows.
//
// M2M: target = an occupied parent (list tgt), sources = its children (child cells flagged in
// occ), op per child position.
struct FmLevel
{
    int n;        // cells per dimension
    int div;      // cells of this level per cell of the level above (per dimension)
    long long base;  // index of the level's first cell in the level-concatenated cell arrays
    double side;  // cell side
};

__device__ __forceinline__ long long fm_cell(const FmLevel& L, int x, int y, int z)
{
    return L.base + ((long long) x * L.n + y) * L.n + z;
}

// sum_k op[k K + row] x[k]: one row of a column-major K x K operator times x, in four
// independent chains over k mod 4 (a single accumulator is a 2K-step dependent chain, the
// translation kernels' latency with one right-hand side)
__device__ __forceinline__ double fm_op_row(const double* __restrict__ op, int row, int K, const double* x)
{
    double a0 = 0., a1 = 0., a2 = 0., a3 = 0.;
    int k = 0;
    for (; k + 3 < K; k += 4) {
        a0 = fma(op[(size_t) k * K + row], x[k], a0);
        a1 = fma(op[(size_t) (k + 1) * K + row], x[k + 1], a1);
        a2 = fma(op[(size_t) (k + 2) * K + row], x[k + 2], a2);
        a3 = fma(op[(size_t) (k + 3) * K + row], x[k + 3], a3);
    }
    for (; k < K; k++)
        a0 = fma(op[(size_t) k * K + row], x[k], a0);
    return (a0 + a1) + (a2 + a3);
}

template<int NR>
__global__ void fm_m2m_kernel(const int* __restrict__ parents, int nparents, FmLevel Lp, FmLevel Lc,
                              const unsigned char* __restrict__ occ, const double* __restrict__ ops, int K,
                              double* __restrict__ M, int nrhs, size_t mstride)
{
    extern __shared__ double fm_x[];
    const int b = blockIdx.x;
    if (b >= nparents)
        return;
    const long long pc = parents[b];
    const int pz = (int) (pc % Lp.n), py = (int) ((pc / Lp.n) % Lp.n), px = (int) (pc / ((long long) Lp.n * Lp.n));
    const int d = Lc.div;
    double acc[NR];
#pragma unroll
    for (int r = 0; r < NR; r++)
        acc[r] = 0.;
    const int row = threadIdx.x;
    const int nr = NR == 1 ? 1 : nrhs;
    for (int cx = 0; cx < d; cx++)
        for (int cy = 0; cy < d; cy++)
            for (int cz = 0; cz < d; cz++) {
                const long long ci = fm_cell(Lc, px * d + cx, py * d + cy, pz * d + cz);
                if (!occ[ci])
                    continue;
                __syncthreads();
                for (int r = 0; r < nr; r++)
                    for (int i = threadIdx.x; i < K; i += blockDim.x)
                        fm_x[r * K + i] = M[r * mstride + ci * K + i];
                __syncthreads();
                if (row < K) {
                    const double* op = ops + (size_t) ((cx * d + cy) * d + cz) * K * K;
                    if (NR == 1)
                        acc[0] += fm_op_row(op, row, K, fm_x);
                    else if (nrhs == NR) {
                        for (int k = 0; k < K; k++) {
                            const double o = op[(size_t) k * K + row];
#pragma unroll
                            for (int r = 0; r < NR; r++)
                                acc[r] = fma(o, fm_x[r * K + k], acc[r]);
                        }
                    }
                    else {
                        for (int k = 0; k < K; k++) {
                            const double o = op[(size_t) k * K + row];
#pragma unroll
                            for (int r = 0; r < NR; r++)
                                if (r < nrhs)
                                    acc[r] = fma(o, fm_x[r * K + k], acc[r]);
                        }
                    }
                }
            }
    if (row < K)
#pragma unroll
        for (int r = 0; r < NR; r++)
            if (NR == 1 || r < nrhs)
                M[r * mstride + (Lp.base + pc) * K + row] += acc[r];
}

// L2L: every flagged child of level Lc receives its parent's local expansion
template<int NR>
__global__ void fm_l2l_kernel(const int* __restrict__ children, int nchildren, FmLevel Lp, FmLevel Lc,
                              const double* __restrict__ ops, int K, double* __restrict__ Lx, int nrhs,
                              size_t lstride)
{
    extern __shared__ double fm_x[];
    const int b = blockIdx.x;
    if (b >= nchildren)
        return;
    const long long cc = children[b];
    const int cz = (int) (cc % Lc.n), cy = (int) ((cc / Lc.n) % Lc.n), cx = (int) (cc / ((long long) Lc.n * Lc.n));
    const int d = Lc.div;
    const long long pi = fm_cell(Lp, cx / d, cy / d, cz / d);
    const int nr = NR == 1 ? 1 : nrhs;
    for (int r = 0; r < nr; r++)
        for (int i = threadIdx.x; i < K; i += blockDim.x)
            fm_x[r * K + i] = Lx[r * lstride + pi * K + i];
    __syncthreads();
    const int row = threadIdx.x;
    if (row >= K)
        return;
    const double* op = ops + (size_t) (((cx % d) * d + (cy % d)) * d + (cz % d)) * K * K;
    if (NR == 1)
        Lx[(Lc.base + cc) * K + row] += fm_op_row(op, row, K, fm_x);
    else {
        double acc[NR];
#pragma unroll
        for (int r = 0; r < NR; r++)
            acc[r] = 0.;
        for (int k = 0; k < K; k++) {
            const double o = op[(size_t) k * K + row];
#pragma unroll
            for (int r = 0; r < NR; r++)
                if (r < nrhs)
                    acc[r] = fma(o, fm_x[r * K + k], acc[r]);
        }
#pragma unroll
        for (int r = 0; r < NR; r++)
            if (r < nrhs)
                Lx[r * lstride + (Lc.base + cc) * K + row] += acc[r];
    }
}

// M2L at one level: every flagged target cell receives the moments of the occupied cells of its
// interaction list (children of its parent's neighbours that are not its own neighbours, the
// neighbours being the cells within zm cells in every direction), in a fixed order. op_index
// maps an offset (source - target, cell units, |o_i| <= R) to its operator, or -1.
template<int NR>
__global__ void fm_m2l_kernel(const int* __restrict__ targets, int ntargets, FmLevel L, int zm, int R,
                              const int* __restrict__ op_index, const unsigned char* __restrict__ occ,
                              const double* __restrict__ ops, int K, const double* __restrict__ M,
                              double* __restrict__ Lx, int nrhs, size_t mstride, size_t lstride)
{
    extern __shared__ double fm_x[];
    const int b = blockIdx.x;
    if (b >= ntargets)
        return;
    const long long tc = targets[b];
    const int tz = (int) (tc % L.n), ty = (int) ((tc / L.n) % L.n), tx = (int) (tc / ((long long) L.n * L.n));
    const int d = L.div;
    // parent-level neighbourhood in this level's cells: [lo, hi) per dimension
    int lo[3], hi[3];
    const int t[3] = {tx, ty, tz};
    for (int a = 0; a < 3; a++) {
        if (L.n == d) {  // the level below the root: every cell is a child of the root
            lo[a] = 0;
            hi[a] = L.n;
        }
        else {
            lo[a] = max(0, (t[a] / d - zm) * d);
            hi[a] = min(L.n, (t[a] / d + zm + 1) * d);
        }
    }
    const int row = threadIdx.x;
    double acc[NR];
#pragma unroll
    for (int r = 0; r < NR; r++)
        acc[r] = 0.;
    const int W = 2 * R + 1;
    for (int sx = lo[0]; sx < hi[0]; sx++)
        for (int sy = lo[1]; sy < hi[1]; sy++)
            for (int sz = lo[2]; sz < hi[2]; sz++) {
                const int ox = sx - tx, oy = sy - ty, oz = sz - tz;
                if (abs(ox) <= zm && abs(oy) <= zm && abs(oz) <= zm)
                    continue;
                const long long si = fm_cell(L, sx, sy, sz);
                if (!occ[si])
                    continue;
                const int oi = op_index[((ox + R) * W + (oy + R)) * W + (oz + R)];
                __syncthreads();
                for (int r = 0; r < (NR == 1 ? 1 : nrhs); r++)
                    for (int i = threadIdx.x; i < K; i += blockDim.x)
                        fm_x[r * K + i] = M[r * mstride + si * K + i];
                __syncthreads();
                if (row < K && oi >= 0) {
                    const double* op = ops + (size_t) oi * K * K;
                    if (NR == 1)
                        acc[0] += fm_op_row(op, row, K, fm_x);
                    else if (nrhs == NR) {
                        for (int k = 0; k < K; k++) {
                            const double o = op[(size_t) k * K + row];
#pragma unroll
                            for (int r = 0; r < NR; r++)
                                acc[r] = fma(o, fm_x[r * K + k], acc[r]);
                        }
                    }
                    else {
                        for (int k = 0; k < K; k++) {
                            const double o = op[(size_t) k * K + row];
#pragma unroll
                            for (int r = 0; r < NR; r++)
                                if (r < nrhs)
                                    acc[r] = fma(o, fm_x[r * K + k], acc[r]);
                        }
                    }
                }
            }
    if (row < K)
#pragma unroll
        for (int r = 0; r < NR; r++)
            if (NR == 1 || r < nrhs)
                Lx[r * lstride + (L.base + tc) * K + row] += acc[r];
}

// ------------------------------------------------------------------------- L2P
// potential and field of the local expansion Lh (scaled, K reals) at u = (x - c) / side: the
// regular harmonics by the same recurrences as P2M, streamed (no table), and the gradient by
// the ladder relations of the R_n^m (d/dz R_n^m = sqrt((n-m)(n+m)) R_(n-1)^m,
// (d/dx + i d/dy) R_n^m = sqrt((n-m)(n-m-1)) R_(n-1)^(m+1),
// (d/dx - i d/dy) R_n^m = -sqrt((n+m)(n+m-1)) R_(n-1)^(m-1), and for m = 0
// (d/dx - i d/dy) R_n^0 = sqrt(n(n-1)) conj(R_(n-1)^1)), which hold at the poles too.
__device__ __forceinline__ void fm_l2p(const double* Lh, int p, double ux, double uy, double uz, double inv_side,
                                       double* out4)
{
    const double r2 = ux * ux + uy * uy + uz * uz;
    double phi = 0., dpr = 0., dpi = 0., dz = 0.;
    double sr = 1., si = 0.;
    for (int m = 0; m <= p; m++) {
        if (m > 0) {
            const double c = -sqrt((2. * m - 1.) / (2. * m));
            const double tr = c * (ux * sr - uy * si), ti = c * (ux * si + uy * sr);
            sr = tr;
            si = ti;
        }
        const double w = m == 0 ? 1. : 2.;
        double r1r = sr, r1i = si, r0r = 0., r0i = 0.;
        for (int n = m; n <= p; n++) {
            if (n > m) {
                double nr, ni;
                if (n == m + 1) {
                    const double c = sqrt(2. * m + 1.) * uz;
                    nr = c * r1r;
                    ni = c * r1i;
                }
                else {
                    const double inv = 1. / sqrt((double) (n - m) * (n + m));
                    const double c1 = (2. * n - 1.) * uz * inv;
                    const double c2 = sqrt((double) (n + m - 1) * (n - m - 1)) * r2 * inv;
                    nr = c1 * r1r - c2 * r0r;
                    ni = c1 * r1i - c2 * r0i;
                }
                r0r = r1r;
                r0i = r1i;
                r1r = nr;
                r1i = ni;
            }
            // this R_n^m
            const double Rr = r1r, Ri = r1i;
            const double lr = Lh[fm_re(n, m)], li = m ? Lh[fm_im(n, m)] : 0.;
            phi += w * (lr * Rr - li * Ri);
            if (n < p) {
                const double a = sqrt((double) (n + 1 - m) * (n + 1 + m));
                const double zr = Lh[fm_re(n + 1, m)], zi = m ? Lh[fm_im(n + 1, m)] : 0.;
                dz += w * a * (zr * Rr - zi * Ri);
                if (m >= 1) {
                    const double b = sqrt((double) (n + 2 - m) * (n + 1 - m));
                    const double qr = Lh[fm_re(n + 1, m - 1)], qi = m - 1 ? Lh[fm_im(n + 1, m - 1)] : 0.;
                    dpr += b * (qr * Rr - qi * Ri);
                    dpi += b * (qr * Ri + qi * Rr);
                }
                {
                    const double c = sqrt((double) (n + m + 2) * (n + m + 1));
                    const double qr = Lh[fm_re(n + 1, m + 1)], qi = Lh[fm_im(n + 1, m + 1)];
                    // - conj(L) c conj(R) = -c conj(L R)
                    dpr -= c * (qr * Rr - qi * Ri);
                    dpi += c * (qr * Ri + qi * Rr);
                }
            }
        }
    }
    out4[0] = -dpr * inv_side;
    out4[1] = -dpi * inv_side;
    out4[2] = -dz * inv_side;
    out4[3] = phi;
}

// ------------------------------------------------------------------------- evaluation
// Points sorted by leaf cell; one CTA per occupied leaf (runs of equal leaf keys, the points
// outside the world cube left to the direct sum). Each thread takes points of the leaf in turn:
// the leaf's local expansion, plus the direct sum over the elements owned by the neighbours
// (within zm cells) of each of the leaf's ancestors (level 0 to the leaf's), in order of level,
// neighbour and element (the reference's direct-call lists,
// KFMElectrostaticFastMultipoleFieldSolver.cc:107-133), compensated (Kahan) like the direct
// sum. ANALYTIC evaluates every direct pair with the analytic integrals (as the reference's
// FFTM field solver does, KEBIFactory::MakeAnalytic()), else with the numeric policy.
struct FmTreeView
{
    FmLevel lv[12];
    int depth;       // the leaves' level
    int zm;
    double wx, wy, wz;  // world cube corner (minimum)
    const int* own_ptr;   // owned-element ranges per cell of every level (level-concatenated, +1)
    const int* own_elem;  // elements in owner order
};

//
// Register budget: the analytic integrals (rwg64) take up to 255 registers unbounded, which left
// two CTAs per SM; bounded for 4 resident CTAs they spill a little and the kernel runs 18 %
// faster (coax, 10^6 points, degree 8: 24.8 ms at depth 5, 17.6 ms at depth 6, against 30.2 and
// 22.3; 3 and 5 CTAs measured 25.5 / 18.8 and 25.8 / 17.2 ms; results bit-identical).
constexpr int kFmEvalMinBlocks = 4, kFmMatvecMinBlocks = 5;

template<bool POT, bool FIELD, bool ANALYTIC>
__global__ void __launch_bounds__(128, kFmEvalMinBlocks) fm_eval_kernel(const double* __restrict__ rec, const double* __restrict__ src,
                                                      const double* __restrict__ P, const int* __restrict__ run_key,
                                                      const int* __restrict__ run_off, const int* __restrict__ run_cnt,
                                                      int first_run, FmTreeView T, int p,
                                                      const double* __restrict__ Lx, double* __restrict__ out)
{
    extern __shared__ double fm_x[];
    const int b = blockIdx.x + first_run;
    const int key = run_key[b] - 1;  // leaf index within the leaf level (sorted keys are leaf + 1)
    const int off = run_off[b], cnt = run_cnt[b];
    const int K = (p + 1) * (p + 1);
    const FmLevel& Ld = T.lv[T.depth];
    for (int i = threadIdx.x; i < K; i += blockDim.x)
        fm_x[i] = Lx[(Ld.base + key) * K + i];
    __syncthreads();
    const int lz = key % Ld.n, ly = (key / Ld.n) % Ld.n, lx = key / (Ld.n * Ld.n);
    const double cx = T.wx + (lx + .5) * Ld.side, cy = T.wy + (ly + .5) * Ld.side, cz = T.wz + (lz + .5) * Ld.side;
    const double inv_side = 1. / Ld.side;
    for (int k = threadIdx.x; k < cnt; k += blockDim.x) {
        const int i = off + k;
        const V3 x = v3(P[3 * i], P[3 * i + 1], P[3 * i + 2]);
        double far[4];
        fm_l2p(fm_x, p, (x.x - cx) * inv_side, (x.y - cy) * inv_side, (x.z - cz) * inv_side, inv_side, far);
        double s[4] = {0., 0., 0., 0.}, c[4] = {0., 0., 0., 0.};
        for (int l = 0; l <= T.depth; l++) {
            const FmLevel& L = T.lv[l];
            // the leaf's ancestor at level l
            int ax = lx, ay = ly, az = lz;
            for (int q = T.depth; q > l; q--) {
                ax /= T.lv[q].div;
                ay /= T.lv[q].div;
                az /= T.lv[q].div;
            }
            for (int sx = max(0, ax - T.zm); sx <= min(L.n - 1, ax + T.zm); sx++)
                for (int sy = max(0, ay - T.zm); sy <= min(L.n - 1, ay + T.zm); sy++)
                    for (int sz = max(0, az - T.zm); sz <= min(L.n - 1, az + T.zm); sz++) {
                        const long long ci = fm_cell(L, sx, sy, sz);
                        const int e0 = T.own_ptr[ci], e1 = T.own_ptr[ci + 1];
                        for (int j = e0; j < e1; j++) {
                            const int e = T.own_elem[j];
                            const double* r = rec + (size_t) e * rRecSize;
                            Out4 v;
                            if (ANALYTIC) {
                                const int type = (int) r[rType];
                                v = type == kLineSegment ? line_analytic<POT, FIELD>(r, x)
                                    : type == kTriangle  ? rwg64<3, POT, FIELD>(r, x)
                                                         : rwg64<4, POT, FIELD>(r, x);
                            }
                            else
                                v = epi<false, POT, FIELD>(r, x);
                            const double sg = src[e];
                            const double t4[4] = {v.ex * sg, v.ey * sg, v.ez * sg, v.phi * sg};
#pragma unroll
                            for (int q = 0; q < 4; q++) {
                                const double yk = t4[q] - c[q];
                                const double t = s[q] + yk;
                                c[q] = (t - s[q]) - yk;
                                s[q] = t;
                            }
                        }
                    }
        }
        double* o = out + 4 * (size_t) i;
        o[0] = FIELD ? s[0] + far[0] : 0.;
        o[1] = FIELD ? s[1] + far[1] : 0.;
        o[2] = FIELD ? s[2] + far[2] : 0.;
        o[3] = POT ? s[3] + far[3] : 0.;
    }
}

// FFTM matrix-vector product (the reference's KFastMultipoleMatrixGenerator: the dense part from
// the local expansions, KFMElectrostaticBoundaryIntegrator.hh:355-386, the sparse part from the
// default numeric integrator on the direct-call lists): row t of y is the local expansion of the
// leaf holding element t's collocation point (its potential, or for a Neumann row its field
// along the normal) plus the matrix entries entry() of the elements owned by the neighbours of
// the leaf's ancestors times x, in the order of fm_eval_kernel. One CTA per run of targets
// sorted by leaf (tgt_order lists the elements). NR right-hand sides (nrhs of them used) share
// every entry: x, y are nrhs x n, the local expansions of right-hand side r at Lx + r * lstride.
// (bounded for 5 resident CTAs: 7.35 ms per coax matvec against 8.9 ms unbounded, 7.6 at 4)
template<int NR>
__global__ void __launch_bounds__(128, kFmMatvecMinBlocks) fm_matvec_kernel(const double* __restrict__ rec,
                                                        const TargetRec* __restrict__ tgt,
                                                        const int* __restrict__ tgt_order,
                                                        const int* __restrict__ run_key, const int* __restrict__ run_off,
                                                        const int* __restrict__ run_cnt, FmTreeView T, int p,
                                                        const double* __restrict__ Lx, size_t lstride, int n,
                                                        int nrhs, const double* __restrict__ x, double* __restrict__ y)
{
    extern __shared__ double fm_x[];
    const int b = blockIdx.x;
    const int key = run_key[b] - 1;
    const int off = run_off[b], cnt = run_cnt[b];
    const int K = (p + 1) * (p + 1);
    const FmLevel& Ld = T.lv[T.depth];
    for (int r = 0; r < nrhs; r++)
        for (int i = threadIdx.x; i < K; i += blockDim.x)
            fm_x[r * K + i] = Lx[r * lstride + (Ld.base + key) * K + i];
    __syncthreads();
    const int lz = key % Ld.n, ly = (key / Ld.n) % Ld.n, lx = key / (Ld.n * Ld.n);
    const double cx = T.wx + (lx + .5) * Ld.side, cy = T.wy + (ly + .5) * Ld.side, cz = T.wz + (lz + .5) * Ld.side;
    const double inv_side = 1. / Ld.side;
    for (int k = threadIdx.x; k < cnt; k += blockDim.x) {
        const int ti = tgt_order[off + k];
        const TargetRec t = tgt[ti];
        const V3 C = v3(t.cen[0], t.cen[1], t.cen[2]);
        double s[NR], c[NR];
#pragma unroll
        for (int r = 0; r < NR; r++)
            s[r] = c[r] = 0.;
        for (int l = 0; l <= T.depth; l++) {
            const FmLevel& L = T.lv[l];
            int ax = lx, ay = ly, az = lz;
            for (int q = T.depth; q > l; q--) {
                ax /= T.lv[q].div;
                ay /= T.lv[q].div;
                az /= T.lv[q].div;
            }
            for (int sx = max(0, ax - T.zm); sx <= min(L.n - 1, ax + T.zm); sx++)
                for (int sy = max(0, ay - T.zm); sy <= min(L.n - 1, ay + T.zm); sy++)
                    for (int sz = max(0, az - T.zm); sz <= min(L.n - 1, az + T.zm); sz++) {
                        const long long ci = fm_cell(L, sx, sy, sz);
                        const int e0 = T.own_ptr[ci], e1 = T.own_ptr[ci + 1];
                        for (int j = e0; j < e1; j++) {
                            const int e = T.own_elem[j];
                            const double a = entry<false>(rec + (size_t) e * rRecSize, t, C);
#pragma unroll
                            for (int r = 0; r < NR; r++)
                                if (r < nrhs) {
                                    const double yk = a * x[(size_t) r * n + e] - c[r];
                                    const double tt = s[r] + yk;
                                    c[r] = (tt - s[r]) - yk;
                                    s[r] = tt;
                                }
                        }
                    }
        }
        const double ux = (C.x - cx) * inv_side, uy = (C.y - cy) * inv_side, uz = (C.z - cz) * inv_side;
#pragma unroll
        for (int r = 0; r < NR; r++)
            if (r < nrhs) {
                double far[4];
                fm_l2p(fm_x + r * K, p, ux, uy, uz, inv_side, far);
                const double fv =
                    t.neumann == 0. ? far[3] : far[0] * t.normal[0] + far[1] * t.normal[1] + far[2] * t.normal[2];
                y[(size_t) r * n + ti] = s[r] + fv;
            }
    }
}

// The near part of the matrix kept as a sparse matrix (fm_build_near): per run of targets (one
// leaf) its direct elements, col[coloff[b] .. + ncol[b]], in fm_matvec_kernel's order, and the
// entries of the run's cnt targets column-major at val[valoff[b] + j cnt + k].
struct FmNear
{
    const long long* coloff;
    const int* ncol;
    const long long* valoff;
    const int* col;
    double* val;
};

// the entries entry() of every run's targets with its direct elements; one CTA per run, its
// threads over the (element, target) pairs of the run
__global__ void __launch_bounds__(256) fm_near_fill_kernel(const double* __restrict__ rec,
                                                           const TargetRec* __restrict__ tgt,
                                                           const int* __restrict__ tgt_order,
                                                           const int* __restrict__ run_off,
                                                           const int* __restrict__ run_cnt,
                                                           const long long* __restrict__ coloff,
                                                           const int* __restrict__ ncol,
                                                           const long long* __restrict__ valoff,
                                                           const int* __restrict__ col, double* __restrict__ val)
{
    const int b = blockIdx.x;
    const int off = run_off[b], cnt = run_cnt[b], nc = ncol[b];
    const int* cb = col + coloff[b];
    double* vb = val + valoff[b];
    const long long pairs = (long long) nc * cnt;
    for (long long q = threadIdx.x; q < pairs; q += blockDim.x) {
        const int j = (int) (q / cnt), k = (int) (q % cnt);
        const TargetRec t = tgt[tgt_order[off + k]];
        vb[q] = entry<false>(rec + (size_t) cb[j] * rRecSize, t, v3(t.cen[0], t.cen[1], t.cen[2]));
    }
}

// fm_matvec_kernel with the near part read from the sparse matrix: the same sums in the same
// order (compensated, over the run's columns), plus the local expansion of the leaf
template<int NR>
__global__ void __launch_bounds__(128, kFmMatvecMinBlocks) fm_matvec_near_kernel(
    const TargetRec* __restrict__ tgt, const int* __restrict__ tgt_order, const int* __restrict__ run_key,
    const int* __restrict__ run_off, const int* __restrict__ run_cnt, FmNear nr, FmTreeView T, int p,
    const double* __restrict__ Lx, size_t lstride, int n, int nrhs, const double* __restrict__ x,
    double* __restrict__ y)
{
    extern __shared__ double fm_x[];
    const int b = blockIdx.x;
    const int key = run_key[b] - 1;
    const int off = run_off[b], cnt = run_cnt[b], nc = nr.ncol[b];
    const int* cb = nr.col + nr.coloff[b];
    const double* vb = nr.val + nr.valoff[b];
    const int K = (p + 1) * (p + 1);
    const FmLevel& Ld = T.lv[T.depth];
    for (int r = 0; r < nrhs; r++)
        for (int i = threadIdx.x; i < K; i += blockDim.x)
            fm_x[r * K + i] = Lx[r * lstride + (Ld.base + key) * K + i];
    __syncthreads();
    const int lz = key % Ld.n, ly = (key / Ld.n) % Ld.n, lx = key / (Ld.n * Ld.n);
    const double cx = T.wx + (lx + .5) * Ld.side, cy = T.wy + (ly + .5) * Ld.side, cz = T.wz + (lz + .5) * Ld.side;
    const double inv_side = 1. / Ld.side;
    for (int k = threadIdx.x; k < cnt; k += blockDim.x) {
        const int ti = tgt_order[off + k];
        const TargetRec t = tgt[ti];
        double s[NR], c[NR];
#pragma unroll
        for (int r = 0; r < NR; r++)
            s[r] = c[r] = 0.;
        for (int j = 0; j < nc; j++) {
            const int e = cb[j];
            const double a = vb[(size_t) j * cnt + k];
#pragma unroll
            for (int r = 0; r < NR; r++)
                if (r < nrhs) {
                    const double yk = a * x[(size_t) r * n + e] - c[r];
                    const double tt = s[r] + yk;
                    c[r] = (tt - s[r]) - yk;
                    s[r] = tt;
                }
        }
        const double ux = (t.cen[0] - cx) * inv_side, uy = (t.cen[1] - cy) * inv_side, uz = (t.cen[2] - cz) * inv_side;
#pragma unroll
        for (int r = 0; r < NR; r++)
            if (r < nrhs) {
                double far[4];
                fm_l2p(fm_x + r * K, p, ux, uy, uz, inv_side, far);
                const double fv =
                    t.neumann == 0. ? far[3] : far[0] * t.normal[0] + far[1] * t.normal[1] + far[2] * t.normal[2];
                y[(size_t) r * n + ti] = s[r] + fv;
            }
    }
}

// leaf key (leaf index + 1, or 0 outside the world cube) and index of every point
__global__ void fm_leaf_kernel(const double* __restrict__ P, int n, double wx, double wy, double wz, double side,
                               int nd, int* __restrict__ key, int* __restrict__ idx)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const double fx = (P[3 * i] - wx) / side, fy = (P[3 * i + 1] - wy) / side, fz = (P[3 * i + 2] - wz) / side;
    int k = 0;
    if (fx >= 0. && fy >= 0. && fz >= 0. && fx <= nd && fy <= nd && fz <= nd) {
        const int ix = min(nd - 1, (int) fx), iy = min(nd - 1, (int) fy), iz = min(nd - 1, (int) fz);
        k = (ix * nd + iy) * nd + iz + 1;
    }
    key[i] = k;
    idx[i] = i;
}

// flags the target cells of every level: the ancestors of the leaves of the sorted runs
__global__ void fm_flag_targets_kernel(const int* __restrict__ run_key, int nruns, FmTreeView T,
                                       unsigned char* __restrict__ tflag)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nruns)
        return;
    const int key = run_key[b] - 1;
    if (key < 0)
        return;
    const FmLevel& Ld = T.lv[T.depth];
    int ax = key / (Ld.n * Ld.n), ay = (key / Ld.n) % Ld.n, az = key % Ld.n;
    for (int l = T.depth; l >= 1; l--) {
        tflag[fm_cell(T.lv[l], ax, ay, az)] = 1;
        ax /= T.lv[l].div;
        ay /= T.lv[l].div;
        az /= T.lv[l].div;
    }
}

// compacts the flagged cells of one level into a list (cell index within the level)
__global__ void fm_compact_kernel(const unsigned char* __restrict__ flag, FmLevel L, int* __restrict__ list,
                                  unsigned* __restrict__ count)
{
    const long long ncell = (long long) L.n * L.n * L.n;
    for (long long c = blockIdx.x * (long long) blockDim.x + threadIdx.x; c < ncell;
         c += (long long) gridDim.x * blockDim.x)
        if (flag[L.base + c])
            list[atomicAdd(count, 1u)] = (int) c;
}
}  // namespace kemcu
