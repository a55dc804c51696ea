// Device-side element integrals for the electrostatic BEM hot path (sm_100a).
//
// One element-point interaction (EPI) = the field and/or potential of one charged element
// with unit charge density at one point. The numeric policy of the reference picks the rule
// per (element, point) from the distance ratio |P - centroid| / size
// (KElectrostaticCubatureTriangleIntegrator.cc:453-522, ...RectangleIntegrator.cc:462-520,
// ...QuadratureLineSegmentIntegrator.cc:193-240):
//
//   triangle  : RWG analytic <= 3.42 < 33-point <= 30.4 < 12-point <= 131.4 < 7-point
//   rectangle : RWG analytic <= 4.6  < 33-point <= 44.6 < 12-point <= 196.2 < 7-point
//   line      : analytic     <= 2    < 16-node Gauss <= 27.7 < 4-node Gauss
//
// The band test is evaluated with the same FP64 operations and rounding (no FMA
// contraction) as the reference so that band boundaries agree bit for bit.
//
// Cubature bands are evaluated in FP64 in a quadratic form (cubq below): with the element's
// centroid c, d = P - c and node offsets o_k = s'_k (A N1) + t'_k (B N2) (s', t' relative to
// the rule's centroid), |P - Q_k|^2 = R^2 + s' C1 + t' C2 + s'^2 |A N1|^2 + 2 s't' (A N1).(B N2)
// + t'^2 |B N2|^2 with per-pair C1 = -2 d.(A N1), C2 = -2 d.(B N2): five FMAs per node instead of
// forming the node and the difference vector, and the field sum collapses to
// d S0 - (A N1) Ss - (B N2) St with three scalar node sums. Two reciprocal square roots, both
// from the FP32-class hardware estimate (rsqrt.approx.f64, ~2^-23 relative):
//   * FP64  -- refined by two FP64 Newton steps (within one unit in the last place);
//   * MIXED -- refined by one FP64 Newton step (~1e-13 relative).
// RWG near-field integrals and the analytic line segment are FP64 in both forms.
#pragma once

#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

namespace kemcu
{

enum Shape : int
{
    kTriangle = 0,
    kRectangle = 1,
    kLineSegment = 2
};

// Element record in device memory, 32 doubles (256 B, one element per 2 x 128 B lines).
// Offsets into the record:
enum Rec : int
{
    rA = 0,        // side length A (line: length)
    rB = 1,        // side length B (line: diameter)
    rP0 = 2,       // P0 xyz (line: P0)
    rN1 = 5,       // N1 xyz (line: P1)
    rN2 = 8,       // N2 xyz
    rEa = 11,      // A * N1 (line: P1 - P0)
    rEb = 14,      // B * N2
    rCen = 17,     // centroid (reference formula)
    rAA = 20,      // |A N1|^2      (quadratic-form coefficients of the cubature node
    rAB2 = 21,     // 2 (A N1).(B N2) distances; lines: unused)
    rBB = 22,      // |B N2|^2
    rInvSize = 23, // 1 / size for the distance ratio
    rPrefac = 24,  // area / (4 pi eps0)   (line: diameter / (4 eps0))
    rType = 25,    // shape as double
    rCen2 = 26,    // centroid xyz as KRectangle::Centroid()/KSolidAngle form it (rectangles; else = rCen)
    rCut = 29,     // 3 squared distances (cut / invSize)^2 of the band boundaries, nearest first
    rRecSize = 32
};

static_assert(rCut + 3 <= rRecSize, "element record layout overflows its 32 slots");

struct Constants
{
    double one_over_four_pi_eps0;
    double eps0;
    double pi;
};

// Cubature rules in barycentric-like (s, t) form: node = P0 + s * (A N1) + t * (B N2),
// weights normalised to 1 over the element (tables in kemcu_tables.cuh). Node offsets of the
// rules in the tables below:
//   tri7 [0,7) tri12 [7,19) tri33 [19,52) rect7 [52,59) rect12 [59,71) rect33 [71,104)
// Line Gauss-Legendre half rules (x, w) pairs: gl4 [0,2), gl16 [2,10).
constexpr int kTri7 = 0, kTri12 = 7, kTri33 = 19, kRect7 = 52, kRect12 = 59, kRect33 = 71, kNumNodes = 104;
// per node, relative to the rule centroid (1/3, 1/3) or (1/2, 1/2):
//   -2 s', -2 t', s'^2, s't', t'^2, w, w s', w t'
constexpr int kQ = 8;
__constant__ double c_q[kNumNodes * kQ];
// The rectangle rules are centrally symmetric: node pairs (o, -o) of equal weight, plus at
// most one node at the centroid. Per pair, the values above for the + node; offsets of the
// three rules' pairs and the centroid-node weights (rect7, rect33):
constexpr int kPair7 = 0, kPair12 = 3, kPair33 = 9, kNumPairs = 25;
__constant__ double c_qp[kNumPairs * kQ];
__constant__ double c_qc[2];
// the same three tables rounded to FP32, for the FP32 far-field form (cubq32, cubq_pairs32)
__constant__ float c_q32[kNumNodes * kQ];
__constant__ float c_qp32[kNumPairs * kQ];
__constant__ float c_qc32[2];
__constant__ double c_gl[10 * 2];
__constant__ Constants c_k;

// ------------------------------------------------------------------------- helpers
struct V3
{
    double x, y, z;
};
__device__ __forceinline__ V3 v3(double x, double y, double z)
{
    return V3{x, y, z};
}
__device__ __forceinline__ V3 operator-(V3 a, V3 b)
{
    return v3(a.x - b.x, a.y - b.y, a.z - b.z);
}
__device__ __forceinline__ V3 operator+(V3 a, V3 b)
{
    return v3(a.x + b.x, a.y + b.y, a.z + b.z);
}
__device__ __forceinline__ V3 operator*(double s, V3 a)
{
    return v3(s * a.x, s * a.y, s * a.z);
}
__device__ __forceinline__ double dot(V3 a, V3 b)
{
    return a.x * b.x + a.y * b.y + a.z * b.z;
}
__device__ __forceinline__ V3 cross(V3 a, V3 b)
{
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ double norm(V3 a)
{
    return sqrt(dot(a, a));
}
__device__ __forceinline__ V3 ld3(const double* p)
{
    return v3(p[0], p[1], p[2]);
}
// sum of squares in the reference's left-to-right order without FMA contraction
__device__ __forceinline__ double sumsq_rn(double a, double b, double c)
{
    return __dadd_rn(__dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b)), __dmul_rn(c, c));
}

struct Out4
{
    double ex, ey, ez, phi;
};

// ------------------------------------------------------------------------- band test
// 0 = analytic (RWG / analytic line), 1 = 33-point / 16-node, 2 = 12-point / 4-node, 3 = 7-point
// The squared centre distance is compared with the squared cut distances stored in the record;
// only when it lies within a relative 1e-12 of a cut is the reference's exact expression
// ratio = sqrt(r2) * (1 / size) evaluated, so the decision is the reference's bit for bit.
__device__ __forceinline__ int band_exact(const double* e, double r2)
{
    const double ratio = __dmul_rn(__dsqrt_rn(r2), e[rInvSize]);
    const int type = (int) e[rType];
    if (type == kTriangle)
        return ratio > 131.4 ? 3 : ratio > 30.4 ? 2 : ratio > 3.42 ? 1 : 0;
    if (type == kRectangle)
        return ratio > 196.2 ? 3 : ratio > 44.6 ? 2 : ratio > 4.6 ? 1 : 0;
    return ratio > 27.7 ? 2 : ratio > 2. ? 1 : 0;
}

// The band of (element, P); also returns d = P - centroid and r2 = |d|^2 (formed as the
// reference forms the distance ratio), which the cubature code re-uses.
__device__ __forceinline__ int band_of(const double* e, V3 P, V3& d, double& r2)
{
    const double dx = __dadd_rn(e[rCen], -P.x);
    const double dy = __dadd_rn(e[rCen + 1], -P.y);
    const double dz = __dadd_rn(e[rCen + 2], -P.z);
    r2 = sumsq_rn(dx, dy, dz);
    d = v3(-dx, -dy, -dz);
    // outside a relative 1e-12 of every cut the fast comparison is the reference's decision
    const double lo = r2 * (1. - 1e-12), hi = r2 * (1. + 1e-12);
    int band = 0;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const double c = e[rCut + k];
        if (lo > c)
            band = k + 1;
        else if (hi >= c)
            return band_exact(e, r2);
        else
            break;
    }
    return band;
}
__device__ __forceinline__ int band_of(const double* e, V3 P)
{
    V3 d;
    double r2;
    return band_of(e, P, d, r2);
}

// ------------------------------------------------------------------------- cubature
// Sum over nodes of w (P-Q)/|P-Q|^3 and w/|P-Q| times area/(4 pi eps0)
// (Potential_TriNP / ElectricField_TriNP, KElectrostaticCubatureTriangleIntegrator.cc:271-450;
// the rectangle versions are identical in form), in the quadratic form described at the top.
//
// Twice the FP64 reciprocal square root, from the hardware approximation y0 plus one
// Newton-Raphson step written as 2 y1 = y0 (3 - x y0^2) (quadratic convergence: relative
// error ~1.5 e0^2). Returning 2 y1 saves the halving (three FP64 operations instead of
// four); callers fold the factors 1/2 (potential) and 1/8 (field) into their element sums.
// MIXED form only.
__device__ __forceinline__ double rsqrt2_fast(double x)
{
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    return y * fma(-(x * y), y, 3.);
}
// Twice the FP64 reciprocal square root to within about one unit in the last place: the
// MIXED estimate refined by a second Newton step on z = 2y, 2 y2 = z + (z/8) (4 - x z^2)
// (the correction is ~1e-13 of z, so its own rounding stays below half an ulp). FP64 form.
__device__ __forceinline__ double rsqrt2_acc(double x)
{
    const double z = rsqrt2_fast(x);
    const double e4 = fma(-(x * z), z, 4.);
    return fma(0.125 * z, e4, z);
}
// the reciprocal square root of a form, returned doubled (folded back by kPotScale/kFieldScale)
template<bool FAST> __device__ __forceinline__ double irsq(double x)
{
    return FAST ? rsqrt2_fast(x) : rsqrt2_acc(x);
}
template<bool FAST> constexpr double kPotScale = 0.5;
template<bool FAST> constexpr double kFieldScale = 0.125;

// Nodes per unrolled group of the node loop (rules whose size it divides are run as a loop
// over groups, the others fully unrolled). The reciprocal square root of the MIXED form is
// straight-line code, so a fully unrolled 33-point rule lets the compiler interleave all 33
// nodes and spill; a loop over groups bounds that window.
#ifndef KEMCU_GROUP
#define KEMCU_GROUP 11
#endif

// N nodes of the rule starting at node OFF (both compile-time, so the rule constants are
// constant-bank operands with fixed offsets within a group)
template<int N, int OFF, bool POT, bool FIELD, bool FAST>
__device__ __forceinline__ Out4 cubq(const double* e, V3 d, double R2)
{
    const V3 a = ld3(e + rEa), b = ld3(e + rEb);
    const double C1 = dot(d, a), C2 = dot(d, b);  // the rule tables carry the factor -2
    const double aa = e[rAA], ab2 = e[rAB2], bb = e[rBB];
    double sp = 0., s0 = 0., ss = 0., st = 0.;
    constexpr int G = N % KEMCU_GROUP == 0 ? KEMCU_GROUP : N;
#pragma unroll 1
    for (int g = 0; g < N / G; g++) {
        const double* cg = c_q + kQ * (OFF + g * G);
#pragma unroll
        for (int k = 0; k < G; k++) {
            const double* c = cg + kQ * k;
            double q2 = fma(c[0], C1, R2);
            q2 = fma(c[1], C2, q2);
            q2 = fma(c[2], aa, q2);
            q2 = fma(c[3], ab2, q2);
            q2 = fma(c[4], bb, q2);
            const double ir = irsq<FAST>(q2);
            if (POT)
                sp = fma(c[5], ir, sp);
            if (FIELD) {
                const double ir3 = ir * ir * ir;
                s0 = fma(c[5], ir3, s0);
                ss = fma(c[6], ir3, ss);
                st = fma(c[7], ir3, st);
            }
        }
    }
    const double pf = e[rPrefac];
    Out4 o{0., 0., 0., 0.};
    if (POT)
        o.phi = (kPotScale<FAST> * pf) * sp;
    if (FIELD) {
        const double pff = kFieldScale<FAST> * pf;
        o.ex = pff * (d.x * s0 - a.x * ss - b.x * st);
        o.ey = pff * (d.y * s0 - a.y * ss - b.y * st);
        o.ez = pff * (d.z * s0 - a.z * ss - b.z * st);
    }
    return o;
}

// Centrally symmetric rules (rectangles): with L = s' C1 + t' C2 and
// Q = R^2 + s'^2 |A N1|^2 + ... the pair's squared distances are Q + L and Q - L, and the two
// nodes' field terms combine as w (ir3+ + ir3-) into S0 and w s' (ir3+ - ir3-) into Ss, St:
// 26 FP64 operations per pair instead of 30 for two nodes. NP pairs from pair POFF, plus the
// centroid node of weight c_qc[CENTER] when CENTER >= 0.
#ifndef KEMCU_PAIR_GROUP
#define KEMCU_PAIR_GROUP 16
#endif
template<int NP, int POFF, int CENTER, bool POT, bool FIELD, bool FAST>
__device__ __forceinline__ Out4 cubq_pairs(const double* e, V3 d, double R2)
{
    const V3 a = ld3(e + rEa), b = ld3(e + rEb);
    const double C1 = dot(d, a), C2 = dot(d, b);  // the rule tables carry the factor -2
    const double aa = e[rAA], ab2 = e[rAB2], bb = e[rBB];
    double sp = 0., s0 = 0., ss = 0., st = 0.;
    if (CENTER >= 0) {
        const double ir = irsq<FAST>(R2);
        sp = c_qc[CENTER] * ir;
        s0 = c_qc[CENTER] * (ir * ir * ir);
    }
    constexpr int G = NP % KEMCU_PAIR_GROUP == 0 ? KEMCU_PAIR_GROUP : NP;
#pragma unroll 1
    for (int g = 0; g < NP / G; g++) {
        const double* cg = c_qp + kQ * (POFF + g * G);
#pragma unroll
        for (int k = 0; k < G; k++) {
            const double* c = cg + kQ * k;
            const double L = fma(c[1], C2, c[0] * C1);
            double Q = fma(c[2], aa, R2);
            Q = fma(c[3], ab2, Q);
            Q = fma(c[4], bb, Q);
            const double irp = irsq<FAST>(Q + L);
            const double irm = irsq<FAST>(Q - L);
            if (POT)
                sp = fma(c[5], irp + irm, sp);
            if (FIELD) {
                const double i3p = irp * irp * irp, i3m = irm * irm * irm;
                s0 = fma(c[5], i3p + i3m, s0);
                const double dd = i3p - i3m;
                ss = fma(c[6], dd, ss);
                st = fma(c[7], dd, st);
            }
        }
    }
    const double pf = e[rPrefac];
    Out4 o{0., 0., 0., 0.};
    if (POT)
        o.phi = (kPotScale<FAST> * pf) * sp;
    if (FIELD) {
        const double pff = kFieldScale<FAST> * pf;
        o.ex = pff * (d.x * s0 - a.x * ss - b.x * st);
        o.ey = pff * (d.y * s0 - a.y * ss - b.y * st);
        o.ez = pff * (d.z * s0 - a.z * ss - b.z * st);
    }
    return o;
}

// ------------------------------------------------------------------------- FP32 far field
// The FP32 form of the cubature bands (precision KEMCU_FP32): the per-element set-up stays FP64
// (d = P - centroid, R^2 from the band test, R^-1 to an ulp), and every node works on the
// distance relative to R: with C1, C2 and the quadratic-form coefficients divided by R^2 (then
// rounded to FP32), |P - Q_k|^2 / R^2 = 1 + x_k, x_k = c0 C1' + c1 C2' + c2 |A N1|^2' + ...
// (five FP32 FMAs), and R / |P - Q_k| = rsqrt(1 + x_k) from the FP32 hardware estimate. The
// node sums run in FP32 on values near 1 (the weights sum to 1), then scale back in FP64:
// phi = area/(4 pi eps0) R^-1 sum w f, E = area/(4 pi eps0) R^-3 (d S0 - A N1 Ss - B N2 St).
// Relative error per element-point pair ~1e-7 (FP32 rounding of x and of the estimate); the
// element sums are compensated in FP64 by the callers.
__device__ __forceinline__ float rsqrt_f32(float x)
{
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

struct Far32
{
    float u1, u2, aa, ab, bb;  // C1 / R^2, C2 / R^2, |A N1|^2 / R^2, 2 (A N1).(B N2) / R^2, |B N2|^2 / R^2
    double ir;                 // R^-1
};

__device__ __forceinline__ Far32 far32_setup(const double* e, V3 d, double R2, V3 a, V3 b)
{
    Far32 f;
    f.ir = 0.5 * rsqrt2_acc(R2);
    const double inv = f.ir * f.ir;
    f.u1 = (float) (dot(d, a) * inv);
    f.u2 = (float) (dot(d, b) * inv);
    f.aa = (float) (e[rAA] * inv);
    f.ab = (float) (e[rAB2] * inv);
    f.bb = (float) (e[rBB] * inv);
    return f;
}

template<bool POT, bool FIELD>
__device__ __forceinline__ Out4 far32_finish(const double* e, V3 d, V3 a, V3 b, const Far32& f, float sp, float s0,
                                             float ss, float st)
{
    const double pf = e[rPrefac];
    Out4 o{0., 0., 0., 0.};
    if (POT)
        o.phi = (pf * f.ir) * (double) sp;
    if (FIELD) {
        const double pff = pf * (f.ir * f.ir * f.ir);
        const double S0 = s0, Ss = ss, St = st;
        o.ex = pff * (d.x * S0 - a.x * Ss - b.x * St);
        o.ey = pff * (d.y * S0 - a.y * Ss - b.y * St);
        o.ez = pff * (d.z * S0 - a.z * Ss - b.z * St);
    }
    return o;
}

template<int N, int OFF, bool POT, bool FIELD>
__device__ __forceinline__ Out4 cubq32(const double* e, V3 d, double R2)
{
    const V3 a = ld3(e + rEa), b = ld3(e + rEb);
    const Far32 f = far32_setup(e, d, R2, a, b);
    float sp = 0.f, s0 = 0.f, ss = 0.f, st = 0.f;
    constexpr int G = N % KEMCU_GROUP == 0 ? KEMCU_GROUP : N;
#pragma unroll 1
    for (int g = 0; g < N / G; g++) {
        const float* cg = c_q32 + kQ * (OFF + g * G);
#pragma unroll
        for (int k = 0; k < G; k++) {
            const float* c = cg + kQ * k;
            float x = c[4] * f.bb;
            x = fmaf(c[3], f.ab, x);
            x = fmaf(c[2], f.aa, x);
            x = fmaf(c[1], f.u2, x);
            x = fmaf(c[0], f.u1, x);
            const float r = rsqrt_f32(1.f + x);
            if (POT)
                sp = fmaf(c[5], r, sp);
            if (FIELD) {
                const float r3 = r * r * r;
                s0 = fmaf(c[5], r3, s0);
                ss = fmaf(c[6], r3, ss);
                st = fmaf(c[7], r3, st);
            }
        }
    }
    return far32_finish<POT, FIELD>(e, d, a, b, f, sp, s0, ss, st);
}

template<int NP, int POFF, int CENTER, bool POT, bool FIELD>
__device__ __forceinline__ Out4 cubq_pairs32(const double* e, V3 d, double R2)
{
    const V3 a = ld3(e + rEa), b = ld3(e + rEb);
    const Far32 f = far32_setup(e, d, R2, a, b);
    float sp = 0.f, s0 = 0.f, ss = 0.f, st = 0.f;
    if (CENTER >= 0) {  // the centroid node: distance R, relative 1
        sp = c_qc32[CENTER];
        s0 = c_qc32[CENTER];
    }
#pragma unroll
    for (int k = 0; k < NP; k++) {
        const float* c = c_qp32 + kQ * (POFF + k);
        const float L = fmaf(c[1], f.u2, c[0] * f.u1);
        float Q = fmaf(c[4], f.bb, 1.f);
        Q = fmaf(c[3], f.ab, Q);
        Q = fmaf(c[2], f.aa, Q);
        const float rp = rsqrt_f32(Q + L), rm = rsqrt_f32(Q - L);
        if (POT)
            sp = fmaf(c[5], rp + rm, sp);
        if (FIELD) {
            const float r3p = rp * rp * rp, r3m = rm * rm * rm;
            s0 = fmaf(c[5], r3p + r3m, s0);
            const float dd = r3p - r3m;
            ss = fmaf(c[6], dd, ss);
            st = fmaf(c[7], dd, st);
        }
    }
    return far32_finish<POT, FIELD>(e, d, a, b, f, sp, s0, ss, st);
}

// ------------------------------------------------------------------------- RWG (analytic)
// Analytic potential and field of a uniformly charged planar polygon (triangle NV = 3,
// rectangle NV = 4): phi = (-h Omega - sum_i t_i L_i) / (4 pi eps0),
// E = (N3 Omega + sum_i m_i L_i) / (4 pi eps0), with Omega the signed solid angle, m_i the
// outward in-plane edge normals, t_i = m_i.(P - edge midpoint) and L_i the log line
// integral of each edge (KElectrostaticRWGTriangleIntegrator.cc:20-208 IqL,
// :607-814 Potential, :817-1011 ElectricField; KElectrostaticRWGRectangleIntegrator.cc:20-240,
// :713-1174). Points on an edge line use the second-order log-argument expansion; points
// on two edge lines (a vertex) are averaged over P +- 1e-7 N3.
template<int NV> struct Polygon
{
    V3 v[NV];    // vertices in positive rotation order
    V3 L[NV];    // edge vectors used for the on-line test
    double len[NV];
    V3 u[NV];    // edge unit vectors
    V3 mid[NV];  // edge midpoints
    V3 m[NV];    // outward edge normals u x N3
    V3 n3;       // unit normal
    V3 n3raw;    // N1 x N2 (rectangle solid-angle plane test)
    V3 cen;
};

__device__ __forceinline__ void make_polygon(const double* g, Polygon<3>& q)
{
    const double A = g[rA], B = g[rB];
    const V3 P0 = ld3(g + rP0), N1 = ld3(g + rN1), N2 = ld3(g + rN2);
    q.v[0] = P0;
    q.v[1] = v3(__dadd_rn(P0.x, __dmul_rn(A, N1.x)), __dadd_rn(P0.y, __dmul_rn(A, N1.y)),
                __dadd_rn(P0.z, __dmul_rn(A, N1.z)));
    q.v[2] = v3(__dadd_rn(P0.x, __dmul_rn(B, N2.x)), __dadd_rn(P0.y, __dmul_rn(B, N2.y)),
                __dadd_rn(P0.z, __dmul_rn(B, N2.z)));
    V3 n = cross(N1, N2);
    q.n3raw = n;
    q.n3 = (1. / norm(n)) * n;
    q.cen = ld3(g + rCen);
    const V3 e12 = q.v[2] - q.v[1];
    const double l12 = norm(e12);
    q.L[0] = A * N1;
    q.L[1] = e12;
    q.L[2] = (-B) * N2;
    q.len[0] = A;
    q.len[1] = l12;
    q.len[2] = B;
    q.u[0] = N1;
    q.u[1] = (1. / l12) * e12;
    q.u[2] = v3(-N2.x, -N2.y, -N2.z);
    for (int i = 0; i < 3; i++) {
        q.mid[i] = (0.5 * q.len[i]) * q.u[i] + q.v[i];
        q.m[i] = cross(q.u[i], q.n3);
    }
}

__device__ __forceinline__ void make_polygon(const double* g, Polygon<4>& q)
{
    const double A = g[rA], B = g[rB];
    const V3 P0 = ld3(g + rP0), N1 = ld3(g + rN1), N2 = ld3(g + rN2);
    const V3 aN1 = v3(__dmul_rn(A, N1.x), __dmul_rn(A, N1.y), __dmul_rn(A, N1.z));
    const V3 bN2 = v3(__dmul_rn(B, N2.x), __dmul_rn(B, N2.y), __dmul_rn(B, N2.z));
    q.v[0] = P0;
    q.v[1] = v3(__dadd_rn(P0.x, aN1.x), __dadd_rn(P0.y, aN1.y), __dadd_rn(P0.z, aN1.z));
    q.v[2] = v3(__dadd_rn(q.v[1].x, bN2.x), __dadd_rn(q.v[1].y, bN2.y), __dadd_rn(q.v[1].z, bN2.z));
    q.v[3] = v3(__dadd_rn(P0.x, bN2.x), __dadd_rn(P0.y, bN2.y), __dadd_rn(P0.z, bN2.z));
    V3 n = cross(N1, N2);
    q.n3raw = n;
    q.n3 = (1. / norm(n)) * n;
    q.cen = ld3(g + rCen2);
    q.L[0] = aN1;
    q.L[1] = bN2;
    q.L[2] = v3(-aN1.x, -aN1.y, -aN1.z);
    q.L[3] = v3(-bN2.x, -bN2.y, -bN2.z);
    q.len[0] = A;
    q.len[1] = B;
    q.len[2] = A;
    q.len[3] = B;
    q.u[0] = N1;
    q.u[1] = N2;
    q.u[2] = v3(-N1.x, -N1.y, -N1.z);
    q.u[3] = v3(-N2.x, -N2.y, -N2.z);
    for (int i = 0; i < 4; i++) {
        q.mid[i] = (0.5 * q.len[i]) * q.u[i] + q.v[i];
        q.m[i] = cross(q.u[i], q.n3);
    }
}

// signed solid angle (Van Oosterom-Strackee), KEMField/Source/Surfaces/include/KSolidAngle.hh:58-…
__device__ __forceinline__ double tri_solid_angle(V3 a, V3 b, V3 c, V3 P)
{
    const V3 ua = (1. / norm(a - P)) * (a - P);
    const V3 ub = (1. / norm(b - P)) * (b - P);
    const V3 uc = (1. / norm(c - P)) * (c - P);
    const double x = 1. + dot(ua, ub) + dot(ua, uc) + dot(ub, uc);
    const double y = fabs(dot(ua, cross(ub, uc)));
    return fabs(2. * atan2(y, x));
}

template<int NV> __device__ double solid_angle(const Polygon<NV>& q, V3 P)
{
    if (NV == 3) {
        const double h = dot(q.n3, P - q.cen);
        double res;
        if (norm(P - q.cen) <= 1e-12)
            res = 2. * c_k.pi;
        else
            res = tri_solid_angle(q.v[0], q.v[1], q.v[2], P);
        return h < 0. ? -res : res;
    }
    else {
        const double h = dot(q.n3raw, P - q.cen);
        double res;
        if (fabs(h) < 1e-12) {
            const V3 dP = q.v[0] - P;
            const double l1 = -dot(dP, q.L[0]) / (q.len[0] * q.len[0]);
            const double l2 = -dot(dP, q.L[1]) / (q.len[1] * q.len[1]);
            res = (l1 > 0. && l1 < 1. && l2 > 0. && l2 < 1.) ? 2. * c_k.pi : 0.;
        }
        else
            res = tri_solid_angle(q.v[0], q.v[1], q.v[2], P) + tri_solid_angle(q.v[2], q.v[3], q.v[0], P);
        return h < 0. ? -res : res;
    }
}

// line integrals of the edges; counter/line/dist describe an on-line field point
template<int NV, bool POT, bool FIELD>
__device__ void edge_logs(const Polygon<NV>& q, V3 P, int counter, int line, double dist, double& il, V3& iv)
{
    il = 0.;
    iv = v3(0., 0., 0.);
    double rm[NV];
    V3 dv[NV];
#pragma unroll
    for (int i = 0; i < NV; i++) {
        dv[i] = q.v[i] - P;
        rm[i] = norm(dv[i]);
    }
#pragma unroll
    for (int i = 0; i < NV; i++) {
        const int j = (i + 1) % NV;
        const double rM = rm[i], rP = rm[j];
        const double sM = dot(dv[i], q.u[i]), sP = dot(dv[j], q.u[i]);
        double term = 0.;
        bool have = false;
        if (counter == 1 && line == i) {
            if (fabs(dist / sM) < 1e-6) {
                double quot = fabs(dist / sM);
                if (quot < 1e-14)
                    quot = 1e-14;
                const double taylor = 0.5 * fabs(sM) * quot * quot;
                term = log(rP + sP) - log(taylor);
                have = true;
            }
        }
        if (line != i) {
            double nom, den;
            if ((rM + sM) > (rP - sP)) {
                nom = rP + sP;
                den = rM + sM;
            }
            else {
                nom = rM - sM;
                den = rP - sP;
            }
            term += log(nom) - log(den);
            have = true;
        }
        if (have) {
            if (POT)
                il += dot(q.m[i], P - q.mid[i]) * term;
            if (FIELD)
                iv = iv + term * q.m[i];
        }
    }
}

template<int NV, bool POT, bool FIELD> __device__ Out4 rwg_at(const Polygon<NV>& q, V3 P, int counter, int line, double dist)
{
    double il;
    V3 iv;
    edge_logs<NV, POT, FIELD>(q, P, counter, line, dist, il, iv);
    const double om = solid_angle<NV>(q, P);
    Out4 o{0., 0., 0., 0.};
    if (POT)
        o.phi = -dot(q.n3, P - q.cen) * om - il;
    if (FIELD) {
        o.ex = q.n3.x * om + iv.x;
        o.ey = q.n3.y * om + iv.y;
        o.ez = q.n3.z * om + iv.z;
    }
    return o;
}

template<int NV, bool POT, bool FIELD> __device__ __noinline__ Out4 rwg64(const double* e, V3 P)
{
    Polygon<NV> q;
    make_polygon(e, q);
    int counter = 0, line = 99;
    double dmin = 0.;
#pragma unroll
    for (int i = 0; i < NV; i++) {
        const V3 dv = q.v[i] - P;
        const double inv = 1. / q.len[i];
        const double dl = norm(cross(q.L[i], dv)) * inv;
        const double lam = -dot(dv, q.L[i]) * (inv * inv);
        if (dl < 1e-14 && lam >= -1e-15 && lam <= 1. + 1e-15) {
            dmin = dl;
            counter++;
            line = i;
        }
    }
    const double k = c_k.one_over_four_pi_eps0;
    Out4 o;
    if (counter == 2) {
        const V3 up = P + 1e-7 * q.n3, dn = P - 1e-7 * q.n3;
        const Out4 a = rwg_at<NV, POT, FIELD>(q, up, 9, 9, 9.), b = rwg_at<NV, POT, FIELD>(q, dn, 9, 9, 9.);
        o = Out4{0.5 * (a.ex + b.ex), 0.5 * (a.ey + b.ey), 0.5 * (a.ez + b.ez), 0.5 * (a.phi + b.phi)};
    }
    else
        o = rwg_at<NV, POT, FIELD>(q, P, counter, line, dmin);
    return Out4{k * o.ex, k * o.ey, k * o.ez, k * o.phi};
}

// ------------------------------------------------------------------------- line segments
// Gauss-Legendre over the segment (KElectrostaticQuadratureLineSegmentIntegrator.cc:8-185)
template<bool POT, bool FIELD> __device__ __forceinline__ Out4 line_gauss(const double* e, V3 P, int off, int half)
{
    const V3 p0 = ld3(e + rP0), p1 = ld3(e + rN1);
    const double len = e[rA];
    const V3 c = 0.5 * (p0 + p1);
    const V3 u = (1. / len) * (p1 - p0);
    const double hl = 0.5 * len;
    double sp = 0.;
    V3 sv = v3(0., 0., 0.);
    for (int i = 0; i < half; i++) {
        const double wf = c_gl[2 * (off + i) + 1] * hl, x = c_gl[2 * (off + i)] * hl;
        const V3 dp = P - (c + x * u), dn = P - (c - x * u);
        const double ip = rsqrt(dot(dp, dp)), in = rsqrt(dot(dn, dn));
        if (POT)
            sp += wf * (ip + in);
        if (FIELD)
            sv = sv + wf * ((ip * ip * ip) * dp + (in * in * in) * dn);
    }
    const double pf = 0.25 * e[rB] / c_k.eps0;
    return Out4{pf * sv.x, pf * sv.y, pf * sv.z, pf * sp};
}

// analytic line segment (KElectrostaticAnalyticLineSegmentIntegrator.cc:15-82)
template<bool POT, bool FIELD> __device__ __noinline__ Out4 line_analytic(const double* e, V3 P)
{
    const V3 p0 = ld3(e + rP0), p1 = ld3(e + rN1);
    const double diam = e[rB];
    const double L = norm(p1 - p0);
    Out4 o{0., 0., 0., 0.};
    const double Da0 = norm(p0 - P), Db0 = norm(p1 - P);
    // shared "inside the wire" classification
    bool inside = false;
    V3 pp = v3(0., 0., 0.);
    if (!((Da0 + Db0) > (L + diam))) {
        const V3 u = (1. / L) * (p1 - p0);
        const double p = dot(P - p0, u);
        if (!(p < -diam * .5 || p > L + diam * .5)) {
            pp = p0 + p * u;
            if (!(norm(P - pp) >= diam * .5))
                inside = true;
        }
    }
    if (POT) {
        double Da = Da0, Db = Db0;
        if (inside) {
            Da = sqrt(dot(p0 - pp, p0 - pp) + diam * diam * .25);
            Db = sqrt(dot(p1 - pp, p1 - pp) + diam * diam * .25);
        }
        o.phi = diam / (4. * c_k.eps0) * log((Da + Db + L) / (Da + Db - L));
    }
    if (FIELD) {
        double Da = Da0, Db = Db0;
        if (inside) {
            Da = norm(p0 - pp);
            Db = norm(p1 - pp);
        }
        double den = (Da * (Da + Db + L) * (Da + Db - L) * Db) * 4. * c_k.eps0;
        den = -1. / den;
        const double s = 2. * L * diam * den;
        o.ex = s * (p1.x * Da - P.x * (Da + Db) + p0.x * Db);
        o.ey = s * (p1.y * Da - P.y * (Da + Db) + p0.y * Db);
        o.ez = s * (p1.z * Da - P.z * (Da + Db) + p0.z * Db);
    }
    return o;
}

// ------------------------------------------------------------------------- one EPI
// MIXED selects the Newton-refined hardware reciprocal square root for the cubature bands;
// everything else is the same FP64 code. Triangles and rectangles have separate unrolled
// cubature code (the element type is uniform across a warp, which evaluates one element).
//
// epi_far: a pair in a quadrature band (band_of(e, P, d, r2) returned band >= 1, with its d and
// r2); no analytic near-field code, so callers that route the analytic pairs elsewhere carry
// none of its registers or calls.
// F32 selects the FP32 far-field form for the triangle and rectangle cubature bands (wires keep
// their FP64 Gauss-Legendre sums).
template<bool MIXED, bool POT, bool FIELD, bool F32 = false>
__device__ __forceinline__ Out4 epi_far(const double* e, V3 P, V3 d, double r2, int band)
{
    const int type = (int) e[rType];
    if (type == kLineSegment)
        return band == 1 ? line_gauss<POT, FIELD>(e, P, 2, 8) : line_gauss<POT, FIELD>(e, P, 0, 2);
    if (F32) {
        if (type == kTriangle) {
            if (band == 1)
                return cubq32<33, kTri33, POT, FIELD>(e, d, r2);
            return band == 2 ? cubq32<12, kTri12, POT, FIELD>(e, d, r2) : cubq32<7, kTri7, POT, FIELD>(e, d, r2);
        }
        if (band == 1)
            return cubq_pairs32<16, kPair33, 1, POT, FIELD>(e, d, r2);
        return band == 2 ? cubq_pairs32<6, kPair12, -1, POT, FIELD>(e, d, r2)
                         : cubq_pairs32<3, kPair7, 0, POT, FIELD>(e, d, r2);
    }
    if (type == kTriangle) {
        if (band == 1)
            return cubq<33, kTri33, POT, FIELD, MIXED>(e, d, r2);
        return band == 2 ? cubq<12, kTri12, POT, FIELD, MIXED>(e, d, r2) : cubq<7, kTri7, POT, FIELD, MIXED>(e, d, r2);
    }
    if (band == 1)
        return cubq_pairs<16, kPair33, 1, POT, FIELD, MIXED>(e, d, r2);
    return band == 2 ? cubq_pairs<6, kPair12, -1, POT, FIELD, MIXED>(e, d, r2) : cubq_pairs<3, kPair7, 0, POT, FIELD, MIXED>(e, d, r2);
}

// epi for a pair known to lie outside the analytic band (the caller has shown that its centre
// distance exceeds the band-0 cut): the same band decision and quadrature as epi, with no call
// to the analytic integrals in the code path
template<bool MIXED, bool POT, bool FIELD, bool F32 = false> __device__ __forceinline__ Out4 epi_beyond_near(const double* e,
                                                                                                           V3 P)
{
    V3 d;
    double r2;
    const int band = band_of(e, P, d, r2);
    return epi_far<MIXED, POT, FIELD, F32>(e, P, d, r2, band);
}

template<bool MIXED, bool POT, bool FIELD, bool F32 = false> __device__ __forceinline__ Out4 epi(const double* e, V3 P)
{
    V3 d;
    double r2;
    const int band = band_of(e, P, d, r2);
    if (band == 0) {
        const int type = (int) e[rType];
        if (type == kLineSegment)
            return line_analytic<POT, FIELD>(e, P);
        return type == kTriangle ? rwg64<3, POT, FIELD>(e, P) : rwg64<4, POT, FIELD>(e, P);
    }
    return epi_far<MIXED, POT, FIELD, F32>(e, P, d, r2, band);
}

}  // namespace kemcu
