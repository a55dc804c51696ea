// K5: adjoint (vector-Jacobian product) of the direct sum. No counterpart in the reference.
//
// With out_p = sum_j sigma_j F_j(P_p), F = (E, phi) per unit charge density, and upstream
// weights w_p = (wE, wphi), L = sum_p w_p . out_p. Per element j this kernel returns
//   dL/dsigma_j = S_j = sum_p w_p . F_j(P_p)
//   dL/dV_j     = sigma_j * sum_p d(w_p . F_j(P_p)) / dV      (V = the element's 3 defining
//                 vertices P0, P1 = P0 + A N1, P2 = P0 + B N2; triangles and rectangles)
// Cubature bands are differentiated node by node: with node Q_k = (1-s-t) P0 + s P1 + t P2,
// d = P - Q_k, r = |d| and prefactor pf (area / (4 pi eps0)),
//   d(w.F)/dQ_k = pf w_k [ wphi d / r^3 - wE / r^3 + 3 (wE . d) d / r^5 ]
// plus the area term (w.F) dA / A. The rule band is frozen at its value for the given
// geometry (gradients are taken within a band). RWG near-field pairs are differentiated by
// central differences (step 1e-6 of the element size) of the FP64 analytic integral on the
// device. Line-segment vertex gradients are not provided (zero).
//
// Layout mirrors K1 with the roles of points and elements exchanged: one thread per element,
// points and weights streamed through shared memory, the point list split over gridDim.y.
#pragma once

#include "kemcu_kernels.cuh"

namespace kemcu
{

constexpr int kAdjThreads = 128;
constexpr int kPtTile = 64;

// element record rebuilt from three defining vertices (triangle / rectangle), same derived
// fields as the host-side record builder
__device__ void record_from_vertices(const double* e, V3 v0, V3 v1, V3 v2, double* r)
{
    for (int i = 0; i < rRecSize; i++)
        r[i] = e[i];
    const int type = (int) e[rType];
    const V3 a = v1 - v0, b = v2 - v0;
    const double A = norm(a), B = norm(b);
    const V3 n1 = (1. / A) * a, n2 = (1. / B) * b;
    r[rA] = A;
    r[rB] = B;
    r[rP0] = v0.x; r[rP0 + 1] = v0.y; r[rP0 + 2] = v0.z;
    r[rN1] = n1.x; r[rN1 + 1] = n1.y; r[rN1 + 2] = n1.z;
    r[rN2] = n2.x; r[rN2 + 1] = n2.y; r[rN2 + 2] = n2.z;
    const V3 ea = A * n1, eb = B * n2;
    r[rEa] = ea.x; r[rEa + 1] = ea.y; r[rEa + 2] = ea.z;
    r[rEb] = eb.x; r[rEb + 1] = eb.y; r[rEb + 2] = eb.z;
    const double cm = norm(cross(n1, n2));
    r[rAA] = dot(ea, ea);
    r[rAB2] = 2. * dot(ea, eb);
    r[rBB] = dot(eb, eb);
    if (type == kTriangle) {
        const V3 cen = v0 + (1. / 3.) * (ea + eb);
        r[rCen] = r[rCen2] = cen.x;
        r[rCen + 1] = r[rCen2 + 1] = cen.y;
        r[rCen + 2] = r[rCen2 + 2] = cen.z;
        r[rPrefac] = 0.5 * A * B * cm * c_k.one_over_four_pi_eps0;
    }
    else {
        const V3 cen = v0 + 0.5 * (ea + eb);
        r[rCen] = r[rCen2] = cen.x;
        r[rCen + 1] = r[rCen2 + 1] = cen.y;
        r[rCen + 2] = r[rCen2 + 2] = cen.z;
        r[rPrefac] = A * B * c_k.one_over_four_pi_eps0;
    }
}

// d(w . F)/dV for one RWG pair by central differences; g[9] accumulates (P0, P1, P2)
__device__ __noinline__ void rwg_vertex_grad(const double* e, V3 P, const double* w, double* g)
{
    const int type = (int) e[rType];
    const V3 v0 = ld3(e + rP0), v1 = v0 + ld3(e + rEa), v2 = v0 + ld3(e + rEb);
    const double h = 1e-6 / e[rInvSize];
    double r[rRecSize];
    for (int q = 0; q < 9; q++) {
        double f[2];
        for (int sgn = 0; sgn < 2; sgn++) {
            V3 u0 = v0, u1 = v1, u2 = v2;
            V3* u = q < 3 ? &u0 : q < 6 ? &u1 : &u2;
            const double dh = sgn ? -h : h;
            if (q % 3 == 0) u->x += dh;
            else if (q % 3 == 1) u->y += dh;
            else u->z += dh;
            record_from_vertices(e, u0, u1, u2, r);
            const Out4 o = type == kTriangle ? rwg64<3, true, true>(r, P) : rwg64<4, true, true>(r, P);
            f[sgn] = w[0] * o.ex + w[1] * o.ey + w[2] * o.ez + w[3] * o.phi;
        }
        g[q] += (f[0] - f[1]) / (2. * h);
    }
}

// Node-gradient moments of one (element, point) pair for a rule of N nodes from node OFF.
// With d = P - centroid, node offsets o_k = s'_k (A N1) + t'_k (B N2), r_k = |d - o_k| and
//   c1_k = w_k (wphi / r^3 + 3 (wE . (d - o_k)) / r^5),  c2_k = w_k / r^3,
// the gradient of w . F with respect to node k is pf (c1_k (d - o_k) - c2_k wE), and a vertex
// gradient is its barycentric weight times that, summed over nodes. Both sums are linear in
// the node moments m = (sum c1, sum s'c1, sum t'c1, sum s'^2 c1, sum s't' c1, sum t'^2 c1,
// sum c2, sum s'c2, sum t'c2), accumulated here (9 FMAs per node, no per-node vectors).
constexpr int kQA = 6;
__constant__ double c_qa[kNumNodes * kQA];  // per node: w, w s', w t', w s'^2, w s't', w t'^2
template<int N, int OFF, bool FAST>
__device__ __forceinline__ void node_moments(const double* e, V3 d, V3 wE, double wphi, double m[9])
{
    const V3 a = ld3(e + rEa), b = ld3(e + rEb);
    const double R2 = dot(d, d), Da = dot(d, a), Db = dot(d, b);
    const double aa = e[rAA], ab2 = e[rAB2], bb = e[rBB];
    // 3 wE.(d - o_k) = 3 wE.d + (-2 s') (1.5 wE.a) + (-2 t') (1.5 wE.b)
    const double w3d = 3. * dot(wE, d), w3a = 1.5 * dot(wE, a), w3b = 1.5 * dot(wE, b);
    constexpr int G = N % KEMCU_GROUP == 0 ? KEMCU_GROUP : N;
#pragma unroll 1
    for (int g = 0; g < N / G; g++) {
        const double* cg = c_q + kQ * (OFF + g * G);
        const double* ag = c_qa + kQA * (OFF + g * G);
#pragma unroll
        for (int k = 0; k < G; k++) {
            const double* c = cg + kQ * k;
            const double* w = ag + kQA * k;
            double q2 = fma(c[0], Da, R2);
            q2 = fma(c[1], Db, q2);
            q2 = fma(c[2], aa, q2);
            q2 = fma(c[3], ab2, q2);
            q2 = fma(c[4], bb, q2);
            const double ir = 0.5 * irsq<FAST>(q2), ir2 = ir * ir, ir3 = ir2 * ir;
            const double wd3 = fma(c[1], w3b, fma(c[0], w3a, w3d));
            const double c1 = ir3 * fma(wd3, ir2, wphi);
#pragma unroll
            for (int q = 0; q < 6; q++)
                m[q] = fma(w[q], c1, m[q]);
#pragma unroll
            for (int q = 0; q < 3; q++)
                m[6 + q] = fma(w[q], ir3, m[6 + q]);
        }
    }
}

template<bool MIXED>
__global__ void __launch_bounds__(kAdjThreads) vjp_kernel(const double* __restrict__ rec, int n_elem,
                                                          const double* __restrict__ pts, const double* __restrict__ wts,
                                                          int n_pts, double* __restrict__ part_s,
                                                          double* __restrict__ part_g)
{
    __shared__ double s_p[kPtTile][3];
    __shared__ double s_w[kPtTile][4];
    // the CTA's element records, one per thread, rows padded to 33 doubles so that the threads'
    // reads of the same field fall in different banks (read once per point by the owner)
    __shared__ double s_e[kAdjThreads][rRecSize + 1];
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = j < n_elem;
    {
        const int first = blockIdx.x * blockDim.x, cnt = min((int) blockDim.x, n_elem - first);
        for (int q = threadIdx.x; q < cnt * rRecSize; q += blockDim.x)
            s_e[q / rRecSize][q % rRecSize] = rec[(size_t) first * rRecSize + q];
    }
    __syncthreads();
    const double* e = s_e[threadIdx.x];
    const int type = active ? (int) e[rType] : 0;
    const int per = (n_pts + gridDim.y - 1) / gridDim.y;
    const int p0 = blockIdx.y * per, p1 = min(n_pts, p0 + per);
    Kahan S;
    double g[9] = {0., 0., 0., 0., 0., 0., 0., 0., 0.};
    // gradients of log(area) with respect to P1 and P2 (the element's constant part of the
    // area term), formed once per element
    V3 dA1 = v3(0., 0., 0.), dA2 = v3(0., 0., 0.);
    if (active && type != kLineSegment) {
        const V3 ea = ld3(e + rEa), eb = ld3(e + rEb);
        if (type == kTriangle) {
            const V3 c = cross(ea, eb);
            const V3 ch = (1. / norm(c)) * c;
            const double A2 = 0.5 * norm(c);
            dA1 = (0.5 / A2) * cross(eb, ch);
            dA2 = (0.5 / A2) * cross(ch, ea);
        }
        else {
            dA1 = (1. / dot(ea, ea)) * ea;
            dA2 = (1. / dot(eb, eb)) * eb;
        }
    }
    for (int t0 = p0; t0 < p1; t0 += kPtTile) {
        const int cnt = min(kPtTile, p1 - t0);
        __syncthreads();
        for (int q = threadIdx.x; q < cnt; q += blockDim.x) {
            for (int c = 0; c < 3; c++)
                s_p[q][c] = pts[3 * (size_t) (t0 + q) + c];
            for (int c = 0; c < 4; c++)
                s_w[q][c] = wts[4 * (size_t) (t0 + q) + c];
        }
        __syncthreads();
        if (!active)
            continue;
        for (int q = 0; q < cnt; q++) {
            const V3 P = v3(s_p[q][0], s_p[q][1], s_p[q][2]);
            const double* w = s_w[q];
            const Out4 F = epi<MIXED, true, true>(e, P);
            S.add(w[0] * F.ex + w[1] * F.ey + w[2] * F.ez + w[3] * F.phi);
            if (type == kLineSegment)
                continue;
            const int band = band_of(e, P);
            if (band == 0) {
                rwg_vertex_grad(e, P, w, g);
                continue;
            }
            // node gradients from the rule's node moments (node_moments), mapped to the vertices
            const V3 dc = P - ld3(e + rCen), a = ld3(e + rEa), b = ld3(e + rEb);
            const V3 wE = v3(w[0], w[1], w[2]);
            double m[9] = {0., 0., 0., 0., 0., 0., 0., 0., 0.};
            if (type == kTriangle) {
                if (band == 1)
                    node_moments<33, kTri33, MIXED>(e, dc, wE, w[3], m);
                else if (band == 2)
                    node_moments<12, kTri12, MIXED>(e, dc, wE, w[3], m);
                else
                    node_moments<7, kTri7, MIXED>(e, dc, wE, w[3], m);
            }
            else {
                if (band == 1)
                    node_moments<33, kRect33, MIXED>(e, dc, wE, w[3], m);
                else if (band == 2)
                    node_moments<12, kRect12, MIXED>(e, dc, wE, w[3], m);
                else
                    node_moments<7, kRect7, MIXED>(e, dc, wE, w[3], m);
            }
            {
                // barycentric weights of the nodes: P1 weight s = s' + sc, P2 weight t = t' + sc
                const double sc = type == kTriangle ? 1. / 3. : 0.5;
                const double pf = e[rPrefac];
                // sum over nodes of weight x (c1 (d - o) - c2 wE) for weights 1, s, t
                const double T1[3] = {m[0], m[1] + sc * m[0], m[2] + sc * m[0]};           // c1 . {1, s, t}
                const double Ts[3] = {m[1], m[3] + sc * m[1], m[4] + sc * m[1]};           // c1 s' . {1, s, t}
                const double Tt[3] = {m[2], m[4] + sc * m[2], m[5] + sc * m[2]};           // c1 t' . {1, s, t}
                const double T2[3] = {m[6], m[7] + sc * m[6], m[8] + sc * m[6]};           // c2 . {1, s, t}
                V3 G[3];
#pragma unroll
                for (int v = 0; v < 3; v++)
                    G[v] = v3(pf * (dc.x * T1[v] - a.x * Ts[v] - b.x * Tt[v] - wE.x * T2[v]),
                              pf * (dc.y * T1[v] - a.y * Ts[v] - b.y * Tt[v] - wE.y * T2[v]),
                              pf * (dc.z * T1[v] - a.z * Ts[v] - b.z * Tt[v] - wE.z * T2[v]));
                // vertex P0 has weight 1 - s - t
                g[0] += G[0].x - G[1].x - G[2].x;
                g[1] += G[0].y - G[1].y - G[2].y;
                g[2] += G[0].z - G[1].z - G[2].z;
                g[3] += G[1].x;
                g[4] += G[1].y;
                g[5] += G[1].z;
                g[6] += G[2].x;
                g[7] += G[2].y;
                g[8] += G[2].z;
            }
            // area term for this point: (w . F) dA / A, added per point so the frozen band holds
            const double wf = w[0] * F.ex + w[1] * F.ey + w[2] * F.ez + w[3] * F.phi;
            g[0] -= wf * (dA1.x + dA2.x);
            g[1] -= wf * (dA1.y + dA2.y);
            g[2] -= wf * (dA1.z + dA2.z);
            g[3] += wf * dA1.x;
            g[4] += wf * dA1.y;
            g[5] += wf * dA1.z;
            g[6] += wf * dA2.x;
            g[7] += wf * dA2.y;
            g[8] += wf * dA2.z;
        }
    }
    if (!active)
        return;
    part_s[(size_t) blockIdx.y * n_elem + j] = S.s;
    for (int q = 0; q < 9; q++)
        part_g[((size_t) blockIdx.y * n_elem + j) * 9 + q] = g[q];
}

}  // namespace kemcu
