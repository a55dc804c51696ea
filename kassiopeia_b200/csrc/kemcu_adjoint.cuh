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
            int n;
            const int off = rule_offset(type, band, n);
            const V3 d0 = P - ld3(e + rP0), a = ld3(e + rEa), b = ld3(e + rEb);
            const V3 wE = v3(w[0], w[1], w[2]);
            const double pf = e[rPrefac];
            for (int k = 0; k < n; k++) {
                const double s = c_rules[3 * (off + k)], t = c_rules[3 * (off + k) + 1], wk = c_rules[3 * (off + k) + 2];
                const V3 d = d0 - s * a - t * b;
                const double ir = 0.5 * rsqrt2_acc(dot(d, d));
                const double ir3 = ir * ir * ir, ir5 = ir3 * ir * ir;
                const double c1 = pf * wk * (w[3] * ir3 + 3. * dot(wE, d) * ir5), c2 = pf * wk * ir3;
                const V3 gk = v3(c1 * d.x - c2 * wE.x, c1 * d.y - c2 * wE.y, c1 * d.z - c2 * wE.z);
                const double cw[3] = {1. - s - t, s, t};
#pragma unroll
                for (int v = 0; v < 3; v++) {
                    g[3 * v] += cw[v] * gk.x;
                    g[3 * v + 1] += cw[v] * gk.y;
                    g[3 * v + 2] += cw[v] * gk.z;
                }
            }
            // area term for this point: (w . F) dA / A, added per point so the frozen band holds
            const V3 ea = ld3(e + rEa), eb = ld3(e + rEb);
            V3 dA1, dA2;
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
