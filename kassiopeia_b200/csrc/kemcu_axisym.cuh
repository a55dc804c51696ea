// Axisymmetric elements: conic sections (a straight generator from (r0, z0) to (r1, z1) turned
// about the z axis, KConicSection.hh) and rings (a charged circle of radius R at height Z,
// KRing.hh), with KEMField's analytic integrators for both
// (KElectrostaticAnalyticConicSectionIntegrator.cc:9-221, KElectrostaticAnalyticRingIntegrator.cc:26-208).
//
// A context whose elements are all axisymmetric keeps one record per element:
//   [aType] 0 conic section, 1 ring
//   [aZa, aRa, aZb, aRb] generator end points (a ring has a = b)
//   [aLen] generator length (1 for a ring: its integrand does not depend on the position p)
//   [aPre] prefactor: 1 / (pi eps0) for a conic section, 1 / (2 pi^2 eps0 R) for a ring
//   [aCx, aCy, aCz] centroid, the collocation point of the element's matrix row
// and its own field, matrix-free matvec and assembly kernels; the dense operator, GMRES and
// refinement on top are shared with the planar elements.
#pragma once

namespace kemcu
{
enum AxRec
{
    aType = 0,
    aZa,
    aRa,
    aZb,
    aRb,
    aLen,
    aPre,
    aCx,
    aCy,
    aCz,
    aRecUsed
};
constexpr double kAxConic = 0., kAxRing = 1.;
constexpr double kLn4 = 1.386294361119890;

// The geometric steps (ring position on the generator, node positions, the split point, the
// distances) and eta = 1 - k^2 in the elliptic integrals are rounded operation by operation
// (__dmul_rn / __dadd_rn are never contracted into FMAs), as the reference's host code rounds
// them: near the generator the integrand varies like 1 / eta and ln eta, and a value one
// rounding apart changes it visibly.
__device__ __forceinline__ double mul(double a, double b)
{
    return __dmul_rn(a, b);
}
__device__ __forceinline__ double add(double a, double b)
{
    return __dadd_rn(a, b);
}
__device__ __forceinline__ double sub(double a, double b)
{
    return __dsub_rn(a, b);
}

// Complete elliptic integrals of the first and second kind in W. J. Cody's form (Math. Comp.
// 19 (1965) 105): with eta = 1 - k^2,
//   K = ln 4 + sum_n a_n eta^n - (1/2 + sum_n b_n eta^n) ln eta,
//   E = 1 + sum_n c_n eta^n - (sum_n d_n eta^n) ln eta,
// n = 1..10, Cody's published coefficient sets (the ones KEllipticIntegrals.cc:21-103 uses,
// needed for identical element integrals); the E series stops once eta^n < 1e-20.
__constant__ double c_cody_ka[10] = {9.657359028085625e-2, 3.088514627130518e-2, 1.493801353268716e-2, 8.789801874555064e-3,
                                     6.179627446053317e-3, 6.847909282624505e-3, 9.848929322176893e-3, 8.003003980649985e-3,
                                     2.296634898396958e-3, 1.393087857006646e-4};
__constant__ double c_cody_kb[10] = {1.249999999999080e-1, 7.031249973903835e-2, 4.882804190686239e-2, 3.737773975862360e-2,
                                     3.012484901289893e-2, 2.393191332311079e-2, 1.553094163197720e-2, 5.973904299155429e-3,
                                     9.215546349632498e-4, 2.970028096655561e-5};
__constant__ double c_cody_ec[10] = {4.431471805608895e-1, 5.680519456755915e-2, 2.183181167613048e-2, 1.156959574529540e-2,
                                     7.595093422559432e-3, 7.820404060959554e-3, 1.077063503986645e-2, 8.638442173604074e-3,
                                     2.468503330460722e-3, 1.494662175718132e-4};
__constant__ double c_cody_ed[10] = {2.499999999999017e-1, 9.374999972120314e-2, 5.859366125553149e-2, 4.271789054738309e-2,
                                     3.347894366576162e-2, 2.614501470031387e-2, 1.680402334636338e-2, 6.432146586438301e-3,
                                     9.898332846225384e-4, 3.185919565550157e-5};

__device__ __forceinline__ double ell_K(double k)
{
    const double eta = sub(1., mul(k, k));  // as rounded on the host: eta can be tiny here
    double en = eta, sa = 0., sb = 0.;
#pragma unroll
    for (int i = 0; i < 10; i++) {
        sa += c_cody_ka[i] * en;
        sb += c_cody_kb[i] * en;
        en *= eta;
    }
    return kLn4 + sa - (0.5 + sb) * log(fabs(eta) + 1.e-19);
}

// K(k), E(k) and (E - K) / k^2 together; one logarithm serves both of Cody's series.
//
// (E - K) / k^2 is the difference of the two for k^2 > 0.8, as KEllipticIntegrals.cc:108-131
// forms it (near the generator, where k -> 1, the integrand is sensitive to each rounding, and
// this branch keeps the reference's). For k^2 <= 0.8 the reference sums the power series
// sum_n (b_n - a_n) k^(2(n-1)) until k^(2n) < 1e-16: up to 166 terms, as many as the point's
// distance requires, so the 32 points of a warp ran up to 5x the mean number of terms. Here
// that branch comes from the arithmetic-geometric mean instead (Abramowitz & Stegun 17.6.3-4,
// Gauss's method): with a_0 = 1, b_0 = k', c_0 = k, a_{n+1} = (a_n + b_n) / 2,
// b_{n+1} = sqrt(a_n b_n) and c_{n+1} = c_n^2 / (4 a_{n+1}),
//     E = K (1 - sum_{n>=0} 2^(n-1) c_n^2),   so   (E - K) / k^2 = -K (1/2 + sum_{n>=1} 2^(n-1) c_n^2 / k^2),
// a sum of positive terms with no cancellation. For k^2 <= 0.8, c_4^2 < 1e-15 and c_5^2 < 1e-31:
// four terms give the full double precision (4.4e-16 relative against a 40-digit evaluation
// over [1e-12, 0.8], where the reference's series reaches 1.7e-15), a fixed cost of three square
// roots and three divisions. c_4 uses a_3 for a_4 (their relative difference, c_4 / a_3 < 4e-8,
// scales a term already below 1e-14 of the sum). K is Cody's, as in the potential.
__device__ __forceinline__ void ell_KE_EK(double k, double& K, double& E, double& EK)
{
    const double eta = sub(1., mul(k, k));
    const double lg = log(fabs(eta) + 1.e-19);
    double en = eta, sa = 0., sb = 0., sc = 0., sd = 0.;
    bool e_on = true;  // E stops at the first eta^n below 1e-20, K runs all ten terms
#pragma unroll
    for (int i = 0; i < 10; i++) {
        sa += c_cody_ka[i] * en;
        sb += c_cody_kb[i] * en;
        if (e_on) {
            sc += c_cody_ec[i] * en;
            sd += c_cody_ed[i] * en;
        }
        en *= eta;
        if (en < 1.e-20)
            e_on = false;
    }
    K = kLn4 + sa - (0.5 + sb) * lg;
    E = 1. + sc - sd * lg;
    const double k2 = k * k;
    if (k2 > 0.8) {
        EK = (E - K) / k2;
        return;
    }
    const double kp = sqrt(eta);
    const double a1 = 0.5 * (1. + kp), b1 = sqrt(kp);
    const double t1 = k2 / (16. * a1 * a1);  // c_1^2 / k^2
    const double q1 = k2 * t1;               // c_1^2
    const double a2 = 0.5 * (a1 + b1), b2 = sqrt(a1 * b1);
    const double f2 = q1 / (16. * a2 * a2);  // c_2^2 / c_1^2
    const double t2 = t1 * f2, q2 = q1 * f2;
    const double a3 = 0.5 * (a2 + b2);
    const double i3 = 1. / (16. * a3 * a3);
    const double f3 = q2 * i3;
    const double t3 = t2 * f3, q3 = q2 * f3;
    const double t4 = t3 * (q3 * i3);
    EK = -K * (0.5 + t1 + 2. * t2 + 4. * t3 + 8. * t4);
}

// evaluation point (z, r) and generator (za, ra) -> (zb, rb) of length len; the ring sits at
// distance p along the generator (KElectrostaticAnalyticRingIntegrator.cc:70-94)
struct AxPar
{
    double z, r, za, ra, zb, rb, len;
};

struct RingGeom
{
    double R, dz, dr, sumr, eta, S;
};

__device__ __forceinline__ RingGeom ring_at(double p, const AxPar& q)
{
    RingGeom g;
    const double t = p / q.len;
    const double Z = add(q.za, mul(t, sub(q.zb, q.za)));
    g.R = add(q.ra, mul(t, sub(q.rb, q.ra)));
    g.dz = sub(q.z, Z);
    g.dr = sub(q.r, g.R);
    g.sumr = add(g.R, q.r);
    const double dz2 = mul(g.dz, g.dz), s2 = add(mul(g.sumr, g.sumr), dz2);
    g.eta = add(mul(g.dr, g.dr), dz2) / s2;
    g.S = sqrt(s2);
    return g;
}

// R K / S (potential of the ring, before the prefactor)
struct RingPotential
{
    static constexpr int M = 1;
    __device__ __forceinline__ void operator()(double p, const AxPar& q, double* v) const
    {
        const RingGeom g = ring_at(p, q);
        const double k = g.eta > 1. ? 0. : sqrt(1. - g.eta);
        v[0] = g.R * ell_K(k) / g.S;
    }
};

// (E_r, E_z) of the ring before the prefactor: R / S^3 (-2 R EK + dr E / eta) and
// dz / S^3 E / eta R (KElectrostaticAnalyticRingIntegrator.cc:121-208)
struct RingField
{
    static constexpr int M = 2;
    __device__ __forceinline__ void operator()(double p, const AxPar& q, double* v) const
    {
        const RingGeom g = ring_at(p, q);
        const double k = g.eta > 1. ? 0. : sqrt(1. - g.eta);  // eta <= 1 for r, R >= 0
        double K, E, EK;
        ell_KE_EK(k, K, E, EK);
        const double S3 = g.S * g.S * g.S;
        v[0] = g.R / S3 * add(mul(mul(-2., g.R), EK), mul(g.dr / g.eta, E));
        v[1] = g.dz / S3 * E / g.eta * g.R;
    }
};

// both at once: (E_r, E_z, potential) from one ring geometry per node; each component is the
// value the two integrands above give, so the sums are theirs
struct RingFieldAndPotential
{
    static constexpr int M = 3;
    __device__ __forceinline__ void operator()(double p, const AxPar& q, double* v) const
    {
        const RingGeom g = ring_at(p, q);
        const double k = g.eta > 1. ? 0. : sqrt(1. - g.eta);  // eta <= 1 for r, R >= 0
        double K, E, EK;
        ell_KE_EK(k, K, E, EK);
        const double S3 = g.S * g.S * g.S;
        v[0] = g.R / S3 * add(mul(mul(-2., g.R), EK), mul(g.dr / g.eta, E));
        v[1] = g.dz / S3 * E / g.eta * g.R;
        v[2] = g.R * K / g.S;
    }
};

// F. Glueck's composite rule on [a, b] with n >= 20 intervals: n + 1 equidistant nodes,
// end-corrected weights on the first and last ten and weight 1 inside, times (b - a) / n
// (KGaussianQuadrature.cc:18-86, its n >= 20 branch, the only one the conic-section
// integrator reaches)
__constant__ double c_glueck_w9[10] = {0.2803440531305107e0, 0.1648702325837748e1, -0.2027449845679092e0,
                                       0.2797927414021179e1, -0.9761199294532843e0, 0.2556499393738999e1,
                                       0.1451083002645404e0, 0.1311227127425048e1, 0.9324249063051143e0,
                                       0.1006631393298060e1};

template<class F> __device__ void glueck_quad(const F& f, const AxPar& q, double a, double b, int n, double* ans)
{
    const double deln = (b - a) / n;
    for (int j = 0; j < F::M; j++)
        ans[j] = 0.;
    for (int i = 0; i <= n; i++) {
        const double x = add(a, mul(deln, (double) i));
        double v[F::M];
        f(x, q, v);
        if (i < 10 || i > n - 10) {
            const double w = c_glueck_w9[i < 10 ? i : n - i];
            for (int j = 0; j < F::M; j++)
                ans[j] += w * v[j];
        }
        else
            for (int j = 0; j < F::M; j++)
                ans[j] += v[j];
    }
    for (int j = 0; j < F::M; j++)
        ans[j] *= deln;
}

// integral over the generator of a conic section of the ring integrand F (potential or field),
// as KElectrostaticAnalyticConicSectionIntegrator.cc:33-93 / 113-198: with D the relative
// excess of the distances to the end points over the length, 20, 100 or 500 intervals far
// from the generator; closer, the generator is cut at the foot point of the evaluation point
// and each side integrated in pieces shrinking by 0.3 towards it (50 intervals each, at most
// 35 pieces), the last piece of length h taken as h (ln 4 + ln(2 r + 1e-12) + 1 - ln h) / 2.
// The reference adds that logarithmic remainder to both field components as well; so does
// this code.
//
// The three far bands share one inlined quadrature loop; the subdivided near branch, which few
// pairs reach, is a separate (not inlined) function so that its loops do not raise the
// register count of the far path.
template<class F> __device__ __noinline__ void conic_near(const F& f, const AxPar& q, double* out);

template<class F> __device__ __forceinline__ void conic_integral(const F& f, const AxPar& q, double* out)
{
    const double Da = sqrt(add(mul(sub(q.za, q.z), sub(q.za, q.z)), mul(sub(q.ra, q.r), sub(q.ra, q.r))));
    const double Db = sqrt(add(mul(sub(q.zb, q.z), sub(q.zb, q.z)), mul(sub(q.rb, q.r), sub(q.rb, q.r))));
    const double D = fabs(sub(add(Da, Db), q.len)) / q.len;
    if (D >= 5.e-4)
        glueck_quad(f, q, 0., q.len, D >= 5.e-2 ? 20 : D >= 5.e-3 ? 100 : 500, out);
    else
        conic_near(f, q, out);
}

template<class F> __device__ __noinline__ void conic_near(const F& f, const AxPar& q, double* out)
{
    const double L = q.len;
    const double u0 = (q.zb - q.za) / L, u1 = (q.rb - q.ra) / L;
    const double pp = add(mul(sub(q.z, q.za), u0), mul(sub(q.r, q.ra), u1));
    for (int j = 0; j < F::M; j++)
        out[j] = 0.;
    double tmp[F::M];
    if (pp < L) {
        const double pmax = L;
        double pmin = pp;
        if (pp < 0.)
            pmin = 0.;
        double b = pmax;
        double a = add(pmin, mul(sub(b, pmin), 0.3));
        for (int n = 1; n <= 35; n++) {
            glueck_quad(f, q, a, b, 50, tmp);
            for (int j = 0; j < F::M; j++)
                out[j] += tmp[j];
            if (fabs(a - pmin) / L < 1.e-8)
                break;
            b = a;
            a = add(pmin, mul(sub(b, pmin), 0.3));
        }
        const double h = fabs(a - pmin);
        const double rem = h * (kLn4 + log(2. * q.r + 1.e-12) + 1. - log(h)) / 2.;
        for (int j = 0; j < F::M; j++)
            out[j] += rem;
    }
    if (pp > 0.) {
        double pmax = pp;
        const double pmin = 0.;
        if (pp > L)
            pmax = L;
        double b = pmin;
        double a = sub(pmax, mul(sub(pmax, b), 0.3));
        for (int n = 1; n <= 35; n++) {
            glueck_quad(f, q, b, a, 50, tmp);
            for (int j = 0; j < F::M; j++)
                out[j] += tmp[j];
            if (fabs(pmax - a) / L < 1.e-8)
                break;
            b = a;
            a = sub(pmax, mul(sub(pmax, b), 0.3));
        }
        const double h = fabs(pmax - a);
        const double rem = h * (kLn4 + log(2. * q.r + 1.e-12) + 1. - log(h)) / 2.;
        for (int j = 0; j < F::M; j++)
            out[j] += rem;
    }
}

__device__ __forceinline__ AxPar ax_par(const double* e, double x, double y, double z)
{
    AxPar q;
    q.z = z;
    q.r = sqrt(add(mul(x, x), mul(y, y)));
    q.za = e[aZa];
    q.ra = e[aRa];
    q.zb = e[aZb];
    q.rb = e[aRb];
    q.len = e[aLen];
    return q;
}

// potential per unit charge density of element e at (x, y, z)
__device__ __forceinline__ double ax_potential(const double* e, double x, double y, double z)
{
    const AxPar q = ax_par(e, x, y, z);
    double v[1];
    if (e[aType] == kAxRing)
        RingPotential()(x, q, v);  // the ring integrand does not depend on its position argument
    else
        conic_integral(RingPotential(), q, v);
    return e[aPre] * v[0];
}

// field per unit charge density; E_r is turned into (E_x, E_y), zero on the axis (r < 1e-14)
__device__ __forceinline__ void ax_field(const double* e, double x, double y, double z, double* E)
{
    const AxPar q = ax_par(e, x, y, z);
    double v[2];
    if (e[aType] == kAxRing)
        RingField()(x, q, v);
    else
        conic_integral(RingField(), q, v);
    const double er = e[aPre] * v[0];
    E[2] = e[aPre] * v[1];
    if (q.r < 1.e-14)
        E[0] = E[1] = 0.;
    else {
        E[0] = x / q.r * er;
        E[1] = y / q.r * er;
    }
}

// field and potential per unit charge density in one pass over the generator
__device__ __forceinline__ void ax_field_potential(const double* e, double x, double y, double z, double* out)
{
    const AxPar q = ax_par(e, x, y, z);
    double v[3];
    if (e[aType] == kAxRing)
        RingFieldAndPotential()(x, q, v);
    else
        conic_integral(RingFieldAndPotential(), q, v);
    const double er = e[aPre] * v[0];
    out[2] = e[aPre] * v[1];
    out[3] = e[aPre] * v[2];
    if (q.r < 1.e-14)
        out[0] = out[1] = 0.;
    else {
        out[0] = x / q.r * er;
        out[1] = y / q.r * er;
    }
}

constexpr int kAxThreads = 128;
// resident CTAs per SM the field kernel's registers are bounded for (96 registers a thread): on
// the axisymmetric coax at 100,000 points, 216 ms against 224 ms at four CTAs and 264 ms
// unbounded (154 registers, three CTAs); the local-memory spills this costs stay in L1
constexpr int kAxFieldMinBlocks = 5;

// direct sum over the elements [e0, e1) of split blockIdx.y at each point, compensated (Kahan)
// over the elements as KIntegratingFieldSolver does (KElectrostaticIntegratingFieldSolver.hh:
// 261-339); out n x 4, or partial[split][n][4] summed by reduce_splits in split order
template<bool POT, bool FIELD>
__global__ void __launch_bounds__(kAxThreads, kAxFieldMinBlocks)
    axisym_field_kernel(const double* __restrict__ rec, int rec_stride, const double* __restrict__ sigma, int ne,
                        const double* __restrict__ P, int np, double* __restrict__ out, double* __restrict__ partial)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np)
        return;
    const int per = (ne + gridDim.y - 1) / gridDim.y;
    const int e0 = blockIdx.y * per, e1 = min(ne, e0 + per);
    const double x = P[3 * i], y = P[3 * i + 1], z = P[3 * i + 2];
    double s[4] = {0., 0., 0., 0.}, c[4] = {0., 0., 0., 0.};
    for (int j = e0; j < e1; j++) {
        const double* e = rec + (size_t) j * rec_stride;
        const double sg = sigma[j];
        double v[4] = {0., 0., 0., 0.};
        if (FIELD && POT)
            ax_field_potential(e, x, y, z, v);
        else if (FIELD)
            ax_field(e, x, y, z, v);
        else
            v[3] = ax_potential(e, x, y, z);
#pragma unroll
        for (int m = 0; m < 4; m++) {
            const double yk = v[m] * sg - c[m];
            const double t = s[m] + yk;
            c[m] = (t - s[m]) - yk;
            s[m] = t;
        }
    }
    double* dst = partial ? partial + (size_t) blockIdx.y * np * 4 : out;
#pragma unroll
    for (int m = 0; m < 4; m++)
        dst[4 * (size_t) i + m] = s[m];
}

// y[r][i] = sum_j A_ij x[r][j], A_ij = potential of element j at the centroid of element i
// (Dirichlet rows, KBoundaryIntegralMatrix.hh:31-55); one thread per row, the columns split
// over gridDim.y (partial[split][nrhs][n] when split > 1)
template<int NR>
__global__ void __launch_bounds__(kAxThreads) axisym_matvec_kernel(const double* __restrict__ rec, int rec_stride, int n,
                                                                    const double* __restrict__ x, int nrhs,
                                                                    double* __restrict__ y, double* __restrict__ partial)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const int per = (n + gridDim.y - 1) / gridDim.y;
    const int j0 = blockIdx.y * per, j1 = min(n, j0 + per);
    const double* t = rec + (size_t) i * rec_stride;
    const double cx = t[aCx], cy = t[aCy], cz = t[aCz];
    double acc[NR];
#pragma unroll
    for (int r = 0; r < NR; r++)
        acc[r] = 0.;
    for (int j = j0; j < j1; j++) {
        const double a = ax_potential(rec + (size_t) j * rec_stride, cx, cy, cz);
#pragma unroll
        for (int r = 0; r < NR; r++)
            if (r < nrhs)
                acc[r] += a * x[(size_t) r * n + j];
    }
    double* dst = partial ? partial + (size_t) blockIdx.y * nrhs * n : y;
#pragma unroll
    for (int r = 0; r < NR; r++)
        if (r < nrhs)
            dst[(size_t) r * n + i] = acc[r];
}

// the operator column-major with leading dimension ld, FP64 and (when a32) FP32; one thread
// per row, the columns [0, n) split over gridDim.y
__global__ void __launch_bounds__(kAxThreads) axisym_assemble_kernel(const double* __restrict__ rec, int rec_stride,
                                                                      int n, size_t ld, double* __restrict__ a64,
                                                                      float* __restrict__ a32)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const int per = (n + gridDim.y - 1) / gridDim.y;
    const int j0 = blockIdx.y * per, j1 = min(n, j0 + per);
    const double* t = rec + (size_t) i * rec_stride;
    const double cx = t[aCx], cy = t[aCy], cz = t[aCz];
    for (int j = j0; j < j1; j++) {
        const double a = ax_potential(rec + (size_t) j * rec_stride, cx, cy, cz);
        a64[(size_t) j * ld + i] = a;
        if (a32)
            a32[(size_t) j * ld + i] = (float) a;
    }
}

// blocks along the element (or column) range: about four waves of resident CTAs in all, each
// block keeping at least 8 elements
inline int axisym_split(int num_sms, size_t rows, size_t cols)
{
    const size_t blocks = (rows + kAxThreads - 1) / kAxThreads;
    const size_t want = (size_t) num_sms * kAxFieldMinBlocks * 4;
    size_t split = blocks >= want ? 1 : (want + blocks - 1) / blocks;
    split = std::min(split, std::max((size_t) 1, cols / 8));
    return (int) std::min(split, (size_t) 65535);
}

// the diagonal A(i, i) (Robin Hood on the assembled operator)
__global__ void axisym_diag_kernel(const double* __restrict__ rec, int rec_stride, int n, double* __restrict__ diag)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const double* t = rec + (size_t) i * rec_stride;
    diag[i] = ax_potential(t, t[aCx], t[aCy], t[aCz]);
}

// one matrix entry
__global__ void axisym_entry_kernel(const double* __restrict__ rec, int rec_stride, int i, int j, double* __restrict__ a)
{
    const double* t = rec + (size_t) i * rec_stride;
    *a = ax_potential(rec + (size_t) j * rec_stride, t[aCx], t[aCy], t[aCz]);
}
}  // namespace kemcu
