// Cubature and quadrature rule tables, built on the host at context creation and copied to
// __constant__ memory.
//
// The rules are the published ones the reference's numeric integrator uses; their nodes and
// weights must be identical for parity, so they are restated here in orbit form (a few
// parameters per symmetry orbit plus the orbit's permutations), expanded in the same node
// order as the reference:
//   triangle 7-point  : Radon / Stroud T2 5-1 (KElectrostaticCubatureTriangleIntegrator.hh:68-86, .cc:36-70)
//   triangle 12-point : Gatermann 1988 (…Triangle….hh:88-116, .cc:72-118)
//   triangle 33-point : Papanicolopulos 2011 (…Triangle….hh:208-258, .cc:211-268)
//   rectangle 7-point : Stroud C2 5-1 (KElectrostaticCubatureRectangleIntegrator.hh:9,60-66, .cc:46-102)
//   rectangle 12-point: Stroud C2 7-1 / Tyler 1953 (…Rectangle….hh:82-98, .cc:120-160)
//   rectangle 33-point: Cools-Haegemans 1988 (…Rectangle….hh:141-158, .cc:235-290)
// Line segments use Gauss-Legendre rules of 4 and 16 nodes
// (KElectrostaticQuadratureLineSegmentIntegrator.hh:47-80); their nodes are computed here by
// Newton iteration on the Legendre polynomial instead of being tabulated.
#pragma once

#include <cmath>

namespace kemcu
{
namespace tables
{

struct TriOrbit
{
    int n_perm;   // 1, 3 (cyclic), 3 (swap pattern) or 6
    int pattern;  // 0 centroid, 1 = {abg, bag, gba}, 2 = cyclic {abg, bga, gab}, 3 = all six
    double alpha, beta, weight;
};

// permutations of (alpha, beta, gamma) -> coefficients of (P0, P1, P2)
static const int kSwap3[3][3] = {{0, 1, 2}, {1, 0, 2}, {2, 1, 0}};
static const int kCyclic3[3][3] = {{0, 1, 2}, {1, 2, 0}, {2, 0, 1}};
static const int kAll6[6][3] = {{0, 1, 2}, {1, 0, 2}, {2, 1, 0}, {0, 2, 1}, {2, 0, 1}, {1, 2, 0}};

inline int expand_tri(const TriOrbit* orb, int n_orb, double* out /* s, t, w triples */)
{
    int k = 0;
    for (int o = 0; o < n_orb; o++) {
        const double g = 1. - orb[o].alpha - orb[o].beta;
        const double abg[3] = {orb[o].alpha, orb[o].beta, g};
        const int(*perm)[3] = orb[o].pattern == 2 ? kCyclic3 : orb[o].pattern == 3 ? kAll6 : kSwap3;
        const int np = orb[o].pattern == 0 ? 1 : orb[o].pattern == 3 ? 6 : 3;
        for (int p = 0; p < np; p++) {
            // node = c0*P0 + c1*P1 + c2*P2 = P0 + c1*(A N1) + c2*(B N2)
            out[3 * k] = abg[perm[p][1]];
            out[3 * k + 1] = abg[perm[p][2]];
            out[3 * k + 2] = orb[o].weight;
            k++;
        }
    }
    return k;
}

inline int expand_rect(const double* x, const double* y, const double* w, int n, double* out)
{
    for (int k = 0; k < n; k++) {
        out[3 * k] = 0.5 * (1. + x[k]);
        out[3 * k + 1] = 0.5 * (1. + y[k]);
        out[3 * k + 2] = w[k];
    }
    return n;
}

// Gauss-Legendre positive half rule of order n (n even): x_i > 0, w_i
inline void gauss_legendre_half(int n, double* x, double* w)
{
    for (int i = 0; i < n / 2; i++) {
        long double z = cosl(3.14159265358979323846264338327950288L * (n / 2 - i - 0.25L) / (n + 0.5L));
        long double dp = 0.L;
        for (int it = 0; it < 100; it++) {
            long double p0 = 1.L, p1 = z;
            for (int k = 2; k <= n; k++) {
                const long double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            dp = n * (z * p1 - p0) / (z * z - 1.L);
            const long double dz = p1 / dp;
            z -= dz;
            if (fabsl(dz) < 1e-30L)
                break;
        }
        x[i] = (double) z;
        w[i] = (double) (2.L / ((1.L - z * z) * dp * dp));
    }
}

// rules: 104 (s, t, w) triples in the kTri7 ... kRect33 layout; gl: 10 (x, w) pairs
inline void build(double* rules, double* gl)
{
    const double c = 1. / 3., q15 = std::sqrt(15.);
    const double r7 = (1. + q15) / 7., s7 = (1. - q15) / 7.;
    const TriOrbit tri7[3] = {
        {1, 0, c, c, 9. / 40.},
        {3, 1, c + 2. * c * s7, c - c * s7, (155. + q15) / 1200.},
        {3, 1, c + 2. * c * r7, c - c * r7, (155. - q15) / 1200.},
    };
    const TriOrbit tri12[4] = {
        {3, 2, 0.6238226509439084e-1, 0.6751786707392436e-1, 2. * 0.2651702815743450e-1},
        {3, 2, 0.5522545665692000e-1, 0.3215024938520156, 2. * 0.4388140871444811e-1},
        {3, 2, 0.3432430294509488e-1, 0.6609491961867980, 2. * 0.2877504278497528e-1},
        {3, 2, 0.5158423343536001, 0.2777161669764050, 2. * 0.6749318700980879e-1},
    };
    const TriOrbit tri33[8] = {
        {3, 1, 4.570749859701478e-01, 2.714625070149261e-01, 6.254121319590276e-02},
        {3, 1, 1.197767026828138e-01, 4.401116486585931e-01, 4.991833492806094e-02},
        {3, 1, 2.359249810891690e-02, 4.882037509455416e-01, 2.426683808145203e-02},
        {3, 1, 7.814843446812914e-01, 1.092578276593543e-01, 2.848605206887754e-02},
        {3, 1, 9.507072731273288e-01, 2.464636343633559e-02, 7.931642509973638e-03},
        {6, 3, 1.162960196779266e-01, 2.554542286385173e-01, 4.322736365941421e-02},
        {6, 3, 2.303415635526714e-02, 2.916556797383410e-01, 2.178358503860756e-02},
        {6, 3, 2.138249025617059e-02, 1.272797172335894e-01, 1.508367757651144e-02},
    };
    int k = 0;
    k += expand_tri(tri7, 3, rules + 3 * k);
    k += expand_tri(tri12, 4, rules + 3 * k);
    k += expand_tri(tri33, 8, rules + 3 * k);

    // rectangle 7-point (Stroud C2 5-1, the variant the reference selects with GRECTCUB7INDEX1)
    const double r1 = std::sqrt(3. / 5.), s1 = std::sqrt(1. / 3.), t1 = std::sqrt(14. / 15.);
    const double x7[7] = {0., 0., 0., r1, r1, -r1, -r1}, y7[7] = {0., t1, -t1, s1, -s1, s1, -s1};
    const double w7[7] = {2. / 7., 5. / 63., 5. / 63., 5. / 36., 5. / 36., 5. / 36., 5. / 36.};
    k += expand_rect(x7, y7, w7, 7, rules + 3 * k);

    // rectangle 12-point
    const double q583 = std::sqrt(583.);
    const double r12 = std::sqrt(6. / 7.), s12 = std::sqrt((114. - 3. * q583) / 287.),
                 t12 = std::sqrt((114. + 3. * q583) / 287.);
    const double x12[12] = {r12, -r12, 0., 0., s12, s12, -s12, -s12, t12, t12, -t12, -t12};
    const double y12[12] = {0., 0., r12, -r12, s12, -s12, s12, -s12, t12, -t12, t12, -t12};
    const double B1 = 49. / 810., B2 = (178981. + 2769. * q583) / 1888920., B3 = (178981. - 2769. * q583) / 1888920.;
    const double w12[12] = {B1, B1, B1, B1, B2, B2, B2, B2, B3, B3, B3, B3};
    k += expand_rect(x12, y12, w12, 12, rules + 3 * k);

    // rectangle 33-point: centre plus eight orbits of the 90-degree rotation group
    const double X[9] = {0.00000000000000000000, 0.77880971155441942252, 0.95729769978630736566,
                         0.13818345986246535375, 0.94132722587292523695, 0.47580862521827590507,
                         0.75580535657208143627, 0.69625007849174941396, 0.34271655604040678941};
    const double Y[9] = {0.00000000000000000000, 0.98348668243987226379, 0.85955600564163892859,
                         0.95892517028753485754, 0.39073621612946100068, 0.85007667369974857597,
                         0.64782163718701073204, 0.70741508996444936217e-1, 0.40930456169403884330};
    const double W[9] = {0.30038211543122536139, 0.29991838864499131666e-1, 0.38174421317083669640e-1,
                         0.60424923817749980681e-1, 0.77492738533105339358e-1, 0.11884466730059560108,
                         0.12976355037000271129, 0.21334158145718938943, 0.25687074948196783651};
    double x33[33], y33[33], w33[33];
    x33[0] = X[0];
    y33[0] = Y[0];
    w33[0] = W[0] / 4.;
    for (int o = 1; o < 9; o++) {
        const double xs[4] = {X[o], -X[o], -Y[o], Y[o]}, ys[4] = {Y[o], -Y[o], X[o], -X[o]};
        for (int p = 0; p < 4; p++) {
            x33[1 + 4 * (o - 1) + p] = xs[p];
            y33[1 + 4 * (o - 1) + p] = ys[p];
            w33[1 + 4 * (o - 1) + p] = W[o] / 4.;
        }
    }
    k += expand_rect(x33, y33, w33, 33, rules + 3 * k);

    double x[8], w[8];
    gauss_legendre_half(4, x, w);
    for (int i = 0; i < 2; i++) {
        gl[2 * i] = x[i];
        gl[2 * i + 1] = w[i];
    }
    gauss_legendre_half(16, x, w);
    for (int i = 0; i < 8; i++) {
        gl[2 * (2 + i)] = x[i];
        gl[2 * (2 + i) + 1] = w[i];
    }
}

}  // namespace tables
}  // namespace kemcu
