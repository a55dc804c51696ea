/* kem_oracle.c -- plain-C restatement of the reference's FP64 CPU hot path.
 *
 * TEST INFRASTRUCTURE: only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
 * use it, as a checker. It is pinned against the reference's own outputs (the golden
 * fixtures made by tests/golden/make_golden.py from oracle/_ref, the reference compiled from
 * its sources) in tests/test_cpu_oracle.py.
 *
 * Paths below are relative to the reference project (KEMField/Source/...).
 */
#include "kem_oracle.h"

#include <math.h>
#include <string.h>

static double R_tri[3][33 * 3], R_rect[3][33 * 3], R_gl4[2 * 2], R_gl16[8 * 2];
static const int N_RULE[3] = {33, 12, 7}; /* band 1, 2, 3 */
static double K4PE = 8.987551792261171e9, EPS0 = 8.8541878128e-12;

void kemo_set_rules(const double* tri7, const double* tri12, const double* tri33, const double* rect7,
                    const double* rect12, const double* rect33, const double* gl4, const double* gl16)
{
    memcpy(R_tri[0], tri33, 33 * 3 * sizeof(double));
    memcpy(R_tri[1], tri12, 12 * 3 * sizeof(double));
    memcpy(R_tri[2], tri7, 7 * 3 * sizeof(double));
    memcpy(R_rect[0], rect33, 33 * 3 * sizeof(double));
    memcpy(R_rect[1], rect12, 12 * 3 * sizeof(double));
    memcpy(R_rect[2], rect7, 7 * 3 * sizeof(double));
    memcpy(R_gl4, gl4, sizeof R_gl4);
    memcpy(R_gl16, gl16, sizeof R_gl16);
}

void kemo_set_constants(double one_over_four_pi_eps0, double eps0)
{
    K4PE = one_over_four_pi_eps0;
    EPS0 = eps0;
}

/* ------------------------------------------------------------------ small vector helpers */
typedef struct {
    double x, y, z;
} v3;
static v3 V(double x, double y, double z)
{
    v3 r = {x, y, z};
    return r;
}
static v3 sub(v3 a, v3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
static v3 add(v3 a, v3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
static v3 scl(double s, v3 a) { return V(s * a.x, s * a.y, s * a.z); }
static double dot3(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static v3 crs(v3 a, v3 b) { return V(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static double nrm(v3 a) { return sqrt(dot3(a, a)); }
static v3 ld(const double* p) { return V(p[0], p[1], p[2]); }

/* ------------------------------------------------------------------ cubature
 * Potential_TriNP / ElectricField_TriNP (Numeric/src/KElectrostaticCubatureTriangleIntegrator.cc:271-450)
 * and the rectangle analogues (…CubatureRectangleIntegrator.cc:290-460): nodes
 * Q = P0 + s A N1 + t B N2, sum w (P-Q)/|P-Q|^3 and w/|P-Q|, times area / (4 pi eps0). */
static void cubature(const double* g, double area, const double* rule, int n, v3 P, double* o)
{
    const v3 P0 = ld(g + 2), a = scl(g[0], ld(g + 5)), b = scl(g[1], ld(g + 8));
    double s[4] = {0, 0, 0, 0};
    for (int k = 0; k < n; k++) {
        const v3 Q = add(P0, add(scl(rule[3 * k], a), scl(rule[3 * k + 1], b)));
        const v3 d = sub(P, Q);
        const double ir = 1. / sqrt(dot3(d, d)), w = rule[3 * k + 2];
        s[0] += w * ir * ir * ir * d.x;
        s[1] += w * ir * ir * ir * d.y;
        s[2] += w * ir * ir * ir * d.z;
        s[3] += w * ir;
    }
    const double pf = area * K4PE;
    for (int c = 0; c < 4; c++)
        o[c] = pf * s[c];
}

/* ------------------------------------------------------------------ RWG near field
 * KElectrostaticRWGTriangleIntegrator.cc:8-18 (log-argument expansion), :20-605 (edge line
 * integrals), :607-1239 (point classification, vertex averaging); the rectangle version
 * KElectrostaticRWGRectangleIntegrator.cc; solid angles KSurfaces/include/KSolidAngle.hh:58-…. */
typedef struct {
    int nv;
    v3 v[4], L[4], u[4], mid[4], m[4], n3, n3raw, cen;
    double len[4];
} poly;

static void make_poly(int shape, const double* g, poly* q)
{
    const double A = g[0], B = g[1];
    const v3 P0 = ld(g + 2), N1 = ld(g + 5), N2 = ld(g + 8);
    const v3 a = scl(A, N1), b = scl(B, N2);
    q->n3raw = crs(N1, N2);
    q->n3 = scl(1. / nrm(q->n3raw), q->n3raw);
    if (shape == 0) {
        q->nv = 3;
        q->v[0] = P0;
        q->v[1] = add(P0, a);
        q->v[2] = add(P0, b);
        for (int c = 0; c < 3; c++)
            ((double*) &q->cen)[c] = g[2 + c] + (A * g[5 + c] + B * g[8 + c]) / 3.;
        const v3 e12 = sub(q->v[2], q->v[1]);
        q->L[0] = a;
        q->L[1] = e12;
        q->L[2] = scl(-1., b);
        q->len[0] = A;
        q->len[1] = nrm(e12);
        q->len[2] = B;
        q->u[0] = N1;
        q->u[1] = scl(1. / q->len[1], e12);
        q->u[2] = scl(-1., N2);
    }
    else {
        q->nv = 4;
        q->v[0] = P0;
        q->v[1] = add(P0, a);
        q->v[2] = add(q->v[1], b);
        q->v[3] = add(P0, b);
        for (int c = 0; c < 3; c++)
            ((double*) &q->cen)[c] = (g[2 + c] + A * g[5 + c] * .5) + B * g[8 + c] * .5;
        q->L[0] = a;
        q->L[1] = b;
        q->L[2] = scl(-1., a);
        q->L[3] = scl(-1., b);
        q->len[0] = A;
        q->len[1] = B;
        q->len[2] = A;
        q->len[3] = B;
        q->u[0] = N1;
        q->u[1] = N2;
        q->u[2] = scl(-1., N1);
        q->u[3] = scl(-1., N2);
    }
    for (int i = 0; i < q->nv; i++) {
        q->mid[i] = add(scl(0.5 * q->len[i], q->u[i]), q->v[i]);
        q->m[i] = crs(q->u[i], q->n3);
    }
}

static double tri_omega(v3 a, v3 b, v3 c, v3 P)
{
    const v3 ua = scl(1. / nrm(sub(a, P)), sub(a, P)), ub = scl(1. / nrm(sub(b, P)), sub(b, P)),
             uc = scl(1. / nrm(sub(c, P)), sub(c, P));
    const double x = 1. + dot3(ua, ub) + dot3(ua, uc) + dot3(ub, uc);
    const double y = fabs(dot3(ua, crs(ub, uc)));
    return fabs(2. * atan2(y, x));
}

static double omega(const poly* q, v3 P)
{
    const double pi = 3.141592653589793238462643383279502884;
    double res, h;
    if (q->nv == 3) {
        h = dot3(q->n3, sub(P, q->cen));
        res = nrm(sub(P, q->cen)) <= 1e-12 ? 2. * pi : tri_omega(q->v[0], q->v[1], q->v[2], P);
    }
    else {
        h = dot3(q->n3raw, sub(P, q->cen));
        if (fabs(h) < 1e-12) {
            const v3 dP = sub(q->v[0], P);
            const double l1 = -dot3(dP, q->L[0]) / (q->len[0] * q->len[0]);
            const double l2 = -dot3(dP, q->L[1]) / (q->len[1] * q->len[1]);
            res = (l1 > 0. && l1 < 1. && l2 > 0. && l2 < 1.) ? 2. * pi : 0.;
        }
        else
            res = tri_omega(q->v[0], q->v[1], q->v[2], P) + tri_omega(q->v[2], q->v[3], q->v[0], P);
    }
    return h < 0. ? -res : res;
}

static void rwg_at(const poly* q, v3 P, int counter, int line, double dist, double* o)
{
    double il = 0.;
    v3 iv = V(0, 0, 0);
    for (int i = 0; i < q->nv; i++) {
        const int j = (i + 1) % q->nv;
        const v3 dm = sub(q->v[i], P), dp = sub(q->v[j], P);
        const double rM = nrm(dm), rP = nrm(dp), sM = dot3(dm, q->u[i]), sP = dot3(dp, q->u[i]);
        double term = 0.;
        int have = 0;
        if (counter == 1 && line == i && fabs(dist / sM) < 1e-6) {
            double qt = fabs(dist / sM);
            if (qt < 1e-14)
                qt = 1e-14;
            term = log(rP + sP) - log(0.5 * fabs(sM) * qt * qt);
            have = 1;
        }
        if (line != i) {
            const int upper = (rM + sM) > (rP - sP);
            term += upper ? log(rP + sP) - log(rM + sM) : log(rM - sM) - log(rP - sP);
            have = 1;
        }
        if (have) {
            il += dot3(q->m[i], sub(P, q->mid[i])) * term;
            iv = add(iv, scl(term, q->m[i]));
        }
    }
    const double om = omega(q, P);
    o[0] = q->n3.x * om + iv.x;
    o[1] = q->n3.y * om + iv.y;
    o[2] = q->n3.z * om + iv.z;
    o[3] = -dot3(q->n3, sub(P, q->cen)) * om - il;
}

static void rwg(int shape, const double* g, v3 P, double* o)
{
    poly q;
    make_poly(shape, g, &q);
    int counter = 0, line = 99;
    double dmin = 0.;
    for (int i = 0; i < q.nv; i++) {
        const v3 dv = sub(q.v[i], P);
        const double inv = 1. / q.len[i];
        const double dl = nrm(crs(q.L[i], dv)) * inv, lam = -dot3(dv, q.L[i]) * inv * inv;
        if (dl < 1e-14 && lam >= -1e-15 && lam <= 1. + 1e-15) {
            dmin = dl;
            counter++;
            line = i;
        }
    }
    if (counter == 2) {
        double a[4], b[4];
        rwg_at(&q, add(P, scl(1e-7, q.n3)), 9, 9, 9., a);
        rwg_at(&q, sub(P, scl(1e-7, q.n3)), 9, 9, 9., b);
        for (int c = 0; c < 4; c++)
            o[c] = K4PE * 0.5 * (a[c] + b[c]);
        return;
    }
    rwg_at(&q, P, counter, line, dmin, o);
    for (int c = 0; c < 4; c++)
        o[c] *= K4PE;
}

/* ------------------------------------------------------------------ line segments
 * Gauss-Legendre (Numeric/src/KElectrostaticQuadratureLineSegmentIntegrator.cc:126-190) and the
 * analytic wire (Analytic/src/KElectrostaticAnalyticLineSegmentIntegrator.cc:15-82). */
static void line_gauss(const double* g, const double* rule, int half, v3 P, double* o)
{
    const v3 p0 = ld(g), p1 = ld(g + 3);
    const double L = nrm(sub(p1, p0)), hl = 0.5 * L;
    const v3 c = scl(0.5, add(p0, p1)), u = scl(1. / L, sub(p1, p0));
    double s[4] = {0, 0, 0, 0};
    for (int i = 0; i < half; i++) {
        const double wf = rule[2 * i + 1] * hl, x = rule[2 * i] * hl;
        const v3 dp = sub(P, add(c, scl(x, u))), dn = sub(P, sub(c, scl(x, u)));
        const double ip = 1. / nrm(dp), in = 1. / nrm(dn);
        s[3] += wf * (ip + in);
        s[0] += wf * (ip * ip * ip * dp.x + in * in * in * dn.x);
        s[1] += wf * (ip * ip * ip * dp.y + in * in * in * dn.y);
        s[2] += wf * (ip * ip * ip * dp.z + in * in * in * dn.z);
    }
    const double pf = 0.25 * g[6] / EPS0;
    for (int k = 0; k < 4; k++)
        o[k] = pf * s[k];
}

static void line_analytic(const double* g, v3 P, double* o)
{
    const v3 p0 = ld(g), p1 = ld(g + 3);
    const double d = g[6], L = nrm(sub(p1, p0)), Da0 = nrm(sub(p0, P)), Db0 = nrm(sub(p1, P));
    int inside = 0;
    v3 pp = V(0, 0, 0);
    if (!((Da0 + Db0) > (L + d))) {
        const v3 u = scl(1. / L, sub(p1, p0));
        const double p = dot3(sub(P, p0), u);
        if (!(p < -d * .5 || p > L + d * .5)) {
            pp = add(p0, scl(p, u));
            inside = !(nrm(sub(P, pp)) >= d * .5);
        }
    }
    double Da = Da0, Db = Db0;
    if (inside) {
        Da = sqrt(dot3(sub(p0, pp), sub(p0, pp)) + d * d * .25);
        Db = sqrt(dot3(sub(p1, pp), sub(p1, pp)) + d * d * .25);
    }
    o[3] = d / (4. * EPS0) * log((Da + Db + L) / (Da + Db - L));
    Da = Da0;
    Db = Db0;
    if (inside) {
        Da = nrm(sub(p0, pp));
        Db = nrm(sub(p1, pp));
    }
    const double den = -1. / ((Da * (Da + Db + L) * (Da + Db - L) * Db) * 4. * EPS0);
    const double s = 2. * L * d * den;
    o[0] = s * (p1.x * Da - P.x * (Da + Db) + p0.x * Db);
    o[1] = s * (p1.y * Da - P.y * (Da + Db) + p0.y * Db);
    o[2] = s * (p1.z * Da - P.z * (Da + Db) + p0.z * Db);
}

/* ------------------------------------------------------------------ axisymmetric elements
 * conic section geom = (r0, z0, r1, z1), ring geom = (r, z): KConicSection.hh, KRing.hh */

/* complete elliptic integrals in W. J. Cody's form (Math. Comp. 19 (1965) 105) with his
   coefficient sets, as Math/src/KEllipticIntegrals.cc:17-103 (its build without GSL) */
#define KEMO_PI 3.14159265358979323846 /* KEMConstants::Pi, KConst::Pi() */
static const double CODY_KA[10] = {9.657359028085625e-2, 3.088514627130518e-2, 1.493801353268716e-2,
                                   8.789801874555064e-3, 6.179627446053317e-3, 6.847909282624505e-3,
                                   9.848929322176893e-3, 8.003003980649985e-3, 2.296634898396958e-3,
                                   1.393087857006646e-4};
static const double CODY_KB[10] = {1.249999999999080e-1, 7.031249973903835e-2, 4.882804190686239e-2,
                                   3.737773975862360e-2, 3.012484901289893e-2, 2.393191332311079e-2,
                                   1.553094163197720e-2, 5.973904299155429e-3, 9.215546349632498e-4,
                                   2.970028096655561e-5};
static const double CODY_EC[10] = {4.431471805608895e-1, 5.680519456755915e-2, 2.183181167613048e-2,
                                   1.156959574529540e-2, 7.595093422559432e-3, 7.820404060959554e-3,
                                   1.077063503986645e-2, 8.638442173604074e-3, 2.468503330460722e-3,
                                   1.494662175718132e-4};
static const double CODY_ED[10] = {2.499999999999017e-1, 9.374999972120314e-2, 5.859366125553149e-2,
                                   4.271789054738309e-2, 3.347894366576162e-2, 2.614501470031387e-2,
                                   1.680402334636338e-2, 6.432146586438301e-3, 9.898332846225384e-4,
                                   3.185919565550157e-5};

static double ell_K(double k)
{
    const double eta = 1. - k * k;
    double en = eta, sa = 0., sb = 0.;
    for (int i = 0; i < 10; i++) {
        sa += CODY_KA[i] * en;
        sb += CODY_KB[i] * en;
        en *= eta;
    }
    return 1.386294361119890 + sa - (1. / 2. + sb) * log(fabs(eta) + 1.e-19);
}

static double ell_E(double k)
{
    const double eta = 1. - k * k;
    double en = eta, sc = 0., sd = 0.;
    for (int i = 0; i < 10; i++) {
        sc += CODY_EC[i] * en;
        sd += CODY_ED[i] * en;
        en *= eta;
        if (en < 1.e-20)
            break;
    }
    return 1. + sc - sd * log(fabs(eta) + 1.e-19);
}

/* (E - K) / k^2: difference for k^2 > 0.8, power series below (KEllipticIntegrals.cc:108-131) */
static double ell_EK(double k)
{
    const double k2 = k * k;
    if (k2 > 0.8)
        return (ell_E(k) - ell_K(k)) / k2;
    double a = KEMO_PI / 2., k2n = 1., ek = 0.;
    for (int n = 1; n <= 900; n++) {
        const double cn = (2. * n - 1) / (2. * n);
        a *= cn * cn;
        const double b = -a / (2. * n - 1.);
        ek += (b - a) * k2n;
        k2n *= k2;
        if (k2n < 1.e-16)
            break;
    }
    return ek;
}

/* ring at distance p along the generator par = (z, r, zA, rA, zB, rB, L): potential R K / S and
   field components R / S^3 (-2 R EK + dr E / eta), dz / S^3 E / eta R
   (BoundaryIntegrals/Electrostatic/Analytic/src/KElectrostaticAnalyticRingIntegrator.cc:95-208) */
static double ring_potential(double p, const double* par)
{
    const double Z = par[2] + p / par[6] * (par[4] - par[2]);
    const double R = par[3] + p / par[6] * (par[5] - par[3]);
    const double dz = par[0] - Z, dr = par[1] - R, sumr = R + par[1];
    const double eta = (dr * dr + dz * dz) / (sumr * sumr + dz * dz);
    const double k = (eta > 1. ? 0. : sqrt(1. - eta));
    const double K = ell_K(k);
    const double S = sqrt(sumr * sumr + dz * dz);
    return R * K / S;
}

static double ring_er(double p, const double* par)
{
    const double Z = par[2] + p / par[6] * (par[4] - par[2]);
    const double R = par[3] + p / par[6] * (par[5] - par[3]);
    const double dz = par[0] - Z, dr = par[1] - R, sumr = R + par[1];
    const double eta = (dr * dr + dz * dz) / (sumr * sumr + dz * dz);
    const double k = sqrt(1. - eta);
    const double E = ell_E(k);
    const double S = sqrt(sumr * sumr + dz * dz);
    const double EK = ell_EK(k);
    return R / (S * S * S) * (-2. * R * EK + dr / eta * E);
}

static double ring_ez(double p, const double* par)
{
    const double Z = par[2] + p / par[6] * (par[4] - par[2]);
    const double R = par[3] + p / par[6] * (par[5] - par[3]);
    const double dz = par[0] - Z, dr = par[1] - R, sumr = R + par[1];
    const double eta = (dr * dr + dz * dz) / (sumr * sumr + dz * dz);
    const double k = sqrt(1. - eta);
    const double E = ell_E(k);
    const double S = sqrt(sumr * sumr + dz * dz);
    return dz / (S * S * S) * E / eta * R;
}

/* F. Glueck's composite rule, its n >= 20 branch (Math/src/KGaussianQuadrature.cc:18-86): m = 1
   integrates the ring potential, m = 2 the two field components */
static void glueck(int m, double a, double b, const double* par, int n, double* ans)
{
    static const double w9[10] = {0.2803440531305107e0,  0.1648702325837748e1, -0.2027449845679092e0,
                                  0.2797927414021179e1,  -0.9761199294532843e0, 0.2556499393738999e1,
                                  0.1451083002645404e0,  0.1311227127425048e1,  0.9324249063051143e0,
                                  0.1006631393298060e1};
    const double deln = (b - a) / n;
    double x;
    for (int j = 0; j < m; j++)
        ans[j] = 0;
#define KEMO_F(j, x) ((m == 1) ? ring_potential((x), par) : ((j) == 0 ? ring_er((x), par) : ring_ez((x), par)))
    for (int i = 0; i < 10; i++) {
        x = a + deln * i;
        for (int j = 0; j < m; j++)
            ans[j] += w9[i] * KEMO_F(j, x);
    }
    for (int i = 10; i < n - 9; i++) {
        x = a + deln * i;
        for (int j = 0; j < m; j++)
            ans[j] += KEMO_F(j, x);
    }
    for (int i = n - 9; i <= n; i++) {
        x = a + deln * i;
        for (int j = 0; j < m; j++)
            ans[j] += w9[n - i] * KEMO_F(j, x);
    }
#undef KEMO_F
    for (int j = 0; j < m; j++)
        ans[j] *= deln;
}

/* the conic-section integral of m ring integrands: 20 / 100 / 500 intervals by the distance
   excess D, else the generator cut at the foot point and each side integrated in pieces
   shrinking by 0.3, plus the logarithmic remainder (added to every component, as the
   reference does) (Analytic/src/KElectrostaticAnalyticConicSectionIntegrator.cc:33-93, 113-198) */
static void conic_integral(int m, const double* par, double* q)
{
    const double ln4 = 1.386294361119890;
    const double z = par[0], r = par[1], za = par[2], ra = par[3], zb = par[4], rb = par[5], L = par[6];
    const double Da = sqrt((za - z) * (za - z) + (ra - r) * (ra - r));
    const double Db = sqrt((zb - z) * (zb - z) + (rb - r) * (rb - r));
    const double D = fabs(Da + Db - L) / L;
    if (D >= 5.e-2) {
        glueck(m, 0., L, par, 20, q);
        return;
    }
    if (D >= 5.e-3 && D < 5.e-2) {
        glueck(m, 0., L, par, 100, q);
        return;
    }
    if (D >= 5.e-4 && D < 5.e-3) {
        glueck(m, 0., L, par, 500, q);
        return;
    }
    const double u0 = (zb - za) / L, u1 = (rb - ra) / L;
    const double pp = (z - za) * u0 + (r - ra) * u1;
    double tmp[2], a, b, h;
    for (int j = 0; j < m; j++)
        q[j] = 0.;
    if (pp < L) {
        const double pmax = L;
        double pmin = pp;
        if (pp < 0.)
            pmin = 0.;
        b = pmax;
        a = pmin + (b - pmin) * 0.3;
        for (int n = 1; n <= 35; n++) {
            glueck(m, a, b, par, 50, tmp);
            for (int j = 0; j < m; j++)
                q[j] += tmp[j];
            if (fabs(a - pmin) / L < 1.e-8)
                break;
            b = a;
            a = pmin + (b - pmin) * 0.3;
        }
        h = fabs(a - pmin);
        for (int j = 0; j < m; j++)
            q[j] += h * (ln4 + log(2. * par[1] + 1.e-12) + 1. - log(h)) / 2.;
    }
    if (pp > 0.) {
        double pmax = pp;
        const double pmin = 0.;
        if (pp > L)
            pmax = L;
        b = pmin;
        a = pmax - (pmax - b) * 0.3;
        for (int n = 1; n <= 35; n++) {
            glueck(m, b, a, par, 50, tmp);
            for (int j = 0; j < m; j++)
                q[j] += tmp[j];
            if (fabs(pmax - a) / L < 1.e-8)
                break;
            b = a;
            a = pmax - (pmax - b) * 0.3;
        }
        h = fabs(pmax - a);
        for (int j = 0; j < m; j++)
            q[j] += h * (ln4 + log(2. * par[1] + 1.e-12) + 1. - log(h)) / 2.;
    }
}

/* field and potential per unit charge density of a conic section (shape 3) or ring (shape 4);
   E_r turned into (E_x, E_y), zero within 1e-14 of the axis
   (KElectrostaticAnalyticConicSectionIntegrator.cc:9-221, KElectrostaticAnalyticRingIntegrator.cc:26-68) */
static void axisym_element(int shape, const double* g, v3 P, double* o)
{
    double par[7];
    par[0] = P.z;
    par[1] = sqrt(P.x * P.x + P.y * P.y);
    double c, er, ez, pot;
    if (shape == 4) {
        par[2] = par[4] = g[1];
        par[3] = par[5] = g[0];
        par[6] = 1.;
        c = 1. / (par[3] * 2. * KEMO_PI * KEMO_PI * EPS0);
        pot = c * ring_potential(P.x, par);
        ez = c * ring_ez(P.x, par);
        er = c * ring_er(P.x, par);
    }
    else {
        par[2] = g[1];
        par[3] = g[0];
        par[4] = g[3];
        par[5] = g[2];
        par[6] = sqrt((g[0] - g[2]) * (g[0] - g[2]) + 0. * 0. + (g[1] - g[3]) * (g[1] - g[3]));
        double q1[1], q2[2];
        conic_integral(1, par, q1);
        conic_integral(2, par, q2);
        c = 1. / (KEMO_PI * EPS0);
        pot = c * q1[0];
        er = c * q2[0];
        ez = c * q2[1];
    }
    o[2] = ez;
    o[3] = pot;
    if (par[1] < 1.e-14)
        o[0] = o[1] = 0.;
    else {
        o[0] = P.x / par[1] * er;
        o[1] = P.y / par[1] * er;
    }
}

/* ------------------------------------------------------------------ dispatch
 * distance ratio |P - centroid| / size and the rule bands
 * (…CubatureTriangleIntegrator.cc:453-522, .hh:51-53; …CubatureRectangleIntegrator.cc:462-520,
 * .hh:52-54; …QuadratureLineSegmentIntegrator.cc:193-240, .hh:43-44) */
void kemo_element(int shape, const double* g, const double* Pp, double* o)
{
    const v3 P = ld(Pp);
    if (shape == 3 || shape == 4) {
        axisym_element(shape, g, P, o);
        return;
    }
    if (shape == 2) {
        const double L = sqrt((g[3] - g[0]) * (g[3] - g[0]) + (g[4] - g[1]) * (g[4] - g[1]) +
                              (g[5] - g[2]) * (g[5] - g[2]));
        const double c[3] = {(g[0] + g[3]) * .5, (g[1] + g[4]) * .5, (g[2] + g[5]) * .5};
        const double ratio =
            sqrt((c[0] - P.x) * (c[0] - P.x) + (c[1] - P.y) * (c[1] - P.y) + (c[2] - P.z) * (c[2] - P.z)) * (1. / L);
        if (ratio > 27.7)
            line_gauss(g, R_gl4, 2, P, o);
        else if (ratio > 2.)
            line_gauss(g, R_gl16, 8, P, o);
        else
            line_analytic(g, P, o);
        return;
    }
    const double A = g[0], B = g[1];
    double cen[3], size, area;
    if (shape == 0) {
        double p1[3], p2[3];
        for (int k = 0; k < 3; k++) {
            p1[k] = g[2 + k] + A * g[5 + k];
            p2[k] = g[2 + k] + B * g[8 + k];
            cen[k] = g[2 + k] + (A * g[5 + k] + B * g[8 + k]) / 3.;
        }
        size = (A + B + sqrt((p2[0] - p1[0]) * (p2[0] - p1[0]) + (p2[1] - p1[1]) * (p2[1] - p1[1]) +
                             (p2[2] - p1[2]) * (p2[2] - p1[2]))) / 3.;
        const v3 cr = crs(ld(g + 5), ld(g + 8));
        area = 0.5 * A * B * nrm(cr);
    }
    else {
        for (int k = 0; k < 3; k++)
            cen[k] = g[2 + k] + 0.5 * (A * g[5 + k] + B * g[8 + k]);
        size = 0.5 * (A + B);
        area = A * B;
    }
    const double ratio = sqrt((cen[0] - P.x) * (cen[0] - P.x) + (cen[1] - P.y) * (cen[1] - P.y) +
                              (cen[2] - P.z) * (cen[2] - P.z)) *
                         (1. / size);
    const double* cut = shape == 0 ? (const double[]){3.42, 30.4, 131.4} : (const double[]){4.6, 44.6, 196.2};
    int band = ratio > cut[2] ? 3 : ratio > cut[1] ? 2 : ratio > cut[0] ? 1 : 0;
    if (band == 0) {
        rwg(shape, g, P, o);
        return;
    }
    cubature(g, area, shape == 0 ? R_tri[band - 1] : R_rect[band - 1], N_RULE[band - 1], P, o);
}

/* Kahan-summed direct sum (FieldSolvers/Integrating/include/KElectrostaticIntegratingFieldSolver.hh:301-339) */
void kemo_field(size_t n, const int* shape, const double* geom, const double* sigma, size_t m, const double* P,
                double* out)
{
    for (size_t p = 0; p < m; p++) {
        double s[4] = {0, 0, 0, 0}, c[4] = {0, 0, 0, 0};
        for (size_t j = 0; j < n; j++) {
            double o[4];
            kemo_element(shape[j], geom + 11 * j, P + 3 * p, o);
            for (int k = 0; k < 4; k++) {
                const double y = o[k] * sigma[j] - c[k];
                const double t = s[k] + y;
                c[k] = (t - s[k]) - y;
                s[k] = t;
            }
        }
        memcpy(out + 4 * p, s, sizeof s);
    }
}

/* target centroid and normal of element i (KTriangle/KRectangle/KLineSegment Centroid(), Normal()) */
static void target(int shape, const double* g, double* c, double* nv)
{
    if (shape == 3 || shape == 4) {  /* (P0 + P1) / 2 (KConicSection.hh:29-32), P (KRing.hh:29-32) */
        c[0] = shape == 3 ? (g[0] + g[2]) * .5 : g[0];
        c[1] = 0.;
        c[2] = shape == 3 ? (g[1] + g[3]) * .5 : g[1];
        nv[0] = nv[1] = nv[2] = 0.;
        return;
    }
    if (shape == 2) {
        for (int k = 0; k < 3; k++)
            c[k] = (g[k] + g[3 + k]) * .5;
        const v3 d = sub(ld(g + 3), ld(g));
        const v3 nn = d.x > 1e-10 ? crs(d, V(1, 0, 0)) : crs(d, V(0, 1, 0));
        const v3 u = scl(1. / nrm(nn), nn);
        nv[0] = u.x;
        nv[1] = u.y;
        nv[2] = u.z;
        return;
    }
    const v3 cr = crs(ld(g + 5), ld(g + 8));
    for (int k = 0; k < 3; k++)
        c[k] = shape == 0 ? g[2 + k] + (g[0] * g[5 + k] + g[1] * g[8 + k]) / 3.
                          : (g[2 + k] + g[0] * g[5 + k] * .5) + g[1] * g[8 + k] * .5;
    const v3 u = shape == 0 ? scl(1. / nrm(cr), cr) : cr;
    nv[0] = u.x;
    nv[1] = u.y;
    nv[2] = u.z;
}

/* A(i, j) = Dirichlet: phi_j(c_i); Neumann: E_j(c_i) . n_i, or (1+eps)/(1-eps)/(2 eps0) when the
   centroids coincide (BoundaryIntegrals/Electrostatic/Core/include/KElectrostaticBoundaryIntegrator.hh:260-280) */
void kemo_matrix(size_t n, const int* shape, const int* boundary, const double* geom, const double* value, double* A,
                 double* b)
{
    for (size_t i = 0; i < n; i++) {
        double ci[3], ni[3];
        target(shape[i], geom + 11 * i, ci, ni);
        b[i] = boundary[i] == 0 ? value[i] : 0.;
        for (size_t j = 0; j < n; j++) {
            double o[4];
            if (boundary[i] == 0) {
                kemo_element(shape[j], geom + 11 * j, ci, o);
                A[i * n + j] = o[3];
                continue;
            }
            double cj[3], nj[3];
            target(shape[j], geom + 11 * j, cj, nj);
            const double dist = nrm(sub(ld(cj), ld(ci)));
            if (dist >= 1e-12) {
                kemo_element(shape[j], geom + 11 * j, ci, o);
                A[i * n + j] = o[0] * ni[0] + o[1] * ni[1] + o[2] * ni[2];
            }
            else
                A[i * n + j] = ((1. + value[i]) / (1. - value[i])) / (2. * EPS0);
        }
    }
}

/* GMRES from x0 = 0: modified Gram-Schmidt, Givens rotations, back-substitution
   (LinearAlgebra/Solvers/include/KGeneralizedMinimalResidual.hh:178-337 with UseBackSubstitution;
   relative tolerance |p_{j+1}| / |b|, KSimpleIterativeKrylovSolver.hh:84-103) */
int kemo_gmres(size_t n, const double* A, const double* b, double tol, int max_iter, double* x, double* resid)
{
    enum { MAXK = 512 };
    if (max_iter > MAXK - 1)
        max_iter = MAXK - 1;
    static double V[MAXK][4096];
    static double H[MAXK][MAXK], cs[MAXK], sn[MAXK], p[MAXK + 1], y[MAXK];
    if (n > 4096)
        return -1;
    double bn = 0.;
    for (size_t i = 0; i < n; i++)
        bn += b[i] * b[i];
    bn = sqrt(bn);
    for (size_t i = 0; i < n; i++)
        V[0][i] = b[i] / bn;
    p[0] = bn;
    int j = 0;
    for (; j < max_iter; j++) {
        double* w = V[j + 1];
        for (size_t i = 0; i < n; i++) {
            double s = 0.;
            for (size_t k = 0; k < n; k++)
                s += A[i * n + k] * V[j][k];
            w[i] = s;
        }
        for (int r = 0; r <= j; r++) {
            double h = 0.;
            for (size_t i = 0; i < n; i++)
                h += w[i] * V[r][i];
            H[j][r] = h;
            for (size_t i = 0; i < n; i++)
                w[i] -= h * V[r][i];
        }
        double beta = 0.;
        for (size_t i = 0; i < n; i++)
            beta += w[i] * w[i];
        beta = sqrt(beta);
        for (size_t i = 0; i < n; i++)
            w[i] /= beta;
        for (int r = 0; r < j; r++) {
            const double a = H[j][r], c = H[j][r + 1];
            H[j][r] = cs[r] * a + sn[r] * c;
            H[j][r + 1] = -sn[r] * a + cs[r] * c;
        }
        const double g = sqrt(H[j][j] * H[j][j] + beta * beta);
        cs[j] = H[j][j] / g;
        sn[j] = beta / g;
        H[j][j] = g;
        p[j + 1] = -sn[j] * p[j];
        p[j] = cs[j] * p[j];
        if (fabs(p[j + 1]) / bn <= tol) {
            j++;
            break;
        }
    }
    for (int i = j - 1; i >= 0; i--) {
        double s = p[i];
        for (int c = i + 1; c < j; c++)
            s -= H[c][i] * y[c];
        y[i] = s / H[i][i];
    }
    for (size_t i = 0; i < n; i++) {
        double s = 0.;
        for (int k = 0; k < j; k++)
            s += y[k] * V[k][i];
        x[i] = s;
    }
    if (resid)
        *resid = fabs(p[j]) / bn;
    return j;
}

/* 13-stage RK8 (Kassiopeia/Math/Include/KSMathRK8.h:45-226) with the exact-trajectory derivative
   (1, |v|, v, qE), v = p / (m gamma) (Kassiopeia/Trajectories/Source/KSTrajTrajectoryExact.cxx:302-316,
   KSTrajTermPropagation.cxx:25-35) */
static const double RK[13][13] = {
    {1. / 4.},
    {5. / 72., 1. / 72.},
    {1. / 32., 0., 3. / 32.},
    {106. / 125., 0., -408. / 125., 352. / 125.},
    {1. / 48., 0., 0., 8. / 33., 125. / 528.},
    {-1263. / 2401., 0., 0., 39936. / 26411., -64125. / 26411., 5520. / 2401.},
    {37. / 392., 0., 0., 0., 1625. / 9408., -2. / 15., 61. / 6720.},
    {17176. / 25515., 0., 0., -47104. / 25515., 1325. / 504., -41792. / 25515., 20237. / 145800., 4312. / 6075.},
    {-23834. / 180075., 0., 0., -77824. / 1980825., -636635. / 633864., 254048. / 300125., -183. / 7000., 8. / 11.,
     -324. / 3773.},
    {12733. / 7600., 0., 0., -20032. / 5225., 456485. / 80256., -42599. / 7125., 339227. / 912000., -1029. / 4180.,
     1701. / 1408., 5145. / 2432.},
    {-27061. / 204120., 0., 0., 40448. / 280665., -1353775. / 1197504., 17662. / 25515., -71687. / 1166400.,
     98. / 225., 1. / 16., 3773. / 11664.},
    {11203. / 8680., 0., 0., -38144. / 11935., 2354425. / 458304., -84046. / 16275., 673309. / 1636800.,
     4704. / 8525., 9477. / 10912., -1029. / 992., 0., 729. / 341.},
    {31. / 720., 0., 0., 0., 0., 16. / 75., 16807. / 79200., 16807. / 79200., 243. / 1760., 0., 0., 243. / 1760.,
     31. / 720.}};

static void deriv(size_t n, const int* shape, const double* geom, const double* sigma, const double* y, double q,
                  double m, double* dy)
{
    const double c = 299792458.0;
    const double p2 = y[5] * y[5] + y[6] * y[6] + y[7] * y[7];
    const double gam = sqrt(1. + p2 / (m * m * c * c));
    const double inv = 1. / (m * gam);
    double E[4];
    kemo_field(n, shape, geom, sigma, 1, y + 2, E);
    dy[0] = 1.;
    dy[2] = inv * y[5];
    dy[3] = inv * y[6];
    dy[4] = inv * y[7];
    dy[1] = sqrt(dy[2] * dy[2] + dy[3] * dy[3] + dy[4] * dy[4]);
    dy[5] = q * E[0];
    dy[6] = q * E[1];
    dy[7] = q * E[2];
}

void kemo_rk8(size_t n, const int* shape, const double* geom, const double* sigma, double* st, double dt, int nsteps,
              double charge, double mass, double* traj)
{
    double k[13][8], v[8];
    for (int s = 0; s < nsteps; s++) {
        deriv(n, shape, geom, sigma, st, charge, mass, k[0]);
        for (int r = 0; r < 13; r++) {
            for (int c = 0; c < 8; c++) {
                double acc = 0.;
                for (int q = 0; q <= r; q++)
                    acc += RK[r][q] * k[q][c];
                v[c] = st[c] + dt * acc;
            }
            if (r < 12)
                deriv(n, shape, geom, sigma, v, charge, mass, k[r + 1]);
        }
        memcpy(st, v, sizeof v);
        if (traj)
            memcpy(traj + 8 * s, st, sizeof v);
    }
}
