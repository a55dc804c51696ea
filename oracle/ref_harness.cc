// C-ABI harness around the reference's own FP64 CPU hot path (test infrastructure).
//
// Every function here drives unmodified reference classes; nothing is re-implemented:
//   * container + integrator: KSurfaceContainer, KSurface<KElectrostaticBasis, Boundary, Shape>
//     (KEMField/Source/Surfaces/src/KSurfaceContainer.cc:36-72), KEBIFactory::MakeNumeric()
//     (KEMField/Source/BoundaryIntegrals/Electrostatic/Core/src/KElectrostaticBoundaryIntegratorFactory.cc:75-87)
//   * direct summation: KIntegratingFieldSolver<KElectrostaticBoundaryIntegrator>
//     (KEMField/Source/FieldSolvers/Integrating/include/KElectrostaticIntegratingFieldSolver.hh:261-339)
//   * matrix entries / matvec / RHS: KBoundaryIntegralMatrix::operator(), KMatrix::Multiply,
//     KBoundaryIntegralVector (KEMField/Source/BoundaryIntegrals/Core/include/KBoundaryIntegralMatrix.hh:31-55,
//     KEMField/Source/LinearAlgebra/Core/include/KMatrix.hh:92-99)
//   * GMRES: KSimpleIterativeKrylovSolver<double, KGeneralizedMinimalResidual>
//     (KEMField/Source/LinearAlgebra/Solvers/include/KSimpleIterativeKrylovSolver.hh:139-194)
//   * Robin Hood: KRobinHood<double> (KEMField/Source/LinearAlgebra/Solvers/include/KRobinHood.hh:61-104)
//   * RK8: Kassiopeia::KSMathRK8 (Kassiopeia/Math/Include/KSMathRK8.h:45-226) driven by the exact
//     trajectory derivative (1, |v|, v, qE) of KSTrajTrajectoryExact::Differentiate and
//     KSTrajTermPropagation::Differentiate (Kassiopeia/Trajectories/Source/KSTrajTrajectoryExact.cxx:302-316,
//     KSTrajTermPropagation.cxx:25-35) with B = 0.
//
// Element encoding (same as the product's C ABI): shape 0 = triangle, 1 = rectangle,
// 2 = line segment; boundary 0 = Dirichlet (value = potential), 1 = Neumann (value =
// normal boundary flux). geom[11] = {A, B, P0xyz, N1xyz, N2xyz} for triangles and
// rectangles, {P0xyz, P1xyz, diameter, 0...} for line segments.

#include "KBoundaryIntegralMatrix.hh"
#include "KBoundaryIntegralSolutionVector.hh"
#include "KBoundaryIntegralVector.hh"
#include "KConst.h"
#include "KElectrostaticBoundaryIntegratorFactory.hh"
#include "KElectrostaticCubatureRectangleIntegrator.hh"
#include "KElectrostaticCubatureTriangleIntegrator.hh"
#include "KElectrostaticQuadratureLineSegmentIntegrator.hh"
#include "KElectrostaticIntegratingFieldSolver.hh"
#include "KGeneralizedMinimalResidual.hh"
#include "KImplicitKrylovPreconditioner.hh"
#include "KJacobiPreconditioner.hh"
#include "KKrylovSolverConfiguration.hh"
#include "KKrylovSolverFactory.hh"
#include "KRobinHood.hh"
#include "KSMathArray.h"
#include "KSMathRK8.h"
#include "KSMathSystem.h"
#include "KSimpleIterativeKrylovSolver.hh"
#include "KSurface.hh"
#include "KSurfaceContainer.hh"

#include <cmath>
#include <type_traits>
#include <vector>

using namespace KEMField;

namespace
{
struct RefCtx
{
    KSurfaceContainer container;
    KElectrostaticBoundaryIntegrator integrator{KEBIFactory::MakeNumeric()};
    std::vector<KSurfacePrimitive*> created;  // element k of the caller's list
};

template<class Boundary, class S> void set_value(S* s, double value)
{
    if constexpr (std::is_same<Boundary, KDirichletBoundary>::value)
        s->SetBoundaryValue(value);
    else
        s->SetNormalBoundaryFlux(value);
}

template<class Boundary, class Shape> KSurfacePrimitive* make_planar(const double* g, double value)
{
    auto* s = new KSurface<KElectrostaticBasis, Boundary, Shape>();
    s->SetA(g[0]);
    s->SetB(g[1]);
    s->SetP0(KPosition(g[2], g[3], g[4]));
    s->SetN1(KDirection(g[5], g[6], g[7]));
    s->SetN2(KDirection(g[8], g[9], g[10]));
    set_value<Boundary>(s, value);
    return s;
}

template<class Boundary> KSurfacePrimitive* make_line(const double* g, double value)
{
    auto* s = new KSurface<KElectrostaticBasis, Boundary, KLineSegment>();
    s->SetValues(KPosition(g[0], g[1], g[2]), KPosition(g[3], g[4], g[5]), g[6]);
    set_value<Boundary>(s, value);
    return s;
}

// axisymmetric elements: conic section g = (r0, z0, r1, z1), ring g = (r, z)
template<class Boundary> KSurfacePrimitive* make_conic(const double* g, double value)
{
    auto* s = new KSurface<KElectrostaticBasis, Boundary, KConicSection>();
    s->SetValues(g[0], g[1], g[2], g[3]);
    set_value<Boundary>(s, value);
    return s;
}

template<class Boundary> KSurfacePrimitive* make_ring(const double* g, double value)
{
    auto* s = new KSurface<KElectrostaticBasis, Boundary, KRing>();
    s->SetValues(g[0], g[1]);
    set_value<Boundary>(s, value);
    return s;
}

template<class Boundary> KSurfacePrimitive* make_element(int shape, const double* g, double value)
{
    if (shape == 0)
        return make_planar<Boundary, KTriangle>(g, value);
    if (shape == 1)
        return make_planar<Boundary, KRectangle>(g, value);
    if (shape == 3)
        return make_conic<Boundary>(g, value);
    if (shape == 4)
        return make_ring<Boundary>(g, value);
    return make_line<Boundary>(g, value);
}

// ---------------------------------------------------------------- RK8 harness
using State = Kassiopeia::KSMathArray<8>;
using System = Kassiopeia::KSMathSystem<State, State, State>;

struct ExactDifferentiator : public Kassiopeia::KSMathDifferentiator<System>
{
    const KIntegratingFieldSolver<KElectrostaticBoundaryIntegrator>* solver;
    double charge, mass;
    void Differentiate(double, const State& y, State& dy) const override
    {
        const double c = katrin::KConst::C();
        const double p2 = y[5] * y[5] + y[6] * y[6] + y[7] * y[7];
        const double gamma = std::sqrt(1. + p2 / (mass * mass * c * c));
        const double inv = 1. / (mass * gamma);
        const double v[3] = {inv * y[5], inv * y[6], inv * y[7]};
        KFieldVector E = solver->ElectricField(KPosition(y[2], y[3], y[4]));
        dy[0] = 1.;
        dy[1] = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        dy[2] = v[0];
        dy[3] = v[1];
        dy[4] = v[2];
        dy[5] = charge * E[0];
        dy[6] = charge * E[1];
        dy[7] = charge * E[2];
    }
};
}  // namespace

extern "C" {

void* kemref_create(int n, const int* shape, const int* boundary, const double* geom, const double* value)
{
    auto* ctx = new RefCtx();
    for (int i = 0; i < n; i++) {
        KSurfacePrimitive* p = boundary[i] == 0 ? make_element<KDirichletBoundary>(shape[i], geom + 11 * i, value[i])
                                                : make_element<KNeumannBoundary>(shape[i], geom + 11 * i, value[i]);
        ctx->container.push_back(p);
        ctx->created.push_back(p);
    }
    return ctx;
}

void kemref_destroy(void* h)
{
    delete static_cast<RefCtx*>(h);
}

// the KSurfaceContainer of a handle (for fm_harness.cc, which builds the reference FFTM tree on it)
void* kemref_container(void* h)
{
    return &static_cast<RefCtx*>(h)->container;
}

// The container groups elements by (boundary, shape) type in first-seen order
// (KSurfaceContainer.cc:36-72), so its index i (the matrix row/column) need not be the
// caller's index k. idx[k] receives the container index of caller element k.
int kemref_container_index(void* h, int* idx)
{
    auto* ctx = static_cast<RefCtx*>(h);
    const unsigned n = ctx->container.size();
    for (unsigned i = 0; i < n; i++) {
        KSurfacePrimitive* p = ctx->container[i];
        for (unsigned k = 0; k < ctx->created.size(); k++)
            if (ctx->created[k] == p)
                idx[k] = (int) i;
    }
    return (int) n;
}

void kemref_set_sigma(void* h, const double* sigma)
{
    auto* ctx = static_cast<RefCtx*>(h);
    KBoundaryIntegralSolutionVector<KElectrostaticBoundaryIntegrator> x(ctx->container, ctx->integrator);
    for (unsigned i = 0; i < x.Dimension(); i++)
        x[i] = sigma[i];
}

void kemref_get_sigma(void* h, double* sigma)
{
    auto* ctx = static_cast<RefCtx*>(h);
    KBoundaryIntegralSolutionVector<KElectrostaticBoundaryIntegrator> x(ctx->container, ctx->integrator);
    for (unsigned i = 0; i < x.Dimension(); i++)
        sigma[i] = x(i);
}

// mode 0: ElectricFieldAndPotential, 1: Potential only, 2: ElectricField only
void kemref_field(void* h, int npts, const double* P, double* out, int mode)
{
    auto* ctx = static_cast<RefCtx*>(h);
    KIntegratingFieldSolver<KElectrostaticBoundaryIntegrator> fs(ctx->container, ctx->integrator);
    for (int i = 0; i < npts; i++) {
        KPosition X(P[3 * i], P[3 * i + 1], P[3 * i + 2]);
        double* o = out + 4 * i;
        if (mode == 1) {
            o[0] = o[1] = o[2] = 0.;
            o[3] = fs.Potential(X);
        }
        else if (mode == 2) {
            KFieldVector E = fs.ElectricField(X);
            o[0] = E[0];
            o[1] = E[1];
            o[2] = E[2];
            o[3] = 0.;
        }
        else {
            auto fp = fs.ElectricFieldAndPotential(X);
            o[0] = fp.first[0];
            o[1] = fp.first[1];
            o[2] = fp.first[2];
            o[3] = fp.second;
        }
    }
}

// normalised (sigma = 1) field and potential of one element at npts points, through the
// integrator's per-shape ElectricFieldAndPotential (the numeric policy's band dispatch)
void kemref_element_field(void* h, int elem, int npts, const double* P, double* out)
{
    auto* ctx = static_cast<RefCtx*>(h);
    KSurfacePrimitive* s = ctx->container[elem];
    auto* tri = dynamic_cast<KTriangle*>(s);
    auto* rect = dynamic_cast<KRectangle*>(s);
    auto* line = dynamic_cast<KLineSegment*>(s);
    auto* conic = dynamic_cast<KConicSection*>(s);
    auto* ring = dynamic_cast<KRing*>(s);
    for (int i = 0; i < npts; i++) {
        KPosition X(P[3 * i], P[3 * i + 1], P[3 * i + 2]);
        std::pair<KFieldVector, double> r;
        if (tri)
            r = ctx->integrator.ElectricFieldAndPotential(tri, X);
        else if (rect)
            r = ctx->integrator.ElectricFieldAndPotential(rect, X);
        else if (conic)
            r = ctx->integrator.ElectricFieldAndPotential(conic, X);
        else if (ring)
            r = ctx->integrator.ElectricFieldAndPotential(ring, X);
        else
            r = ctx->integrator.ElectricFieldAndPotential(line, X);
        out[4 * i] = r.first[0];
        out[4 * i + 1] = r.first[1];
        out[4 * i + 2] = r.first[2];
        out[4 * i + 3] = r.second;
    }
}

// rows [row0, row0 + nrows) of the boundary-integral matrix, row-major
void kemref_matrix_rows(void* h, int row0, int nrows, double* A)
{
    auto* ctx = static_cast<RefCtx*>(h);
    KBoundaryIntegralMatrix<KElectrostaticBoundaryIntegrator> M(ctx->container, ctx->integrator);
    const unsigned n = M.Dimension();
    for (int r = 0; r < nrows; r++)
        for (unsigned j = 0; j < n; j++)
            A[(size_t) r * n + j] = M(row0 + r, j);
}

void kemref_matvec(void* h, const double* x, double* y)
{
    auto* ctx = static_cast<RefCtx*>(h);
    KBoundaryIntegralMatrix<KElectrostaticBoundaryIntegrator> M(ctx->container, ctx->integrator);
    KSimpleVector<double> xv(M.Dimension()), yv(M.Dimension());
    for (unsigned i = 0; i < M.Dimension(); i++)
        xv[i] = x[i];
    M.Multiply(xv, yv);
    for (unsigned i = 0; i < M.Dimension(); i++)
        y[i] = yv[i];
}

void kemref_rhs(void* h, double* b)
{
    auto* ctx = static_cast<RefCtx*>(h);
    KBoundaryIntegralVector<KElectrostaticBoundaryIntegrator> bv(ctx->container, ctx->integrator);
    for (unsigned i = 0; i < bv.Dimension(); i++)
        b[i] = bv(i);
}

// GMRES solve (relative tolerance), sigma written into the container and into x;
// returns the iteration count; *resid = final implicit relative residual estimate
int kemref_gmres(void* h, double tol, int max_iter, double* x, double* resid)
{
    auto* ctx = static_cast<RefCtx*>(h);
    KBoundaryIntegralMatrix<KElectrostaticBoundaryIntegrator> A(ctx->container, ctx->integrator);
    KBoundaryIntegralVector<KElectrostaticBoundaryIntegrator> b(ctx->container, ctx->integrator);
    KBoundaryIntegralSolutionVector<KElectrostaticBoundaryIntegrator> xs(ctx->container, ctx->integrator);
    for (unsigned i = 0; i < xs.Dimension(); i++)
        xs[i] = 0.;
    KSimpleIterativeKrylovSolver<double, KGeneralizedMinimalResidual> S;
    S.SetTolerance(tol);
    if (max_iter > 0)
        S.SetMaximumIterations(max_iter);
    S.Solve(A, xs, b);
    for (unsigned i = 0; i < xs.Dimension(); i++)
        x[i] = xs(i);
    if (resid)
        *resid = S.ResidualNorm();
    return (int) S.GetIteration();
}

// Krylov solve of the direct system through the reference's solver factory (KBuildKrylovSolver,
// KKrylovSolverFactory.hh:83-155, as KKrylovChargeDensitySolver.cc:43-67 uses it): GMRES or
// BiCGStab, a restart every `restart` iterations (0 = never), preconditioner 0 none, 1 Jacobi
// (KJacobiPreconditioner), 2 implicit Krylov (KBuildKrylovPreconditioner: an inner GMRES on the
// same direct matrix to precon_tol, at most precon_max_iter iterations). x from zero; returns
// the iteration count, *resid = the solver's residual norm over |b|.
int kemref_krylov(void* h, int bicgstab, int precon, double tol, int max_iter, int restart, double precon_tol,
                  int precon_max_iter, double* x, double* resid)
{
    auto* ctx = static_cast<RefCtx*>(h);
    auto A = std::make_shared<KBoundaryIntegralMatrix<KElectrostaticBoundaryIntegrator>>(ctx->container,
                                                                                         ctx->integrator);
    KBoundaryIntegralVector<KElectrostaticBoundaryIntegrator> b(ctx->container, ctx->integrator);
    KBoundaryIntegralSolutionVector<KElectrostaticBoundaryIntegrator> xs(ctx->container, ctx->integrator);
    for (unsigned i = 0; i < xs.Dimension(); i++)
        xs[i] = 0.;
    KKrylovSolverConfiguration cfg;
    cfg.SetSolverName(bicgstab ? "bicgstab" : "gmres");
    cfg.SetTolerance(tol);
    cfg.SetMaxIterations((unsigned) max_iter);
    if (restart > 0)
        cfg.SetIterationsBetweenRestart((unsigned) restart);
    std::shared_ptr<const KSquareMatrix<double>> P;
    if (precon == 1)
        P = std::make_shared<KJacobiPreconditioner<double>>(*A);
    else if (precon == 2) {
        KKrylovSolverConfiguration pc;
        pc.SetSolverName("gmres");
        pc.SetTolerance(precon_tol);
        pc.SetMaxIterations((unsigned) precon_max_iter);
        P = KBuildKrylovPreconditioner<double>(pc, A);
    }
    auto solver = KBuildKrylovSolver<double>(cfg, A, P);
    solver->Solve(xs, b);
    for (unsigned i = 0; i < xs.Dimension(); i++)
        x[i] = xs(i);
    if (resid)
        *resid = solver->ResidualNorm();
    return (int) solver->GetIteration();
}

int kemref_robinhood(void* h, double tol, double* x, double* resid)
{
    auto* ctx = static_cast<RefCtx*>(h);
    KBoundaryIntegralMatrix<KElectrostaticBoundaryIntegrator> A(ctx->container, ctx->integrator);
    KBoundaryIntegralVector<KElectrostaticBoundaryIntegrator> b(ctx->container, ctx->integrator);
    KBoundaryIntegralSolutionVector<KElectrostaticBoundaryIntegrator> xs(ctx->container, ctx->integrator);
    for (unsigned i = 0; i < xs.Dimension(); i++)
        xs[i] = 0.;
    KRobinHood<double> rh;
    rh.SetTolerance(tol);
    rh.Solve(A, xs, b);
    for (unsigned i = 0; i < xs.Dimension(); i++)
        x[i] = xs(i);
    if (resid)
        *resid = rh.ResidualNorm();
    return (int) rh.GetIteration();
}

// nsteps fixed-step RK8 steps of one particle in the container's field (sigma as set);
// state[8] = (t, s, x, y, z, px, py, pz) updated in place; traj receives the state after
// every step (nsteps x 8) when non-null. Stops early (returning the steps taken) when
// |x| <= stop_radius after a step (stop_radius <= 0 disables the check).
int kemref_rk8_track(void* h, double* state, double dt, int nsteps, double charge, double mass, double stop_radius,
                     double* traj)
{
    auto* ctx = static_cast<RefCtx*>(h);
    KIntegratingFieldSolver<KElectrostaticBoundaryIntegrator> fs(ctx->container, ctx->integrator);
    ExactDifferentiator d;
    d.solver = &fs;
    d.charge = charge;
    d.mass = mass;
    Kassiopeia::KSMathRK8<System> rk8;
    State y, y1, err;
    for (int k = 0; k < 8; k++)
        y[k] = state[k];
    int s = 0;
    for (; s < nsteps; s++) {
        rk8.Integrate(0., d, y, dt, y1, err);
        y = y1;
        if (traj)
            for (int k = 0; k < 8; k++)
                traj[8 * s + k] = y[k];
        if (stop_radius > 0. && std::sqrt(y[2] * y[2] + y[3] * y[3] + y[4] * y[4]) <= stop_radius) {
            s++;
            break;
        }
    }
    for (int k = 0; k < 8; k++)
        state[k] = y[k];
    return s;
}

double kemref_constant(int which)
{
    switch (which) {
        case 0:
            return KEMConstants::OneOverFourPiEps0;
        case 1:
            return KEMConstants::Eps0;
        case 2:
            return katrin::KConst::C();
        case 3:
            return katrin::KConst::Q();
        case 4:
            return katrin::KConst::M_el_kg();
        default:
            return katrin::KConst::Pi();
    }
}
}

// Cubature nodes and weights of the reference's rules on a canonical element, for pinning
// restated rule tables: triangle P0 = 0, P1 = e_x, P2 = e_y gives node = (s, t, 0) with
// node = P0 + s (P1 - P0) + t (P2 - P0); the unit-square rectangle likewise.
// which: 0..2 triangle 7/12/33, 3..5 rectangle 7/12/33. out: npts x 3 (s, t, w).
extern "C" int kemref_rule_nodes(int which, double* out)
{
    const double data[11] = {1., 1., 0., 0., 0., 1., 0., 0., 0., 1., 0.};
    double Q[99];
    const double* w = nullptr;
    int n = 0;
    if (which == 6 || which == 7) {  // Gauss-Legendre half rules (x, w, 0) of the line segments
        const double* x = which == 6 ? gQuadx4 : gQuadx16;
        const double* wq = which == 6 ? gQuadw4 : gQuadw16;
        n = which == 6 ? 2 : 8;
        for (int k = 0; k < n; k++) {
            out[3 * k] = x[k];
            out[3 * k + 1] = wq[k];
            out[3 * k + 2] = 0.;
        }
        return n;
    }
    switch (which) {
        case 0:
            KElectrostaticCubatureTriangleIntegrator::GaussPoints_Tri7P(data, Q);
            w = gTriCub7w;
            n = 7;
            break;
        case 1:
            KElectrostaticCubatureTriangleIntegrator::GaussPoints_Tri12P(data, Q);
            w = gTriCub12w;
            n = 12;
            break;
        case 2:
            KElectrostaticCubatureTriangleIntegrator::GaussPoints_Tri33P(data, Q);
            w = gTriCub33w;
            n = 33;
            break;
        case 3:
            KElectrostaticCubatureRectangleIntegrator::GaussPoints_Rect7P(data, Q);
            w = gRectCub7w;
            n = 7;
            break;
        case 4:
            KElectrostaticCubatureRectangleIntegrator::GaussPoints_Rect12P(data, Q);
            w = gRectCub12w;
            n = 12;
            break;
        default:
            KElectrostaticCubatureRectangleIntegrator::GaussPoints_Rect33P(data, Q);
            w = gRectCub33w;
            n = 33;
            break;
    }
    for (int k = 0; k < n; k++) {
        out[3 * k] = Q[3 * k];
        out[3 * k + 1] = Q[3 * k + 1];
        out[3 * k + 2] = w[k];
    }
    return n;
}
