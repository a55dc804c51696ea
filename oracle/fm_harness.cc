// C-ABI harness over the reference's fast-multipole (FFTM) code, test infrastructure only: it
// is compiled with the reference's own FastMultipole sources into oracle/_ref/libkemref_fm.so
// and is the checker of the device multipole kernels, never part of the product.
//
//   kemref_fm_moments    KFMElectrostaticMultipoleCalculatorAnalytic / ...Numeric::ConstructExpansion
//                        (KFMElectrostaticMultipoleCalculatorAnalytic.cc:169-224): the moments of a
//                        wire (2 vertices), triangle (3) or rectangle (4) of unit total charge about
//                        an origin, (degree + 1)^2 complex values in the index n(n+1)+m
//   kemref_fm_l2p        KFMElectrostaticLocalCoefficientFieldCalculator::Potential / ElectricField
//                        (KFMElectrostaticLocalCoefficientFieldCalculator.cc:163-360)
//   kemref_fm_response   the M2M, M2L and L2L response functions of the 3D Laplace kernel
//                        (KFMResponseKernel_3DLaplaceM2M.cc, ...M2L.cc, ...L2L.cc) between two
//                        origins, as a dense (degree+1)^2 x (degree+1)^2 complex matrix
//   kemref_fm_matvec     y = A x with the reference's fast-multipole matrix (KFastMultipoleMatrixGenerator,
//                        KFastMultipoleMatrixGenerator.cc:23-41: dense far part from the local
//                        expansions, sparse near part by the numeric integrator), x and y in
//                        container order
//   kemref_fm_bvs        the reference's fast-multipole charge-density solve
//                        (KFMElectrostaticFastMultipoleBoundaryValueSolver.cc:189-233, the solver of
//                        krylov_bem_solver): gmres or bicgstab, preconditioner none, jacobi,
//                        implicit_krylov or independent_implicit_krylov, restarts
//   kemref_fm_field      the whole reference FFTM field solver on a container made by
//                        ref_harness.cc's kemref_create: KFMElectrostaticTreeConstructor with the
//                        single-threaded field mapper, then KFMElectrostaticFastMultipoleFieldSolver
//                        (KFMElectrostaticFastMultipoleFieldSolver.cc:47-163) at each point
#include "KFMElectrostaticFastMultipoleBoundaryValueSolver.hh"
#include "KFMElectrostaticFastMultipoleFieldSolver.hh"
#include "KFMElectrostaticLocalCoefficientFieldCalculator.hh"
#include "KFMElectrostaticLocalCoefficientSet.hh"
#include "KFMElectrostaticMultipoleCalculatorAnalytic.hh"
#include "KFMElectrostaticMultipoleCalculatorNumeric.hh"
#include "KFMElectrostaticParameters.hh"
#include "KFMElectrostaticTree.hh"
#include "KFMElectrostaticTreeConstructor.hh"
#include "KFMResponseKernel_3DLaplaceL2L.hh"
#include "KFMResponseKernel_3DLaplaceM2L.hh"
#include "KFMResponseKernel_3DLaplaceM2M.hh"
#include "KEMFileInterface.hh"
#include "KFastMultipoleMatrixGenerator.hh"
#include "KSimpleVector.hh"
#include "KSurfaceContainer.hh"

#include <complex>
#include <cstdlib>
#include <filesystem>
#include <string>
#include <vector>

using namespace KEMField;

extern "C" void* kemref_container(void* h);
extern "C" void kemref_set_sigma(void* h, const double* sigma);
extern "C" void kemref_get_sigma(void* h, double* sigma);

extern "C" {

int kemref_fm_moments(int nverts, const double* verts, const double* origin, int degree, int numeric, double* out)
{
    if (nverts < 2 || nverts > 4 || degree < 0)
        return -1;
    KFMPointCloud<3> cloud;
    for (int v = 0; v < nverts; v++)
        cloud.AddPoint(KFMPoint<3>(verts + 3 * v));
    KFMScalarMultipoleExpansion moments;
    moments.SetDegree(degree);
    double o[3] = {origin[0], origin[1], origin[2]};
    bool ok;
    if (numeric) {
        KFMElectrostaticMultipoleCalculatorNumeric calc;
        calc.SetDegree(degree);
        ok = calc.ConstructExpansion(o, &cloud, &moments);
    }
    else {
        KFMElectrostaticMultipoleCalculatorAnalytic calc;
        calc.SetDegree(degree);
        ok = calc.ConstructExpansion(o, &cloud, &moments);
    }
    if (!ok)
        return -2;
    std::vector<std::complex<double>> m;
    moments.GetMoments(&m);
    const int size = (degree + 1) * (degree + 1);
    if ((int) m.size() < size)
        return -3;
    for (int i = 0; i < size; i++) {
        out[2 * i] = m[i].real();
        out[2 * i + 1] = m[i].imag();
    }
    return 0;
}

// coeff: (degree+1)(degree+2)/2 complex local coefficients (m >= 0, index n(n+1)/2 + m), as the
// reference's local coefficient set stores them; out4 = (Ex, Ey, Ez, phi) per point
int kemref_fm_l2p(int degree, const double* origin, double expansion_radius, const double* coeff, int n,
                  const double* P, double* out4)
{
    const int terms = (degree + 1) * (degree + 2) / 2;
    std::vector<double> re(terms), im(terms);
    for (int i = 0; i < terms; i++) {
        re[i] = coeff[2 * i];
        im[i] = coeff[2 * i + 1];
    }
    KFMElectrostaticLocalCoefficientSet set;
    set.SetDegree(degree);
    set.SetRealMoments(&re);
    set.SetImaginaryMoments(&im);
    KFMElectrostaticLocalCoefficientFieldCalculator calc;
    calc.SetDegree(degree);
    calc.SetExpansionOrigin(origin);
    calc.SetExpansionRadius(expansion_radius);
    calc.SetLocalCoefficients(&set);
    for (int i = 0; i < n; i++) {
        double f[3];
        calc.ElectricField(P + 3 * i, f);
        out4[4 * i] = f[0];
        out4[4 * i + 1] = f[1];
        out4[4 * i + 2] = f[2];
        out4[4 * i + 3] = calc.Potential(P + 3 * i);
    }
    return 0;
}

// kind 0 M2M, 1 M2L, 2 L2L; out[(t * S + s) * 2 + {0, 1}] = response(s -> t), S = (degree+1)^2,
// zero where the pair is not physical
int kemref_fm_response(int kind, int degree, const double* source_origin, const double* target_origin, double* out)
{
    KFMResponseKernel_3DLaplaceM2M m2m;
    KFMResponseKernel_3DLaplaceM2L m2l;
    KFMResponseKernel_3DLaplaceL2L l2l;
    KFMKernelExpansion<3>* k = kind == 0 ? (KFMKernelExpansion<3>*) &m2m
                               : kind == 1 ? (KFMKernelExpansion<3>*) &m2l
                                           : (KFMKernelExpansion<3>*) &l2l;
    if (kind < 0 || kind > 2)
        return -1;
    k->SetSourceOrigin(source_origin);
    k->SetTargetOrigin(target_origin);
    const int S = (degree + 1) * (degree + 1);
    for (int t = 0; t < S; t++)
        for (int s = 0; s < S; s++) {
            std::complex<double> v(0., 0.);
            if (k->IsPhysical(s, t))
                v = k->GetResponseFunction(s, t);
            out[2 * (t * S + s)] = v.real();
            out[2 * (t * S + s) + 1] = v.imag();
        }
    return 0;
}

// ip, dp as kemref_fm_field; the matrix's tree estimates its world cube the same way. The sparse
// part keeps its blocks in files of KEMFileInterface's active directory: a temporary directory,
// removed afterwards.
int kemref_fm_matvec(void* h, const int* ip, const double* dp, const double* x, double* y)
{
    auto* container = static_cast<KSurfaceContainer*>(kemref_container(h));
    char tmpl[] = "/tmp/kemref_fmXXXXXX";
    if (!mkdtemp(tmpl))
        return -1;
    const std::string dir(tmpl);
    KEMFileInterface::GetInstance()->ActiveDirectory(dir);
    KFastMultipoleMatrixGenerator gen;
    gen.SetStrategy(KFMSubdivisionStrategy::Aggressive);
    gen.SetDegree(ip[0]);
    gen.SetTopLevelDivisions(ip[1]);
    gen.SetDivisions(ip[2]);
    gen.SetZeromask(ip[3]);
    gen.SetMaximumTreeDepth(ip[4]);
    gen.SetInsertionRatio(dp[0]);
    gen.SetRegionExpansionFactor(dp[1]);
    gen.SetUseRegionEstimation(true);
    gen.SetUseCaching(false);
    gen.SetVerbosity(0);
    auto A = gen.Build(*container);
    const unsigned n = container->size();
    KSimpleVector<double> xv(n), yv(n);
    for (unsigned i = 0; i < n; i++)
        xv[i] = x[i];
    A->Multiply(xv, yv);
    for (unsigned i = 0; i < n; i++)
        y[i] = yv[i];
    A.reset();
    std::filesystem::remove_all(dir);
    return 0;
}

// ip = {degree, top_level_divisions, divisions, zeromask, maximum_tree_depth},
// dp = {insertion_ratio, region_expansion_factor}; world4 receives the root cube's centre and
// side length. The charge densities are those last set by kemref_set_sigma.
int kemref_fm_field(void* h, const int* ip, const double* dp, int n, const double* P, double* out4, double* world4)
{
    auto* container = static_cast<KSurfaceContainer*>(kemref_container(h));
    KFMElectrostaticParameters params;
    params.strategy = KFMSubdivisionStrategy::Aggressive;
    params.degree = ip[0];
    params.top_level_divisions = ip[1];
    params.divisions = ip[2];
    params.zeromask = ip[3];
    params.maximum_tree_depth = ip[4];
    params.insertion_ratio = dp[0];
    params.region_expansion_factor = dp[1];
    params.use_region_estimation = true;
    params.use_caching = false;
    params.verbosity = 0;
    KFMElectrostaticTree tree;
    tree.SetParameters(params);
    KFMElectrostaticTreeConstructor<KFMElectrostaticFieldMapper_SingleThread> constructor;
    constructor.ConstructTree(*container, tree);
    KFMCube<3>* cube = KFMObjectRetriever<KFMElectrostaticNodeObjects, KFMCube<3>>::GetNodeObject(tree.GetRootNode());
    const KFMPoint<3> c = cube->GetCenter();
    world4[0] = c[0];
    world4[1] = c[1];
    world4[2] = c[2];
    world4[3] = cube->GetLength();
    KFMElectrostaticFastMultipoleFieldSolver solver(*container, tree);
    for (int i = 0; i < n; i++) {
        const KPosition p(P[3 * i], P[3 * i + 1], P[3 * i + 2]);
        const KFieldVector E = solver.ElectricField(p);
        out4[4 * i] = E[0];
        out4[4 * i + 1] = E[1];
        out4[4 * i + 2] = E[2];
        out4[4 * i + 3] = solver.Potential(p);
    }
    return 0;
}
}

namespace
{
KFMElectrostaticParameters fm_params(const int* ip, const double* dp)
{
    KFMElectrostaticParameters params;
    params.strategy = KFMSubdivisionStrategy::Aggressive;
    params.degree = ip[0];
    params.top_level_divisions = ip[1];
    params.divisions = ip[2];
    params.zeromask = ip[3];
    params.maximum_tree_depth = ip[4];
    params.insertion_ratio = dp[0];
    params.region_expansion_factor = dp[1];
    params.use_region_estimation = true;
    params.use_caching = false;
    params.verbosity = 0;
    return params;
}
}  // namespace

extern "C" {
// ip, dp: the solver tree's parameters as kemref_fm_matvec; solver "gmres" or "bicgstab";
// precon "none", "jacobi", "implicit_krylov" (degree precon_degree on the solver's tree) or
// "independent_implicit_krylov" (the tree of pip, pdp); restart 0 = never. x receives the
// solution in container order (from zero charge densities), *resid the solver's residual norm
// over |b|.
int kemref_fm_bvs(void* h, const int* ip, const double* dp, const char* solver, const char* precon, double tol,
                  int max_iter, int restart, double precon_tol, int precon_max_iter, int precon_degree,
                  const int* pip, const double* pdp, double* x, double* resid)
{
    auto* container = static_cast<KSurfaceContainer*>(kemref_container(h));
    const std::vector<double> zeros(container->size(), 0.);
    kemref_set_sigma(h, zeros.data());
    char tmpl[] = "/tmp/kemref_fmXXXXXX";
    if (!mkdtemp(tmpl))
        return -1;
    const std::string dir(tmpl);
    KEMFileInterface::GetInstance()->ActiveDirectory(dir);
    {
        KFMElectrostaticFastMultipoleBoundaryValueSolver bvs;
        bvs.SetSolverElectrostaticParameters(fm_params(ip, dp));
        if (pip && pdp)
            bvs.SetPreconditionerElectrostaticParameters(fm_params(pip, pdp));
        bvs.SetSolverType(solver);
        bvs.SetPreconditionerType(precon);
        bvs.SetTolerance(tol);
        bvs.SetMaxIterations((unsigned) max_iter);
        if (restart > 0)
            bvs.SetRestart((unsigned) restart);
        bvs.SetPreconditionerTolerance(precon_tol);
        bvs.SetMaxPreconditionerIterations((unsigned) precon_max_iter);
        bvs.SetPreconditionerDegree((unsigned) precon_degree);
        bvs.Solve(*container);
        if (resid)
            *resid = bvs.GetResidualNorm();
    }
    kemref_get_sigma(h, x);
    std::filesystem::remove_all(dir);
    return 0;
}
}
