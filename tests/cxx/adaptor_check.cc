// Drop-in check of include/kemfield_cuda.hh against the reference's unchanged KEMField classes:
// the same KSurfaceContainer is solved on the GPU through KCUDAChargeDensitySolver, then the
// reference's CPU KIntegratingFieldSolver / KBoundaryIntegralMatrix and the CUDA adaptors are
// evaluated side by side; the reference's own GMRES driver also runs on the CUDA matrix. Last,
// the CUDA charge-density solvers run as KChargeDensitySolver subclasses against KEMField's own
// solution cache (SaveSolution / FindSolution through KEMFileInterface) in a scratch directory.
// Exit status 0 when every comparison is within tolerance.
#include "KBoundaryIntegralMatrix.hh"
#include "KBoundaryIntegralSolutionVector.hh"
#include "KBoundaryIntegralVector.hh"
#include "KElectrostaticBoundaryField.hh"
#include "KElectrostaticBoundaryIntegratorFactory.hh"
#include "KEMFileInterface.hh"
#include "KElectrostaticIntegratingFieldSolver.hh"
#include "KIntegratingElectrostaticFieldSolver.hh"
#include "KGeneralizedMinimalResidual.hh"
#include "KRobinHood.hh"
#include "KSimpleIterativeKrylovSolver.hh"
#include "KSurface.hh"
#include "KSurfaceContainer.hh"
#include "kemfield_cuda.hh"

#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <filesystem>
#include <map>
#include <vector>

using namespace KEMField;
using V = std::array<double, 3>;

static V unit(V a)
{
    const double r = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
    return {a[0] / r, a[1] / r, a[2] / r};
}

static void icosphere(int level, KSurfaceContainer& c, double R = 1., double U = 1.)
{
    const double t = (1. + std::sqrt(5.)) / 2.;
    std::vector<V> v = {{-1, t, 0}, {1, t, 0}, {-1, -t, 0}, {1, -t, 0}, {0, -1, t}, {0, 1, t},
                        {0, -1, -t}, {0, 1, -t}, {t, 0, -1}, {t, 0, 1}, {-t, 0, -1}, {-t, 0, 1}};
    for (auto& x : v)
        x = unit(x);
    std::vector<std::array<int, 3>> f = {{0, 11, 5}, {0, 5, 1}, {0, 1, 7}, {0, 7, 10}, {0, 10, 11}, {1, 5, 9}, {5, 11, 4},
                                         {11, 10, 2}, {10, 7, 6}, {7, 1, 8}, {3, 9, 4}, {3, 4, 2}, {3, 2, 6}, {3, 6, 8},
                                         {3, 8, 9}, {4, 9, 5}, {2, 4, 11}, {6, 2, 10}, {8, 6, 7}, {9, 8, 1}};
    for (int s = 0; s < level; s++) {
        std::map<std::pair<int, int>, int> mid;
        std::vector<std::array<int, 3>> g;
        auto M = [&](int a, int b) {
            auto k = std::make_pair(std::min(a, b), std::max(a, b));
            auto it = mid.find(k);
            if (it != mid.end())
                return it->second;
            v.push_back(unit({v[a][0] + v[b][0], v[a][1] + v[b][1], v[a][2] + v[b][2]}));
            return mid[k] = (int) v.size() - 1;
        };
        for (auto& q : f) {
            const int a = M(q[0], q[1]), b = M(q[1], q[2]), d = M(q[2], q[0]);
            g.push_back({q[0], a, d});
            g.push_back({q[1], b, a});
            g.push_back({q[2], d, b});
            g.push_back({a, b, d});
        }
        f = g;
    }
    for (auto& q : f) {
        auto* T = new KSurface<KElectrostaticBasis, KDirichletBoundary, KTriangle>();
        T->SetValues(KPosition(R * v[q[0]][0], R * v[q[0]][1], R * v[q[0]][2]),
                     KPosition(R * v[q[1]][0], R * v[q[1]][1], R * v[q[1]][2]),
                     KPosition(R * v[q[2]][0], R * v[q[2]][1], R * v[q[2]][2]));
        T->SetBoundaryValue(U);
        c.push_back(T);
    }
}

static double sigma_of(KSurfaceContainer& c, unsigned i)
{
    return dynamic_cast<KElectrostaticBasis*>(c[i]->GetBasis())->GetSolution();
}

// an axisymmetric model through the same adaptors: a sphere of 120 conic sections at 1 V solved
// on the device, then the reference's CPU field solver and the CUDA one on its charge densities
static int axisym_check()
{
    KSurfaceContainer c;
    const int ns = 120;
    for (int k = 0; k < ns; k++) {
        const double t0 = M_PI * k / ns, t1 = M_PI * (k + 1) / ns;
        auto* s = new KSurface<KElectrostaticBasis, KDirichletBoundary, KConicSection>();
        s->SetValues(k == 0 ? 0. : std::sin(t0), std::cos(t0), k == ns - 1 ? 0. : std::sin(t1), std::cos(t1));
        s->SetBoundaryValue(1.);
        c.push_back(s);
    }
    KCUDASurfaceContainer gpu(c);
    kemcu_solve_stats st = KCUDAChargeDensitySolver(1e-12, 300, KEMCU_SOLVE_ASSEMBLED).Solve(gpu);
    double q = 0.;
    for (unsigned i = 0; i < c.size(); i++)
        q += sigma_of(c, i) * c[i]->GetShape()->Area();
    const double cap = q / (4. * M_PI * KEMConstants::Eps0);
    KElectrostaticBoundaryIntegrator integrator = KEBIFactory::MakeNumeric();
    KIntegratingFieldSolver<KElectrostaticBoundaryIntegrator> cpu(c, integrator);
    KCUDAIntegratingFieldSolver cuda(gpu);
    gpu.WriteBasisData();
    double worst = 0.;
    for (int i = 0; i < 16; i++) {
        const double r = 1.1 + 0.1 * i, th = 0.37 * i, ph = 1.1 * i;
        KPosition P(r * std::sin(th) * std::cos(ph), r * std::sin(th) * std::sin(ph), r * std::cos(th));
        auto a = cpu.ElectricFieldAndPotential(P);
        auto b = cuda.ElectricFieldAndPotential(P);
        worst = std::max(worst, std::fabs(a.second - b.second) / std::fabs(a.second));
        worst = std::max(worst, (a.first - b.first).Magnitude() / a.first.Magnitude());
    }
    std::printf("axisymmetric sphere (%d conic sections): %d GMRES iterations, C / (4 pi eps0 R) = %.6f, field "
                "CPU vs CUDA max relative difference %.3e\n", ns, st.iterations, cap, worst);
    return !(std::fabs(cap - 1.) < 1e-4 && worst < 1e-11);
}

// KEMField's solution cache with CUDA-solved charge densities, through the reference's own
// FindSolution / SaveSolution (KChargeDensitySolver.cc:51-280):
//  1. nothing stored: solved on the device and stored;
//  2. same shape and boundary values: the stored sigma comes back bit for bit, no device solve.
//     The reference takes a stored solution of matching hashes whatever tolerance it was solved
//     to (FindByHash sets the found flag, KChargeDensitySolver.cc:108-131), so a request at a
//     tighter tolerance is answered from the cache as well;
//  3. same shape at 2 V: composed by the reference's superposition of stored solutions;
//  4. another shape (radius 1.5 m): solved on the device; sigma scales as 1/R.
static int cache_round_trip()
{
    char tmpl[] = "/tmp/kemcu_cacheXXXXXX";
    if (!mkdtemp(tmpl)) {
        std::printf("cache: no scratch directory\n");
        return 1;
    }
    const std::string dir(tmpl);
    KEMFileInterface::GetInstance()->ActiveDirectory(dir);
    KEMFileInterface::GetInstance()->ActiveFile(dir + "/kemcu_cache.kbd");
    int fail = 0;
    auto rel = [](KSurfaceContainer& a, KSurfaceContainer& b, double scale) {
        double w = 0., n = 0.;
        for (unsigned i = 0; i < a.size(); i++) {
            w = std::max(w, std::fabs(sigma_of(a, i) - scale * sigma_of(b, i)));
            n = std::max(n, std::fabs(scale * sigma_of(b, i)));
        }
        return w / n;
    };

    KSurfaceContainer c1;
    icosphere(2, c1);
    KCUDAChargeDensitySolver s1(1e-10, 200, KEMCU_SOLVE_PLAIN);
    s1.Initialize(c1);
    const bool stored = std::filesystem::exists(dir + "/kemcu_cache.kbd");
    std::printf("cache: first solve from cache %d, %d GMRES iterations, cache file written %d\n",
                (int) s1.SolutionFromCache(), s1.LastStats().iterations, (int) stored);
    fail += s1.SolutionFromCache() || s1.LastStats().iterations < 1 || !stored;

    for (double tol : {1e-8, 1e-12}) {
        KSurfaceContainer c2;
        icosphere(2, c2);
        KCUDARobinHoodChargeDensitySolver s2(tol);
        s2.Initialize(c2);
        unsigned differ = c1.size() != c2.size();
        for (unsigned i = 0; !differ && i < c1.size(); i++)
            differ += sigma_of(c1, i) != sigma_of(c2, i);
        std::printf("cache: request at %.0e from cache %d, Robin Hood checks %d, elements differing %u\n", tol,
                    (int) s2.SolutionFromCache(), s2.LastStats().iterations, differ);
        fail += !s2.SolutionFromCache() || s2.LastStats().iterations != 0 || differ != 0;
    }

    KSurfaceContainer c3;
    icosphere(2, c3, 1., 2.);
    KCUDAChargeDensitySolver s3(1e-10, 200, KEMCU_SOLVE_PLAIN);
    s3.Initialize(c3);
    const double r3 = rel(c3, c1, 2.);
    std::printf("cache: 2 V from cache %d (superposition), %d GMRES iterations, max relative difference to 2 sigma "
                "%.3e\n", (int) s3.SolutionFromCache(), s3.LastStats().iterations, r3);
    fail += !s3.SolutionFromCache() || s3.LastStats().iterations != 0 || !(r3 < 1e-12);

    KSurfaceContainer c4;
    icosphere(2, c4, 1.5);
    KCUDAChargeDensitySolver s4(1e-10, 200, KEMCU_SOLVE_PLAIN);
    s4.Initialize(c4);
    const double r4 = rel(c4, c1, 1. / 1.5);
    std::printf("cache: radius 1.5 m from cache %d, %d GMRES iterations, max relative difference to sigma / 1.5 "
                "%.3e\n", (int) s4.SolutionFromCache(), s4.LastStats().iterations, r4);
    fail += s4.SolutionFromCache() || s4.LastStats().iterations < 1 || !(r4 < 1e-8);

    std::filesystem::remove_all(dir);
    return fail;
}

// The boundary field as KEMField users build it (KElectrostaticBoundaryField.cc:29-42, 75-93),
// with the CUDA charge-density solver and the CUDA field solver plugged in where
// KKrylovChargeDensitySolver and KIntegratingElectrostaticFieldSolver go, against the
// reference's CPU field solver on the same charge densities (and on the reference's own
// mixed-precision form of the field, KEMCU_MIXED, within 1e-9). Batched calls agree with single ones.
static int boundary_field_check()
{
    char tmpl[] = "/tmp/kemcu_fieldXXXXXX";
    if (!mkdtemp(tmpl)) {
        std::printf("boundary field: no scratch directory\n");
        return 1;
    }
    const std::string dir(tmpl);
    int fail = 0;
    for (int precision : {KEMCU_FP64, KEMCU_MIXED}) {
        auto container = std::make_shared<KSurfaceContainer>();
        icosphere(2, *container);
        // a cache directory of its own per round, so that each round solves on the device
        const std::string sub = dir + (precision == KEMCU_FP64 ? "/fp64" : "/mixed");
        std::filesystem::create_directories(sub);
        KElectrostaticBoundaryField field;
        field.SetDirectory(sub);
        field.SetFile("field.kbd");
        field.SetContainer(container);
        auto cds = std::make_shared<KCUDAChargeDensitySolver>(1e-12, 300, KEMCU_SOLVE_PLAIN);
        auto fs = std::make_shared<KCUDAElectricFieldSolver>(precision);
        field.SetChargeDensitySolver(cds);
        field.SetFieldSolver(fs);
        field.Initialize();
        KIntegratingElectrostaticFieldSolver cpu;
        cpu.Initialize(*container);
        std::vector<KPosition> pts;
        double worst = 0.;
        for (int i = 0; i < 24; i++) {
            const double r = 1.02 + 0.09 * i, th = 0.61 * i + 0.2, ph = 1.7 * i;
            KPosition P(r * std::sin(th) * std::cos(ph), r * std::sin(th) * std::sin(ph), r * std::cos(th));
            pts.push_back(P);
            const auto a = cpu.ElectricFieldAndPotential(P);
            const auto b = field.ElectricFieldAndPotential(P, 0.);
            const double pb = field.Potential(P, 0.);
            const KFieldVector eb = field.ElectricField(P, 0.);
            worst = std::max(worst, std::fabs(a.second - b.second) / std::fabs(a.second));
            worst = std::max(worst, (a.first - b.first).Magnitude() / a.first.Magnitude());
            worst = std::max(worst, std::fabs(a.second - pb) / std::fabs(a.second));
            worst = std::max(worst, (a.first - eb).Magnitude() / a.first.Magnitude());
        }
        std::vector<KFieldVector> E;
        std::vector<double> phi;
        fs->ElectricFieldAndPotential(pts, E, phi);
        double wb = 0.;
        for (size_t i = 0; i < pts.size(); i++) {
            const auto b = field.ElectricFieldAndPotential(pts[i], 0.);
            wb = std::max(wb, std::fabs(phi[i] - b.second) / std::fabs(b.second));
            wb = std::max(wb, (E[i] - b.first).Magnitude() / b.first.Magnitude());
        }
        const double tol = precision == KEMCU_FP64 ? 1e-12 : 1e-9;
        std::printf("boundary field (%s, CUDA charge densities + CUDA field solver): max relative difference to the "
                    "CPU field solver %.3e, batched vs single %.3e, %d GMRES iterations\n",
                    precision == KEMCU_FP64 ? "FP64" : "MIXED", worst, wb, cds->LastStats().iterations);
        fail += !(worst < tol && wb < 1e-15 && cds->LastStats().iterations > 0);
        field.Deinitialize();
    }
    std::filesystem::remove_all(dir);
    return fail;
}

int main()
{
    KSurfaceContainer container;
    icosphere(2, container);
    KElectrostaticBoundaryIntegrator integrator = KEBIFactory::MakeNumeric();
    int failures = 0;
    try {
        KCUDASurfaceContainer gpu(container);
        kemcu_solve_stats st = KCUDAChargeDensitySolver(1e-12, 200, KEMCU_SOLVE_PLAIN).Solve(gpu);
        std::printf("gpu solve: %d iterations, relative residual %.3e\n", st.iterations, st.rel_residual);

        // field: reference CPU direct sum vs the CUDA field solver on the same sigma
        KIntegratingFieldSolver<KElectrostaticBoundaryIntegrator> cpu(container, integrator);
        KCUDAIntegratingFieldSolver cuda(gpu);
        double worst = 0.;
        for (int i = 0; i < 24; i++) {
            const double r = 1.05 + 0.08 * i, th = 0.7 * i, ph = 1.3 * i;
            KPosition P(r * std::sin(th) * std::cos(ph), r * std::sin(th) * std::sin(ph), r * std::cos(th));
            auto a = cpu.ElectricFieldAndPotential(P);
            auto b = cuda.ElectricFieldAndPotential(P);
            worst = std::max(worst, std::fabs(a.second - b.second) / std::fabs(a.second));
            worst = std::max(worst, (a.first - b.first).Magnitude() / a.first.Magnitude());
        }
        std::printf("field: max relative difference CPU vs CUDA %.3e\n", worst);
        failures += !(worst < 1e-12);

        // matrix entries and the virtual Multiply
        KBoundaryIntegralMatrix<KElectrostaticBoundaryIntegrator> Aref(container, integrator);
        KCUDABoundaryIntegralMatrix Acuda(gpu);
        double wm = 0.;
        for (unsigned k = 0; k < 40; k++) {
            const unsigned i = (k * 37) % Aref.Dimension(), j = (k * 91 + 5) % Aref.Dimension();
            wm = std::max(wm, std::fabs(Aref(i, j) - Acuda(i, j)) / std::fabs(Aref(i, i)));
        }
        std::printf("matrix entries: max relative difference %.3e\n", wm);
        failures += !(wm < 1e-12);
        KSimpleVector<double> x(Aref.Dimension()), y1(Aref.Dimension()), y2(Aref.Dimension());
        for (unsigned i = 0; i < x.Dimension(); i++)
            x[i] = std::sin(0.1 * i);
        Aref.Multiply(x, y1);
        Acuda.Multiply(x, y2);
        double wy = 0., ny = 0.;
        for (unsigned i = 0; i < x.Dimension(); i++) {
            wy = std::max(wy, std::fabs(y1(i) - y2(i)));
            ny = std::max(ny, std::fabs(y1(i)));
        }
        std::printf("Multiply: max relative difference %.3e\n", wy / ny);
        failures += !(wy / ny < 1e-12);

        // the reference's own GMRES driver on the CUDA matrix (drop-in behind KMatrix::Multiply)
        KBoundaryIntegralVector<KElectrostaticBoundaryIntegrator> b(container, integrator);
        KSimpleVector<double> xs(Aref.Dimension());
        for (unsigned i = 0; i < xs.Dimension(); i++)
            xs[i] = 0.;
        KSimpleIterativeKrylovSolver<double, KGeneralizedMinimalResidual> S;
        S.SetTolerance(1e-10);
        S.Solve(Acuda, xs, b);
        std::printf("reference GMRES on the CUDA matrix: %u iterations, estimate %.3e\n", S.GetIteration(),
                    S.ResidualNorm());
        failures += !(S.ResidualNorm() < 1e-10);

        // Robin Hood: the reference's KRobinHood on its own matrix vs the CUDA solver, both from 0
        KSimpleVector<double> xr(Aref.Dimension());
        for (unsigned i = 0; i < xr.Dimension(); i++)
            xr[i] = 0.;
        KRobinHood<double> rh;
        rh.SetTolerance(1e-8);
        rh.Solve(Aref, xr, b);
        for (unsigned i = 0; i < container.size(); i++)
            dynamic_cast<KElectrostaticBasis*>(container[i]->GetBasis())->GetSolution() = 0.;
        kemcu_rh_stats rs = KCUDARobinHoodChargeDensitySolver(1e-8).Solve(gpu);
        double wr = 0., nr = 0.;
        for (unsigned i = 0; i < container.size(); i++) {
            const double g = dynamic_cast<KElectrostaticBasis*>(container[i]->GetBasis())->GetSolution();
            wr = std::max(wr, std::fabs(g - xr(i)));
            nr = std::max(nr, std::fabs(xr(i)));
        }
        std::printf("Robin Hood: reference %u checks, CUDA %d checks (%lld corrections), max relative difference "
                    "%.3e\n", rh.GetIteration(), rs.iterations, rs.subiterations, wr / nr);
        failures += !(wr / nr < 1e-6 && std::abs((int) rh.GetIteration() - rs.iterations) <= 1);

        failures += cache_round_trip();
        failures += axisym_check();
        failures += boundary_field_check();
    }
    catch (std::exception& e) {
        std::printf("exception: %s\n", e.what());
        return 2;
    }
    std::printf("%s\n", failures ? "FAILED" : "OK");
    return failures ? 1 : 0;
}
