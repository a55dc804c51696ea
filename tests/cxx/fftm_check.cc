// Check of include/kemfield_cuda_fftm.hh against the reference's unchanged fast-multipole classes,
// on the 1,280-triangle sphere at 1 V with the same tree parameters and the same explicit world
// cube (degree 8, divisions 2, zeromask 1, depth 3):
//   matrix the products of the matrices KFastMultipoleMatrixGenerator and
//          KCUDAFastMultipoleMatrixGenerator build, on the same vector;
//   solve  the reference's KKrylovChargeDensitySolver (GMRES to 1e-10) with its own generator and
//          with KCUDAFastMultipoleMatrixGenerator, and the all-device KCUDAChargeDensitySolver in
//          KEMCU_SOLVE_FFTM, each judged by its residual under the reference's FFTM matrix (the
//          reference GMRES's least-squares step by SVD leaves its iterate well above its residual
//          estimate, so the two reference-GMRES residuals are compared with each other, the
//          device GMRES with the tolerance);
//   krylov the reference's krylov_bem_solver (KKrylovChargeDensitySolverOld with
//          KFMElectrostaticFastMultipoleBoundaryValueSolver) with gmres + implicit_krylov (degree-1
//          preconditioner tree, inner tolerance 0.01, 30 iterations, restarts every 250) and with
//          bicgstab + jacobi, against KCUDAChargeDensitySolver with the same settings, each to 1e-8:
//          residuals under the reference's FFTM matrix and the densities;
//   field  the reference's KElectricFastMultipoleFieldSolver and KCUDAFastMultipoleFieldSolver
//          (both KElectricFieldSolvers) on those densities, at points inside the world cube.
// Exit status 0 when every comparison is within tolerance.
#include "KElectricFastMultipoleFieldSolver.hh"
#include "KEMFileInterface.hh"
#include "KElectrostaticBoundaryField.hh"
#include "KFastMultipoleMatrixGenerator.hh"
#include "KKrylovChargeDensitySolver.hh"
#include "KKrylovChargeDensitySolverOld.hh"
#include "KFMElectrostaticFastMultipoleBoundaryValueSolverConfiguration.hh"
#include "KSimpleVector.hh"
#include "KSurface.hh"
#include "KSurfaceContainer.hh"
#include "kemfield_cuda_fftm.hh"

#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <filesystem>
#include <map>
#include <memory>
#include <random>
#include <vector>

using namespace KEMField;
using V = std::array<double, 3>;

static V unit(V a)
{
    const double r = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
    return {a[0] / r, a[1] / r, a[2] / r};
}

static std::vector<std::array<V, 3>> icosphere(int level)
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
    std::vector<std::array<V, 3>> tri;
    for (auto& q : f)
        tri.push_back({v[q[0]], v[q[1]], v[q[2]]});
    return tri;
}

static std::shared_ptr<KSurfaceContainer> sphere()
{
    auto c = std::make_shared<KSurfaceContainer>();
    for (auto& t : icosphere(3)) {
        auto* T = new KSurface<KElectrostaticBasis, KDirichletBoundary, KTriangle>();
        T->SetValues(KPosition(t[0][0], t[0][1], t[0][2]), KPosition(t[1][0], t[1][1], t[1][2]),
                     KPosition(t[2][0], t[2][1], t[2][2]));
        T->SetBoundaryValue(1.);
        c->push_back(T);
    }
    return c;
}

static std::vector<double> densities(KSurfaceContainer& c)
{
    std::vector<double> s;
    for (unsigned i = 0; i < c.size(); i++)
        s.push_back(dynamic_cast<KElectrostaticBasis*>(c[i]->GetBasis())->GetSolution());
    return s;
}

static double max_rel(const std::vector<double>& a, const std::vector<double>& b)
{
    double e = 0., m = 0.;
    for (size_t i = 0; i < a.size(); i++) {
        e = std::max(e, std::fabs(a[i] - b[i]));
        m = std::max(m, std::fabs(b[i]));
    }
    return e / m;
}

int main()
{
    char tmpl[] = "/tmp/kemcu_fftmXXXXXX";
    if (!mkdtemp(tmpl))
        return 2;
    const std::string dir(tmpl);
    int fail = 0;
    try {
        // one world cube for every tree: centred near the sphere, side 2.4 m
        const KPosition wc(0.002, -0.003, 0.001);
        const double wl = 2.4;
        auto configure = [&](auto& g) {
            g.SetDegree(8);
            g.SetTopLevelDivisions(2);
            g.SetDivisions(2);
            g.SetZeromask(1);
            g.SetMaximumTreeDepth(3);
            g.SetInsertionRatio(4. / 3.);
            g.SetUseRegionEstimation(false);
            g.SetWorldCenter(wc);
            g.SetWorldLength(wl);
            g.SetVerbosity(0);
        };
        // solve: the reference Krylov solver on the reference FFTM matrix and on the CUDA one
        std::vector<double> s_ref, s_cuda, s_dev;
        for (int pass = 0; pass < 2; pass++) {
            auto container = sphere();
            KEMFileInterface::GetInstance()->ActiveDirectory(dir + "/solve" + std::to_string(pass));
            std::filesystem::create_directories(dir + "/solve" + std::to_string(pass));
            KKrylovChargeDensitySolver krylov;
            krylov.SetTolerance(1e-10);
            krylov.SetMaxIterations(200);
            krylov.SetSolverName("gmres");
            krylov.SetUseDisplay(false);
            if (pass == 0) {
                auto g = std::make_shared<KFastMultipoleMatrixGenerator>();
                configure(*g);
                krylov.SetMatrixGenerator(g);
            }
            else {
                auto g = std::make_shared<KCUDAFastMultipoleMatrixGenerator>();
                configure(*g);
                krylov.SetMatrixGenerator(g);
            }
            krylov.Initialize(*container);
            (pass == 0 ? s_ref : s_cuda) = densities(*container);
        }
        {
            auto container = sphere();
            KCUDASurfaceContainer gpu(*container);
            KCUDAChargeDensitySolver dev(1e-10, 200, KEMCU_SOLVE_FFTM);
            kemcu_fftm_params q;
            kemcu_fftm_default_params(&q);
            q.degree = 8;
            q.maximum_tree_depth = 3;
            q.world_center[0] = wc[0];
            q.world_center[1] = wc[1];
            q.world_center[2] = wc[2];
            q.world_length = wl;
            dev.SetFastMultipoleParameters(q);
            dev.Solve(gpu);
            s_dev = densities(*container);
        }
        // krylov_bem_solver: the reference's boundary-value solver and the device with its settings
        const char* kry[2][2] = {{"gmres", "implicit_krylov"}, {"bicgstab", "jacobi"}};
        std::vector<double> s_old[2], s_devk[2];
        for (int c = 0; c < 2; c++) {
            {
                auto container = sphere();
                const std::string sub = dir + "/old" + std::to_string(c);
                std::filesystem::create_directories(sub);
                KEMFileInterface::GetInstance()->ActiveDirectory(sub);
                KKrylovChargeDensitySolverOld old;
                auto* cfg = old.GetSolverConfig();
                cfg->SetSolverName(kry[c][0]);
                cfg->SetPreconditionerName(kry[c][1]);
                cfg->SetSolverTolerance(1e-8);
                cfg->SetMaxSolverIterations(200);
                cfg->SetIterationsBetweenRestart(250);
                cfg->SetPreconditionerTolerance(0.01);
                cfg->SetMaxPreconditionerIterations(30);
                cfg->SetPreconditionerDegree(1);
                auto* prm = new KFMElectrostaticParameters();
                prm->strategy = KFMSubdivisionStrategy::Aggressive;
                prm->degree = 8;
                prm->top_level_divisions = 2;
                prm->divisions = 2;
                prm->zeromask = 1;
                prm->maximum_tree_depth = 3;
                prm->insertion_ratio = 4. / 3.;
                prm->use_region_estimation = false;
                prm->world_center_x = wc[0];
                prm->world_center_y = wc[1];
                prm->world_center_z = wc[2];
                prm->world_length = wl;
                prm->use_caching = false;
                prm->verbosity = 0;
                cfg->SetFFTMParams(prm);  // owned by the configuration
                old.Initialize(*container);
                s_old[c] = densities(*container);
            }
            {
                auto container = sphere();
                KCUDASurfaceContainer gpu(*container);
                KCUDAChargeDensitySolver dev(1e-8, 200, KEMCU_SOLVE_FFTM);
                kemcu_fftm_params q;
                kemcu_fftm_default_params(&q);
                q.degree = 8;
                q.maximum_tree_depth = 3;
                q.world_center[0] = wc[0];
                q.world_center[1] = wc[1];
                q.world_center[2] = wc[2];
                q.world_length = wl;
                dev.SetFastMultipoleParameters(q);
                dev.SetSolverName(kry[c][0]);
                dev.SetPreconditionerName(kry[c][1]);
                dev.SetIterationsBetweenRestart(250);
                dev.SetPreconditionerTolerance(0.01);
                dev.SetMaxPreconditionerIterations(30);
                dev.SetPreconditionerDegree(1);
                dev.Solve(gpu);
                s_devk[c] = densities(*container);
            }
        }
        // the reference's FFTM matrix and the CUDA one on the same vector, and the residuals of the
        // three solutions under the reference's matrix
        {
            auto container = sphere();
            KEMFileInterface::GetInstance()->ActiveDirectory(dir + "/matrix");
            std::filesystem::create_directories(dir + "/matrix");
            KFastMultipoleMatrixGenerator gr;
            configure(gr);
            KCUDAFastMultipoleMatrixGenerator gc;
            configure(gc);
            auto Ar = gr.Build(*container);
            auto Ac = gc.Build(*container);
            const unsigned n = container->size();
            KSimpleVector<double> x(n), yr(n), yc(n);
            for (unsigned i = 0; i < n; i++)
                x[i] = s_ref[i];
            Ar->Multiply(x, yr);
            Ac->Multiply(x, yc);
            std::vector<double> a(n), b(n);
            for (unsigned i = 0; i < n; i++) {
                a[i] = yc[i];
                b[i] = yr[i];
            }
            const double d_mat = max_rel(a, b);
            auto residual = [&](const std::vector<double>& s) {
                KSimpleVector<double> xs(n), ys(n);
                for (unsigned i = 0; i < n; i++)
                    xs[i] = s[i];
                Ar->Multiply(xs, ys);
                double r2 = 0., b2 = 0.;
                for (unsigned i = 0; i < n; i++) {
                    r2 += (ys[i] - 1.) * (ys[i] - 1.);
                    b2 += 1.;
                }
                return std::sqrt(r2 / b2);
            };
            const double r_ref = residual(s_ref), r_cuda = residual(s_cuda), r_dev = residual(s_dev);
            std::printf("FFTM matrix: CUDA vs reference product, max error / max value %.3e\n", d_mat);
            std::printf("FFTM solve, relative residual under the reference's FFTM matrix: reference Krylov + reference "
                        "matrix %.3e, reference Krylov + CUDA matrix %.3e, device GMRES (KEMCU_SOLVE_FFTM) %.3e\n",
                        r_ref, r_cuda, r_dev);
            fail += !(d_mat < 1e-11);
            fail += !(r_cuda <= 10. * r_ref + 1e-9 && r_dev <= 1e-9);
            for (int c = 0; c < 2; c++) {
                const double ro = residual(s_old[c]), rd = residual(s_devk[c]), ds = max_rel(s_devk[c], s_old[c]);
                std::printf("krylov_bem_solver %s + %s: relative residual under the reference's FFTM matrix, reference "
                            "%.3e, device %.3e; densities max difference / max value %.3e\n",
                            kry[c][0], kry[c][1], ro, rd, ds);
                // both solve the same system to 1e-8 (condition number ~30): the densities agree to
                // a few 1e-7 at most
                fail += !(ro <= 1e-8 && rd <= 1e-8 && ds <= 1e-6);
            }
        }

        // field: the reference FFTM field solver and the CUDA one, each a KElectricFieldSolver
        // initialised on a container holding the reference-solved densities
        std::vector<double> P;
        std::mt19937_64 rng(5);
        std::uniform_real_distribution<double> u(-1.0, 1.0);
        while (P.size() < 3 * 200) {
            const double x = u(rng), y = u(rng), z = u(rng), r = std::sqrt(x * x + y * y + z * z);
            if (std::fabs(r - 1.) > 0.08)
                P.insert(P.end(), {x, y, z});
        }
        std::vector<std::array<double, 4>> out[2];
        for (int pass = 0; pass < 2; pass++) {
            auto container = sphere();
            for (unsigned i = 0; i < container->size(); i++)
                dynamic_cast<KElectrostaticBasis*>((*container)[i]->GetBasis())->GetSolution() = s_ref[i];
            std::shared_ptr<KElectricFieldSolver> fs;
            if (pass == 0) {
                auto f = std::make_shared<KElectricFastMultipoleFieldSolver>();
                KFMElectrostaticParameters* p = f->GetParameters();
                p->degree = 8;
                p->top_level_divisions = 2;
                p->divisions = 2;
                p->zeromask = 1;
                p->maximum_tree_depth = 3;
                p->insertion_ratio = 4. / 3.;
                p->use_region_estimation = false;
                p->world_center_x = wc[0];
                p->world_center_y = wc[1];
                p->world_center_z = wc[2];
                p->world_length = wl;
                p->verbosity = 0;
                fs = f;
            }
            else {
                auto f = std::make_shared<KCUDAFastMultipoleFieldSolver>();
                KFMElectrostaticParameters* p = f->GetParameters();
                p->degree = 8;
                p->maximum_tree_depth = 3;
                p->use_region_estimation = false;
                p->world_center_x = wc[0];
                p->world_center_y = wc[1];
                p->world_center_z = wc[2];
                p->world_length = wl;
                fs = f;
            }
            KEMFileInterface::GetInstance()->ActiveDirectory(dir);
            fs->Initialize(*container);
            for (size_t i = 0; i < P.size() / 3; i++) {
                const KPosition x(P[3 * i], P[3 * i + 1], P[3 * i + 2]);
                const auto ep = fs->ElectricFieldAndPotential(x);
                out[pass].push_back({ep.first[0], ep.first[1], ep.first[2], ep.second});
            }
        }
        double eE = 0., mE = 0., ep = 0., mp = 0.;
        for (size_t i = 0; i < out[0].size(); i++) {
            for (int c = 0; c < 3; c++) {
                eE = std::max(eE, std::fabs(out[1][i][c] - out[0][i][c]));
                mE = std::max(mE, std::fabs(out[0][i][c]));
            }
            ep = std::max(ep, std::fabs(out[1][i][3] - out[0][i][3]));
            mp = std::max(mp, std::fabs(out[0][i][3]));
        }
        std::printf("FFTM field: KCUDAFastMultipoleFieldSolver vs KElectricFastMultipoleFieldSolver, max error / max "
                    "value: field %.3e, potential %.3e\n", eE / mE, ep / mp);
        fail += !(eE / mE < 1e-10 && ep / mp < 1e-12);
    }
    catch (std::exception& e) {
        std::printf("exception: %s\n", e.what());
        fail++;
    }
    std::filesystem::remove_all(dir);
    std::printf("%s\n", fail ? "FAILED" : "OK");
    return fail ? 1 : 0;
}
