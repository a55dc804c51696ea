// Check of include/kassiopeia_cuda.hh (the KSRoot-level batch driver) against the reference: the
// 1,280-triangle sphere at -2 kV is solved and evaluated on the GPU through KEMField's own
// KElectrostaticBoundaryField (KCUDAChargeDensitySolver + KCUDAElectricFieldSolver); electrons
// made by Kassiopeia's KSParticleFactory are tracked as one batch by KSCUDATrackBatch, which fills
// Kassiopeia KSTrack objects; every track is compared with the reference's own KSMathRK8 driven
// by the reference field solver on the same charge densities (oracle/ref_harness.cc,
// kemref_rk8_track: after every step a track ends when |x| <= the electrode radius), step count,
// final state, continuous time / length / energy / momentum change and terminator.
// Exit status 0 when every comparison is within tolerance.
#include "KElectrostaticBoundaryField.hh"
#include "KEMFileInterface.hh"
#include "KSParticleFactory.h"
#include "KSurface.hh"
#include "KSurfaceContainer.hh"
#include "kassiopeia_cuda.hh"
#include "kemfield_cuda.hh"

#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <filesystem>
#include <map>
#include <memory>
#include <vector>

extern "C" {
void* kemref_create(int n, const int* shape, const int* boundary, const double* geom, const double* value);
void kemref_destroy(void* h);
void kemref_set_sigma(void* h, const double* sigma);
int kemref_rk8_track(void* h, double* state, double dt, int nsteps, double charge, double mass, double stop_radius,
                     double* traj);
}

using namespace KEMField;
using V = std::array<double, 3>;

static V unit(V a)
{
    const double r = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
    return {a[0] / r, a[1] / r, a[2] / r};
}

// icosphere of radius 1 m: 20 * 4^level triangles, outward orientation
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

int main()
{
    const double U = -2000., dt = 1e-11, R = 1.;
    const int max_steps = 600;
    char tmpl[] = "/tmp/kemcu_batchXXXXXX";
    if (!mkdtemp(tmpl))
        return 2;
    const std::string dir(tmpl);
    int fail = 0;
    try {
        // the boundary field with the CUDA solvers, as a Kassiopeia KSElectricKEMField holds it
        auto container = std::make_shared<KSurfaceContainer>();
        const auto tri = icosphere(3);
        std::vector<int> shape, boundary;
        std::vector<double> geom, value;
        for (auto& t : tri) {
            auto* T = new KSurface<KElectrostaticBasis, KDirichletBoundary, KTriangle>();
            T->SetValues(KPosition(t[0][0], t[0][1], t[0][2]), KPosition(t[1][0], t[1][1], t[1][2]),
                         KPosition(t[2][0], t[2][1], t[2][2]));
            T->SetBoundaryValue(U);
            container->push_back(T);
        }
        KElectrostaticBoundaryField field;
        field.SetDirectory(dir);
        field.SetFile("batch.kbd");
        field.SetContainer(container);
        field.SetChargeDensitySolver(std::make_shared<KCUDAChargeDensitySolver>(1e-12, 300, KEMCU_SOLVE_PLAIN));
        auto fs = std::make_shared<KCUDAElectricFieldSolver>(KEMCU_FP64);
        field.SetFieldSolver(fs);
        field.Initialize();
        // the reference's field solver on the same container and charge densities
        std::vector<double> sigma;
        for (unsigned i = 0; i < container->size(); i++) {
            auto* s = (*container)[i];
            auto* t = dynamic_cast<KTriangle*>(s->GetShape());
            shape.push_back(0);
            boundary.push_back(0);
            geom.insert(geom.end(), {t->GetA(), t->GetB(), t->GetP0()[0], t->GetP0()[1], t->GetP0()[2], t->GetN1()[0],
                                     t->GetN1()[1], t->GetN1()[2], t->GetN2()[0], t->GetN2()[1], t->GetN2()[2]});
            value.push_back(U);
            sigma.push_back(dynamic_cast<KElectrostaticBasis*>(s->GetBasis())->GetSolution());
        }
        void* ref = kemref_create((int) container->size(), shape.data(), boundary.data(), geom.data(), value.data());
        kemref_set_sigma(ref, sigma.data());

        // electrons: some aimed at the sphere (they hit it against the -2 kV field), some passing
        // it, some flying away
        std::vector<Kassiopeia::KSParticle> batch;
        const double E[8] = {1500., 9000., 18000., 2500., 12000., 4000., 15000., 6000.};
        for (int k = 0; k < 8; k++) {
            Kassiopeia::KSParticle* p = Kassiopeia::KSParticleFactory::GetInstance().Create(11);
            const double r0 = 1.05 + 0.03 * k, th = 0.3 + 0.35 * k, ph = 0.9 * k;
            const V x = {r0 * std::sin(th) * std::cos(ph), r0 * std::sin(th) * std::sin(ph), r0 * std::cos(th)};
            V d = {-x[0], -x[1], -x[2]};  // inward
            if (k % 4 == 2)
                d = {x[0], x[1], x[2]};  // outward
            if (k % 4 == 3)
                d = {-x[1], x[0], 0.3};  // tangential
            d = unit(d);
            p->SetTime(0.);
            p->SetLength(0.);
            p->SetPosition(x[0], x[1], x[2]);
            p->SetMomentum(d[0], d[1], d[2]);
            p->SetKineticEnergy_eV(E[k]);
            batch.push_back(*p);
            delete p;
        }
        Kassiopeia::KSCUDATrackBatch driver(fs->DeviceContainer()->Context());
        driver.SetTime(dt);
        driver.SetMaxSteps(max_steps);
        driver.SetElectrode(R);
        driver.SetStepsPerLaunch(64);
        std::vector<Kassiopeia::KSTrack> tracks = driver.Execute(batch, 100);
        std::printf("batch: %zu tracks, %lld steps in %d launches, %d hit, %d at the step limit\n", tracks.size(),
                    driver.LastStats().steps, driver.LastLaunches(), driver.LastStats().hit,
                    driver.LastStats().max_steps);
        int hits = 0, limits = 0;
        double wx = 0., wp = 0., wt = 0., we = 0., wdp = 0.;
        for (size_t k = 0; k < batch.size(); k++) {
            const Kassiopeia::KSParticle& p0 = batch[k];
            double y[8] = {p0.GetTime(), p0.GetLength()};
            for (int c = 0; c < 3; c++) {
                y[2 + c] = p0.GetPosition()[c];
                y[5 + c] = p0.GetMomentum()[c];
            }
            std::vector<double> traj(8 * max_steps);
            const int n = kemref_rk8_track(ref, y, dt, max_steps, p0.GetCharge(), p0.GetMass(), R, traj.data());
            double dp = 0.;
            for (int s = 0; s < n; s++) {
                const double* a = s == 0 ? nullptr : &traj[8 * (s - 1)];
                const double* b = &traj[8 * s];
                double q = 0.;
                for (int c = 5; c < 8; c++) {
                    const double before = a ? a[c] : p0.GetMomentum()[c - 5];
                    q += (b[c] - before) * (b[c] - before);
                }
                dp += std::sqrt(q);
            }
            Kassiopeia::KSParticle pr = p0;
            pr.SetTime(y[0]);
            pr.SetLength(y[1]);
            pr.SetPosition(y[2], y[3], y[4]);
            pr.SetMomentum(y[5], y[6], y[7]);
            const Kassiopeia::KSTrack& t = tracks[k];
            const Kassiopeia::KSParticle& pf = t.GetFinalParticle();
            const bool hit = std::sqrt(y[2] * y[2] + y[3] * y[3] + y[4] * y[4]) <= R;
            hits += hit;
            limits += n == max_steps && !hit;
            const std::string want = hit ? "electrode_hit" : "term_max_steps";
            if ((int) t.GetTotalSteps() != n || t.GetTerminatorName() != want || t.GetTrackId() != 100 + (int) k ||
                pf.IsActive()) {
                std::printf("track %zu: steps %u vs %d, terminator <%s> vs <%s>\n", k, t.GetTotalSteps(), n,
                            t.GetTerminatorName().c_str(), want.c_str());
                fail++;
            }
            wx = std::max(wx, (pf.GetPosition() - pr.GetPosition()).Magnitude() / pr.GetPosition().Magnitude());
            wp = std::max(wp, (pf.GetMomentum() - pr.GetMomentum()).Magnitude() / pr.GetMomentum().Magnitude());
            wt = std::max(wt, std::fabs(t.GetContinuousTime() - (y[0] - p0.GetTime())) / (y[0] - p0.GetTime()));
            wt = std::max(wt, std::fabs(t.GetContinuousLength() - (y[1] - p0.GetLength())) / (y[1] - p0.GetLength()));
            we = std::max(we, std::fabs(t.GetContinuousEnergyChange() -
                                        (pr.GetKineticEnergy_eV() - p0.GetKineticEnergy_eV())));
            wdp = std::max(wdp, std::fabs(t.GetContinuousMomentumChange() - dp) / dp);
        }
        std::printf("batch vs reference RK8: %d hits, %d at the step limit; max relative difference position %.3e, "
                    "momentum %.3e, time/length %.3e, momentum change %.3e; energy change %.3e eV\n",
                    hits, limits, wx, wp, wt, wdp, we);
        fail += !(wx < 1e-11 && wp < 1e-11 && wt < 1e-12 && wdp < 1e-9 && we < 1e-6);
        fail += !(hits >= 2 && limits >= 2);
        kemref_destroy(ref);
        field.Deinitialize();
    }
    catch (std::exception& e) {
        std::printf("exception: %s\n", e.what());
        fail++;
    }
    std::filesystem::remove_all(dir);
    std::printf("%s\n", fail ? "FAILED" : "OK");
    return fail ? 1 : 0;
}
