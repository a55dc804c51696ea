// Check of include/kemfield_cuda_bindings.hh: a KEMField-style XML configuration is parsed by the
// reference's own Kommon tokenizer and element processor (KXMLTokenizer, KElementProcessor,
// KComplexElement); the CUDA elements are registered by RegisterKEMCUBuilders under a test field
// element that collects solvers exactly as KElectrostaticBoundaryFieldBuilder::AddElement does
// (KEMField/Source/Bindings/Fields/Electric/include/KElectrostaticBoundaryFieldBuilder.hh), then
// drives a KElectrostaticBoundaryField with them on a 320-triangle sphere at 1 V; the field is
// compared with the reference's KIntegratingElectrostaticFieldSolver on the same charge
// densities (a fourth field solves on the fast multipole operator and evaluates with the CUDA FFTM
// field solver; a fifth and a sixth take krylov_bem_solver's solver and preconditioner choices and
// its fftm_multiplication / preconditioner_electrostatic_parameters children, built by the
// reference's KFMElectrostaticParametersBuilder), and the parsed settings with the XML. Exit status 0 when everything agrees. With the
// argument --parse-only the check stops after the settings (no device needed).
#include "KComplexElement.hh"
#include "KElectrostaticBoundaryField.hh"
#include "KElementProcessor.hh"
#include "KEMFileInterface.hh"
#include "KIntegratingElectrostaticFieldSolver.hh"
#include "KSurface.hh"
#include "KTextFile.h"
#include "KXMLTokenizer.hh"
#include "kemfield_cuda_bindings.hh"

#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <filesystem>
#include <fstream>
#include <map>
#include <memory>
#include <vector>

using namespace KEMField;
using V = std::array<double, 3>;

static V unit(V a)
{
    const double r = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
    return {a[0] / r, a[1] / r, a[2] / r};
}

static void icosphere2(KSurfaceContainer& c)
{
    const double t = (1. + std::sqrt(5.)) / 2.;
    std::vector<V> v = {{-1, t, 0}, {1, t, 0}, {-1, -t, 0}, {1, -t, 0}, {0, -1, t}, {0, 1, t},
                        {0, -1, -t}, {0, 1, -t}, {t, 0, -1}, {t, 0, 1}, {-t, 0, -1}, {-t, 0, 1}};
    for (auto& x : v)
        x = unit(x);
    std::vector<std::array<int, 3>> f = {{0, 11, 5}, {0, 5, 1}, {0, 1, 7}, {0, 7, 10}, {0, 10, 11}, {1, 5, 9}, {5, 11, 4},
                                         {11, 10, 2}, {10, 7, 6}, {7, 1, 8}, {3, 9, 4}, {3, 4, 2}, {3, 2, 6}, {3, 6, 8},
                                         {3, 8, 9}, {4, 9, 5}, {2, 4, 11}, {6, 2, 10}, {8, 6, 7}, {9, 8, 1}};
    for (int s = 0; s < 2; s++) {
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
        T->SetValues(KPosition(v[q[0]][0], v[q[0]][1], v[q[0]][2]), KPosition(v[q[1]][0], v[q[1]][1], v[q[1]][2]),
                     KPosition(v[q[2]][0], v[q[2]][1], v[q[2]][2]));
        T->SetBoundaryValue(1.);
        c.push_back(T);
    }
}

// the test's field element: holds what KElectrostaticBoundaryFieldBuilder::AddElement would set
struct TestField
{
    std::shared_ptr<KChargeDensitySolver> cds;
    std::shared_ptr<KElectricFieldSolver> fs;
};
static std::vector<TestField> gFields;
static std::string gScratch;

namespace katrin
{
using TestFieldBuilder = KComplexElement<TestField>;
template<> inline bool TestFieldBuilder::AddElement(KContainer* anElement)
{
    if (anElement->Is<KEMField::KChargeDensitySolver>()) {
        anElement->ReleaseTo(fObject->cds);
        return true;
    }
    if (anElement->Is<KEMField::KElectricFieldSolver>()) {
        anElement->ReleaseTo(fObject->fs);
        return true;
    }
    return false;
}
template<> inline bool TestFieldBuilder::End()
{
    gFields.push_back(*fObject);
    return true;
}
STATICINT sTestField = KElementProcessor::ComplexElement<TestField>("test_electrostatic_field");
STATICINT sKEMCU = RegisterKEMCUBuilders<TestFieldBuilder>();
}  // namespace katrin

static const char* kXML = R"(
<test_electrostatic_field>
    <cuda_krylov_charge_density_solver tolerance="1.e-11" max_iterations="250" mode="assembled"/>
    <integrating_field_solver use_cuda="true" cuda_precision="mixed"/>
</test_electrostatic_field>
<test_electrostatic_field>
    <cuda_robin_hood_charge_density_solver tolerance="1.e-9" check_sub_interval="64" cache_matrix_elements="true"/>
    <cuda_field_solver precision="fp64"/>
</test_electrostatic_field>
<test_electrostatic_field>
    <cuda_krylov_charge_density_solver tolerance="1.e-12" mode="plain"/>
    <integrating_field_solver integrator="numeric" use_opencl="false" use_cuda="false"/>
</test_electrostatic_field>
<test_electrostatic_field>
    <cuda_krylov_charge_density_solver tolerance="1.e-10" mode="fftm" expansion_degree="10" top_level_divisions="2"
        tree_level_divisions="2" neighbor_order="1" maximum_tree_depth="3" use_region_size_estimation="true"
        verbosity="0"/>
    <cuda_fast_multipole_field_solver expansion_degree="10" top_level_divisions="2" tree_level_divisions="2"
        neighbor_order="2" maximum_tree_depth="3" region_expansion_factor="1.1" use_region_size_estimation="false"
        world_cube_center_x="0.001" world_cube_center_y="-0.002" world_cube_center_z="0.0" world_cube_length="6.4"
        insertion_ratio="1.3333333333333333" verbosity="0"/>
</test_electrostatic_field>
<test_electrostatic_field>
    <cuda_krylov_bem_solver solver_name="gmres" preconditioner="implicit_krylov" tolerance="1e-8"
        preconditioner_tolerance="0.01" max_iterations="500" max_preconditioner_iterations="30"
        iterations_between_restarts="250" preconditioner_degree="1" intermediate_save_interval="1"
        use_display="true" show_plot="false" use_timer="true">
        <fftm_multiplication verbosity="0" strategy="aggressive" top_level_divisions="2" tree_level_divisions="2"
            expansion_degree="8" neighbor_order="1" maximum_tree_depth="3" use_region_size_estimation="true"
            region_expansion_factor="1.1" insertion_ratio="1.3333333333333333"/>
    </cuda_krylov_bem_solver>
    <cuda_field_solver precision="fp64"/>
</test_electrostatic_field>
<test_electrostatic_field>
    <cuda_krylov_charge_density_solver solver_name="bicgstab" preconditioner="independent_implicit_krylov"
        tolerance="1e-8" preconditioner_tolerance="0.05" max_preconditioner_iterations="20">
        <fftm_multiplication top_level_divisions="2" tree_level_divisions="2" expansion_degree="8" neighbor_order="1"
            maximum_tree_depth="3" use_region_size_estimation="true" region_expansion_factor="1.1"/>
        <preconditioner_electrostatic_parameters top_level_divisions="2" tree_level_divisions="2"
            expansion_degree="2" neighbor_order="1" maximum_tree_depth="2" use_region_size_estimation="true"
            region_expansion_factor="1.1"/>
    </cuda_krylov_charge_density_solver>
    <cuda_field_solver precision="fp64"/>
</test_electrostatic_field>
)";

// the boundary field with the parsed solvers, against the reference CPU field solver
static double field_difference(TestField& f, const std::string& sub)
{
    auto container = std::make_shared<KSurfaceContainer>();
    icosphere2(*container);
    std::filesystem::create_directories(sub);
    KElectrostaticBoundaryField field;
    field.SetDirectory(sub);
    field.SetFile("field.kbd");
    field.SetContainer(container);
    field.SetChargeDensitySolver(f.cds);
    field.SetFieldSolver(f.fs);
    field.Initialize();
    KIntegratingElectrostaticFieldSolver cpu;
    cpu.Initialize(*container);
    double worst = 0.;
    for (int i = 0; i < 16; i++) {
        const double r = 1.05 + 0.12 * i, th = 0.47 * i + 0.1, ph = 1.9 * i;
        KPosition P(r * std::sin(th) * std::cos(ph), r * std::sin(th) * std::sin(ph), r * std::cos(th));
        const auto a = cpu.ElectricFieldAndPotential(P);
        const auto b = field.ElectricFieldAndPotential(P, 0.);
        worst = std::max(worst, std::fabs(a.second - b.second) / std::fabs(a.second));
        worst = std::max(worst, (a.first - b.first).Magnitude() / a.first.Magnitude());
    }
    field.Deinitialize();
    return worst;
}

int main(int argc, char** argv)
{
    const bool parse_only = argc > 1 && std::string(argv[1]) == "--parse-only";
    char tmpl[] = "/tmp/kemcu_xmlXXXXXX";
    if (!mkdtemp(tmpl))
        return 2;
    gScratch = tmpl;
    const std::string xml = gScratch + "/kemcu.xml";
    {
        std::ofstream out(xml);
        out << kXML;
    }
    int fail = 0;
    try {
        katrin::KXMLTokenizer tokenizer;
        katrin::KElementProcessor processor;
        processor.InsertAfter(&tokenizer);
        katrin::KTextFile file;
        file.AddToNames(xml);
        tokenizer.ProcessFile(&file);
        std::printf("parsed %zu field elements\n", gFields.size());
        if (gFields.size() != 6)
            return 1;
        // settings as written in the XML
        auto* k0 = dynamic_cast<KCUDAChargeDensitySolver*>(gFields[0].cds.get());
        auto* f0 = dynamic_cast<KIntegratingElectrostaticFieldSolverCUDA*>(gFields[0].fs.get());
        auto* r1 = dynamic_cast<KCUDARobinHoodChargeDensitySolver*>(gFields[1].cds.get());
        auto* f1 = dynamic_cast<KCUDAElectricFieldSolver*>(gFields[1].fs.get());
        auto* k2 = dynamic_cast<KCUDAChargeDensitySolver*>(gFields[2].cds.get());
        auto* f2 = dynamic_cast<KIntegratingElectrostaticFieldSolverCUDA*>(gFields[2].fs.get());
        auto* k3 = dynamic_cast<KCUDAChargeDensitySolver*>(gFields[3].cds.get());
        auto* f3 = dynamic_cast<KCUDAFastMultipoleFieldSolver*>(gFields[3].fs.get());
        const bool settings = k0 && f0 && r1 && f1 && k2 && f2 && k0->GetTolerance() == 1e-11 &&
                              k0->GetMaxIterations() == 250 && k0->GetMode() == KEMCU_SOLVE_ASSEMBLED &&
                              f0->UsesCUDA() && f0->CUDASolver().GetPrecision() == KEMCU_MIXED &&
                              r1->GetTolerance() == 1e-9 && r1->GetCheckSubInterval() == 64 &&
                              r1->MatrixElementsCached() && f1->GetPrecision() == KEMCU_FP64 &&
                              k2->GetMode() == KEMCU_SOLVE_PLAIN && !f2->UsesCUDA() && k3 && f3 &&
                              k3->GetMode() == KEMCU_SOLVE_FFTM && k3->GetFastMultipoleParameters().degree == 10 &&
                              k3->GetFastMultipoleParameters().maximum_tree_depth == 3 &&
                              f3->GetParameters()->degree == 10 && f3->GetParameters()->zeromask == 2 &&
                              f3->GetParameters()->maximum_tree_depth == 3 &&
                              !f3->GetParameters()->use_region_estimation &&
                              f3->GetParameters()->world_length == 6.4 &&
                              f3->GetParameters()->world_center_y == -0.002;
        auto* k4 = dynamic_cast<KCUDAChargeDensitySolver*>(gFields[4].cds.get());
        auto* k5 = dynamic_cast<KCUDAChargeDensitySolver*>(gFields[5].cds.get());
        const bool krylov = k4 && k5 && k4->GetMode() == KEMCU_SOLVE_FFTM && k4->GetSolver() == KEMCU_KRYLOV_GMRES &&
                            k4->GetPreconditioner() == KEMCU_PRECON_IMPLICIT_KRYLOV && !k4->IndependentPreconditioner() &&
                            k4->GetIterationsBetweenRestart() == 250 && k4->GetPreconditionerTolerance() == 0.01 &&
                            k4->GetMaxPreconditionerIterations() == 30 && k4->GetPreconditionerDegree() == 1 &&
                            k4->GetMaxIterations() == 500 && k4->GetFastMultipoleParameters().degree == 8 &&
                            k5->GetMode() == KEMCU_SOLVE_FFTM && k5->GetSolver() == KEMCU_KRYLOV_BICGSTAB &&
                            k5->IndependentPreconditioner() && k5->GetMaxPreconditionerIterations() == 20 &&
                            k5->GetPreconditionerFastMultipoleParameters().degree == 2 &&
                            k5->GetPreconditionerFastMultipoleParameters().maximum_tree_depth == 2;
        std::printf("Krylov solver and preconditioner settings from the XML: %s\n", krylov ? "as written" : "WRONG");
        fail += !krylov;
        std::printf("settings from the XML: %s\n", settings ? "as written" : "WRONG");
        fail += !settings;
        if (settings && !parse_only) {
            const double d0 = field_difference(gFields[0], gScratch + "/0");
            const double d1 = field_difference(gFields[1], gScratch + "/1");
            const double d2 = field_difference(gFields[2], gScratch + "/2");
            const double d3 = field_difference(gFields[3], gScratch + "/3");
            std::printf("field vs the reference CPU solver: GMRES assembled + CUDA mixed %.3e, Robin Hood + CUDA "
                        "FP64 %.3e, GMRES plain + reference field solver (use_cuda=false) %.3e, FFTM GMRES + CUDA "
                        "FFTM field %.3e\n", d0, d1, d2, d3);
            // the densities differ by the solve tolerance (1e-11 GMRES, 1e-9 Robin Hood): the CPU
            // comparison solver sees the same densities, so only the field arithmetic differs; the
            // FFTM field differs by its truncation error (degree 10, neighbour order 2)
            fail += !(d0 < 1e-9 && d1 < 1e-12 && d2 < 1e-14 && d3 < 1e-5);
            if (krylov) {
                // fast multipole solves (degree 8) with the preconditioned solvers, the field of their
                // densities by the direct sum: the densities carry the operator's truncation error
                const double d4 = field_difference(gFields[4], gScratch + "/4");
                const double d5 = field_difference(gFields[5], gScratch + "/5");
                std::printf("field vs the reference CPU solver: FFTM GMRES + implicit Krylov (degree 1) %.3e, "
                            "FFTM BiCGStab + independent implicit Krylov %.3e\n", d4, d5);
                fail += !(d4 < 1e-5 && d5 < 1e-5);
            }
        }
    }
    catch (std::exception& e) {
        std::printf("exception: %s\n", e.what());
        fail++;
    }
    std::filesystem::remove_all(gScratch);
    std::printf("%s\n", fail ? "FAILED" : "OK");
    return fail ? 1 : 0;
}
