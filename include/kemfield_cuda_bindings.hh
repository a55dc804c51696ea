// kemfield_cuda_bindings.hh -- XML bindings of the B200 backend for KEMField's configuration files,
// in the reference's binding framework (Kommon's KComplexElement builders, the way
// KEMField/Source/Bindings/FieldSolvers/Electric/src/KIntegratingElectrostaticFieldSolverBuilder.cc
// and .../ChargeDensitySolvers/Electric/src/KRobinHoodChargeDensitySolverBuilder.cc bind theirs).
//
// Elements (children of the electrostatic boundary field element, registered by
// RegisterKEMCUBuilders<KElectrostaticBoundaryFieldBuilder>() in one source file of the build):
//
//   <cuda_krylov_charge_density_solver tolerance max_iterations mode device solver_name preconditioner
//           iterations_between_restarts preconditioner_tolerance max_preconditioner_iterations
//           preconditioner_degree>
//       KCUDAChargeDensitySolver: the Krylov solve on the device; mode = plain | mixed | assembled |
//       assembled_fp64 | fp32 | fftm (the fast multipole operator); solver_name = gmres | bicgstab,
//       preconditioner = none | jacobi | implicit_krylov | independent_implicit_krylov, with the
//       meaning of the reference's krylov_bem_solver (KKrylovChargeDensitySolverOldBuilder.hh);
//       children <fftm_multiplication .../> (the solver's tree; selects mode fftm) and
//       <preconditioner_electrostatic_parameters .../> (the independent preconditioner's tree),
//       built by the reference's KFMElectrostaticParametersBuilder
//   <cuda_krylov_bem_solver .../>
//       the same element under the name of the reference's krylov_bem_solver
//   <cuda_robin_hood_charge_density_solver tolerance check_sub_interval cache_matrix_elements device/>
//       KCUDARobinHoodChargeDensitySolver (attribute names of the reference's robin_hood element)
//   <cuda_field_solver precision device/>
//       KCUDAElectricFieldSolver; precision = fp64 | mixed | fp32
//   <cuda_fast_multipole_field_solver expansion_degree top_level_divisions tree_level_divisions
//           neighbor_order maximum_tree_depth region_expansion_factor use_region_size_estimation
//           world_cube_center_x/y/z world_cube_length insertion_ratio use_caching verbosity device
//           near_field_analytic/>
//       KCUDAFastMultipoleFieldSolver, with the attribute names of the reference's
//       fast_multipole_field_solver element (KElectricFastMultipoleFieldSolverBuilder.hh:16-75);
//       cuda_krylov_charge_density_solver takes the same tree attributes for mode="fftm"
//   <integrating_field_solver integrator use_opencl use_cuda cuda_precision cuda_device/>
//       KIntegratingElectrostaticFieldSolverCUDA: the reference's integrating field solver with a
//       use_cuda switch beside use_opencl (KIntegratingElectrostaticFieldSolverBuilder.cc:20-21);
//       registered under the reference's element name, it takes the place of the reference's
//       builder of that name
//
// Header-only; include after the reference's KEMField and Kommon headers.
#pragma once

#include "KComplexElement.hh"
#include "KElectrostaticBoundaryIntegratorAttributeProcessor.hh"
#include "KFMElectrostaticParametersBuilder.hh"
#include "KIntegratingElectrostaticFieldSolver.hh"
#include "kemfield_cuda.hh"
#include "kemfield_cuda_fftm.hh"

#include <memory>
#include <string>

namespace KEMField
{

// KIntegratingElectrostaticFieldSolver (KIntegratingElectrostaticFieldSolver.hh:22-57) with a
// UseCUDA switch beside UseOpenCL: with the switch set, Initialize builds a KCUDAElectricFieldSolver
// and every field call runs on the GPU; otherwise the reference's own solver runs, configured by
// the integrator policy and UseOpenCL as before.
class KIntegratingElectrostaticFieldSolverCUDA : public KElectricFieldSolver
{
  public:
    void SetIntegratorPolicy(KEBIPolicy& policy)
    {
        fReference.SetIntegratorPolicy(policy);
    }
    void UseOpenCL(bool choice)
    {
        fReference.UseOpenCL(choice);
    }
    void UseCUDA(bool choice)
    {
        fUseCUDA = choice;
    }
    bool UsesCUDA() const
    {
        return fUseCUDA;
    }
    void SetCUDAPrecision(int precision)
    {
        fCUDA.SetPrecision(precision);
    }
    void SetCUDADevice(int device)
    {
        fCUDA.SetDevice(device);
    }
    // the device solver (valid when UseCUDA is set), e.g. for KSCUDATrackBatch
    KCUDAElectricFieldSolver& CUDASolver()
    {
        return fCUDA;
    }

  private:
    void InitializeCore(KSurfaceContainer& container) override
    {
        if (fUseCUDA)
            fCUDA.Initialize(container);
        else
            fReference.Initialize(container);
    }
    void DeinitializeCore() override
    {
        if (fUseCUDA)
            fCUDA.Deinitialize();
        else
            fReference.Deinitialize();
    }
    double PotentialCore(const KPosition& P) const override
    {
        return fUseCUDA ? fCUDA.Potential(P) : fReference.Potential(P);
    }
    KFieldVector ElectricFieldCore(const KPosition& P) const override
    {
        return fUseCUDA ? fCUDA.ElectricField(P) : fReference.ElectricField(P);
    }
    std::pair<KFieldVector, double> ElectricFieldAndPotentialCore(const KPosition& P) const override
    {
        return fUseCUDA ? fCUDA.ElectricFieldAndPotential(P) : fReference.ElectricFieldAndPotential(P);
    }

    bool fUseCUDA = false;
    KIntegratingElectrostaticFieldSolver fReference;
    KCUDAElectricFieldSolver fCUDA;
};

// "fp64" | "mixed" | "fp32" -> kemcu_precision; -1 for anything else
inline int KEMCUPrecisionFromName(const std::string& name)
{
    if (name == "fp64")
        return KEMCU_FP64;
    if (name == "mixed")
        return KEMCU_MIXED;
    if (name == "fp32")
        return KEMCU_FP32;
    return -1;
}

}  // namespace KEMField

namespace katrin
{

using KCUDAChargeDensitySolverBuilder = KComplexElement<KEMField::KCUDAChargeDensitySolver>;
using KCUDARobinHoodChargeDensitySolverBuilder = KComplexElement<KEMField::KCUDARobinHoodChargeDensitySolver>;
using KCUDAElectricFieldSolverBuilder = KComplexElement<KEMField::KCUDAElectricFieldSolver>;
using KIntegratingElectrostaticFieldSolverCUDABuilder = KComplexElement<KEMField::KIntegratingElectrostaticFieldSolverCUDA>;
using KCUDAFastMultipoleFieldSolverBuilder = KComplexElement<KEMField::KCUDAFastMultipoleFieldSolver>;

// the tree attributes of the reference's fast_multipole_field_solver element
// (KElectricFastMultipoleFieldSolverBuilder.hh:16-75) onto KFMElectrostaticParameters
inline bool KEMCUFastMultipoleAttribute(KEMField::KFMElectrostaticParameters& p, KContainer* c)
{
    const std::string& n = c->GetName();
    if (n == "top_level_divisions")
        p.top_level_divisions = c->AsReference<unsigned int>();
    else if (n == "tree_level_divisions")
        p.divisions = c->AsReference<unsigned int>();
    else if (n == "expansion_degree")
        p.degree = c->AsReference<unsigned int>();
    else if (n == "neighbor_order")
        p.zeromask = c->AsReference<unsigned int>();
    else if (n == "maximum_tree_depth")
        p.maximum_tree_depth = c->AsReference<unsigned int>();
    else if (n == "region_expansion_factor")
        p.region_expansion_factor = c->AsReference<double>();
    else if (n == "use_region_size_estimation")
        p.use_region_estimation = c->AsReference<bool>();
    else if (n == "world_cube_center_x")
        p.world_center_x = c->AsReference<double>();
    else if (n == "world_cube_center_y")
        p.world_center_y = c->AsReference<double>();
    else if (n == "world_cube_center_z")
        p.world_center_z = c->AsReference<double>();
    else if (n == "world_cube_length")
        p.world_length = c->AsReference<double>();
    else if (n == "insertion_ratio")
        p.insertion_ratio = c->AsReference<double>();
    else if (n == "use_caching")
        p.use_caching = c->AsReference<bool>();
    else if (n == "verbosity")
        p.verbosity = c->AsReference<unsigned int>();
    else
        return false;
    return true;
}

// the same attributes onto the device solver's FFTM tree (mode="fftm")
inline bool KEMCUFastMultipoleAttribute(KEMField::KCUDAChargeDensitySolver& s, KContainer* c)
{
    kemcu_fftm_params& q = s.FastMultipoleParameters();
    const std::string& n = c->GetName();
    if (n == "top_level_divisions")
        q.top_level_divisions = (int) c->AsReference<unsigned int>();
    else if (n == "tree_level_divisions")
        q.divisions = (int) c->AsReference<unsigned int>();
    else if (n == "expansion_degree")
        q.degree = (int) c->AsReference<unsigned int>();
    else if (n == "neighbor_order")
        q.zeromask = (int) c->AsReference<unsigned int>();
    else if (n == "maximum_tree_depth")
        q.maximum_tree_depth = (int) c->AsReference<unsigned int>();
    else if (n == "region_expansion_factor")
        q.region_expansion_factor = c->AsReference<double>();
    else if (n == "insertion_ratio")
        q.insertion_ratio = c->AsReference<double>();
    else if (n == "use_region_size_estimation")
        s.SetFastMultipoleRegionEstimation(c->AsReference<bool>());
    else if (n == "world_cube_center_x")
        q.world_center[0] = c->AsReference<double>();
    else if (n == "world_cube_center_y")
        q.world_center[1] = c->AsReference<double>();
    else if (n == "world_cube_center_z")
        q.world_center[2] = c->AsReference<double>();
    else if (n == "world_cube_length")
        s.SetFastMultipoleWorldLength(c->AsReference<double>());
    else if (n == "use_caching" || n == "verbosity") {
        // accepted for the reference's attribute set; the device tree is rebuilt per solve and
        // reports nothing
    }
    else
        return false;
    return true;
}

template<> inline bool KCUDAChargeDensitySolverBuilder::AddAttribute(KContainer* aContainer)
{
    const std::string& name = aContainer->GetName();
    if (name == "tolerance")
        aContainer->CopyTo(fObject, &KEMField::KCUDAChargeDensitySolver::SetTolerance);
    else if (name == "max_iterations")
        aContainer->CopyTo(fObject, &KEMField::KCUDAChargeDensitySolver::SetMaxIterations);
    else if (name == "device")
        aContainer->CopyTo(fObject, &KEMField::KCUDAChargeDensitySolver::SetDevice);
    else if (name == "mode" || name == "solver_name" || name == "preconditioner") {
        try {
            if (name == "mode")
                fObject->SetModeName(aContainer->AsString());
            else if (name == "solver_name")
                fObject->SetSolverName(aContainer->AsString());
            else
                fObject->SetPreconditionerName(aContainer->AsString());
        }
        catch (KEMField::KEMSimpleException& e) {
            BINDINGMSG(eWarning) << e.what() << eom;
            return false;
        }
    }
    else if (name == "iterations_between_restarts")
        aContainer->CopyTo(fObject, &KEMField::KCUDAChargeDensitySolver::SetIterationsBetweenRestart);
    else if (name == "preconditioner_tolerance")
        aContainer->CopyTo(fObject, &KEMField::KCUDAChargeDensitySolver::SetPreconditionerTolerance);
    else if (name == "max_preconditioner_iterations")
        aContainer->CopyTo(fObject, &KEMField::KCUDAChargeDensitySolver::SetMaxPreconditionerIterations);
    else if (name == "preconditioner_degree")
        aContainer->CopyTo(fObject, &KEMField::KCUDAChargeDensitySolver::SetPreconditionerDegree);
    else if (name == "intermediate_save_interval" || name == "use_display" || name == "show_plot" ||
             name == "use_timer" || name == "time_limit_in_seconds" || name == "time_check_interval") {
        // accepted for the reference's attribute set: the device solve keeps no checkpoints and
        // shows no display (the iteration callback of kemcu_set_iteration_callback serves both)
    }
    else
        return KEMCUFastMultipoleAttribute(*fObject, aContainer);
    return true;
}

// the children of the reference's krylov_bem_solver (KKrylovChargeDensitySolverOldBuilder.hh:
// AddElement): fftm_multiplication, the solver's tree (it selects mode fftm), and
// preconditioner_electrostatic_parameters, the tree of independent_implicit_krylov
template<> inline bool KCUDAChargeDensitySolverBuilder::AddElement(KContainer* anElement)
{
    if (!anElement->Is<KEMField::KFMElectrostaticParameters>())
        return false;
    const kemcu_fftm_params q =
        KEMField::KCUDAFastMultipoleParameters(anElement->AsReference<KEMField::KFMElectrostaticParameters>());
    if (anElement->GetName() == "fftm_multiplication") {
        fObject->SetFastMultipoleParameters(q);
        fObject->SetMode(KEMCU_SOLVE_FFTM);
        return true;
    }
    if (anElement->GetName() == "preconditioner_electrostatic_parameters") {
        fObject->SetPreconditionerFastMultipoleParameters(q);
        return true;
    }
    return false;
}

template<> inline bool KCUDAFastMultipoleFieldSolverBuilder::AddAttribute(KContainer* aContainer)
{
    const std::string& name = aContainer->GetName();
    if (name == "device")
        aContainer->CopyTo(fObject, &KEMField::KCUDAFastMultipoleFieldSolver::SetDevice);
    else if (name == "near_field_analytic")
        aContainer->CopyTo(fObject, &KEMField::KCUDAFastMultipoleFieldSolver::SetNearFieldAnalytic);
    else
        return KEMCUFastMultipoleAttribute(*fObject->GetParameters(), aContainer);
    return true;
}

template<> inline bool KCUDARobinHoodChargeDensitySolverBuilder::AddAttribute(KContainer* aContainer)
{
    const std::string& name = aContainer->GetName();
    if (name == "tolerance")
        aContainer->CopyTo(fObject, &KEMField::KCUDARobinHoodChargeDensitySolver::SetTolerance);
    else if (name == "check_sub_interval")
        aContainer->CopyTo(fObject, &KEMField::KCUDARobinHoodChargeDensitySolver::SetCheckSubInterval);
    else if (name == "cache_matrix_elements")
        aContainer->CopyTo(fObject, &KEMField::KCUDARobinHoodChargeDensitySolver::CacheMatrixElements);
    else if (name == "device")
        aContainer->CopyTo(fObject, &KEMField::KCUDARobinHoodChargeDensitySolver::SetDevice);
    else
        return false;
    return true;
}

template<> inline bool KCUDAElectricFieldSolverBuilder::AddAttribute(KContainer* aContainer)
{
    const std::string& name = aContainer->GetName();
    if (name == "precision") {
        const int p = KEMField::KEMCUPrecisionFromName(aContainer->AsString());
        if (p < 0) {
            BINDINGMSG(eWarning) << "cuda_field_solver: precision must be <fp64>, <mixed> or <fp32>" << eom;
            return false;
        }
        fObject->SetPrecision(p);
    }
    else if (name == "device")
        aContainer->CopyTo(fObject, &KEMField::KCUDAElectricFieldSolver::SetDevice);
    else
        return false;
    return true;
}

template<> inline bool KIntegratingElectrostaticFieldSolverCUDABuilder::AddAttribute(KContainer* aContainer)
{
    const std::string& name = aContainer->GetName();
    if (name == "integrator")
        return AddElectrostaticIntegratorPolicy(fObject, aContainer);
    if (name == "use_opencl")
        aContainer->CopyTo(fObject, &KEMField::KIntegratingElectrostaticFieldSolverCUDA::UseOpenCL);
    else if (name == "use_cuda")
        aContainer->CopyTo(fObject, &KEMField::KIntegratingElectrostaticFieldSolverCUDA::UseCUDA);
    else if (name == "cuda_device")
        aContainer->CopyTo(fObject, &KEMField::KIntegratingElectrostaticFieldSolverCUDA::SetCUDADevice);
    else if (name == "cuda_precision") {
        const int p = KEMField::KEMCUPrecisionFromName(aContainer->AsString());
        if (p < 0) {
            BINDINGMSG(eWarning) << "integrating_field_solver: cuda_precision must be <fp64>, <mixed> or <fp32>"
                                 << eom;
            return false;
        }
        fObject->SetCUDAPrecision(p);
    }
    else
        return false;
    return true;
}

// Registers the attributes of the five builders and the six elements under the parent builder
// (KElectrostaticBoundaryFieldBuilder in a KEMField build, whose AddElement takes any
// KChargeDensitySolver and KElectricFieldSolver). Call once, e.g.
//   STATICINT sKEMCU = katrin::RegisterKEMCUBuilders<katrin::KElectrostaticBoundaryFieldBuilder>();
template<class XParentBuilder> int RegisterKEMCUBuilders()
{
    KCUDAChargeDensitySolverBuilder::Attribute<double>("tolerance");
    KCUDAChargeDensitySolverBuilder::Attribute<int>("max_iterations");
    KCUDAChargeDensitySolverBuilder::Attribute<std::string>("mode");
    KCUDAChargeDensitySolverBuilder::Attribute<int>("device");
    KCUDAChargeDensitySolverBuilder::Attribute<std::string>("solver_name");
    KCUDAChargeDensitySolverBuilder::Attribute<std::string>("preconditioner");
    KCUDAChargeDensitySolverBuilder::Attribute<double>("preconditioner_tolerance");
    KCUDAChargeDensitySolverBuilder::Attribute<double>("time_limit_in_seconds");
    for (const char* a : {"iterations_between_restarts", "max_preconditioner_iterations", "preconditioner_degree",
                          "intermediate_save_interval", "time_check_interval"})
        KCUDAChargeDensitySolverBuilder::Attribute<unsigned int>(a);
    for (const char* a : {"use_display", "show_plot", "use_timer"})
        KCUDAChargeDensitySolverBuilder::Attribute<bool>(a);
    KCUDAChargeDensitySolverBuilder::ComplexElement<KEMField::KFMElectrostaticParameters>("fftm_multiplication");
    KCUDAChargeDensitySolverBuilder::ComplexElement<KEMField::KFMElectrostaticParameters>(
        "preconditioner_electrostatic_parameters");
    KCUDARobinHoodChargeDensitySolverBuilder::Attribute<double>("tolerance");
    KCUDARobinHoodChargeDensitySolverBuilder::Attribute<unsigned int>("check_sub_interval");
    KCUDARobinHoodChargeDensitySolverBuilder::Attribute<bool>("cache_matrix_elements");
    KCUDARobinHoodChargeDensitySolverBuilder::Attribute<int>("device");
    KCUDAElectricFieldSolverBuilder::Attribute<std::string>("precision");
    KCUDAElectricFieldSolverBuilder::Attribute<int>("device");
    KIntegratingElectrostaticFieldSolverCUDABuilder::Attribute<std::string>("integrator");
    KIntegratingElectrostaticFieldSolverCUDABuilder::Attribute<bool>("use_opencl");
    KIntegratingElectrostaticFieldSolverCUDABuilder::Attribute<bool>("use_cuda");
    KIntegratingElectrostaticFieldSolverCUDABuilder::Attribute<std::string>("cuda_precision");
    KIntegratingElectrostaticFieldSolverCUDABuilder::Attribute<int>("cuda_device");
    XParentBuilder::template ComplexElement<KEMField::KCUDAChargeDensitySolver>("cuda_krylov_charge_density_solver");
    XParentBuilder::template ComplexElement<KEMField::KCUDAChargeDensitySolver>("cuda_krylov_bem_solver");
    XParentBuilder::template ComplexElement<KEMField::KCUDARobinHoodChargeDensitySolver>(
        "cuda_robin_hood_charge_density_solver");
    for (const char* a : {"top_level_divisions", "tree_level_divisions", "expansion_degree", "neighbor_order",
                          "maximum_tree_depth", "verbosity"}) {
        KCUDAChargeDensitySolverBuilder::Attribute<unsigned int>(a);
        KCUDAFastMultipoleFieldSolverBuilder::Attribute<unsigned int>(a);
    }
    for (const char* a : {"region_expansion_factor", "world_cube_center_x", "world_cube_center_y",
                          "world_cube_center_z", "world_cube_length", "insertion_ratio"}) {
        KCUDAChargeDensitySolverBuilder::Attribute<double>(a);
        KCUDAFastMultipoleFieldSolverBuilder::Attribute<double>(a);
    }
    for (const char* a : {"use_region_size_estimation", "use_caching"}) {
        KCUDAChargeDensitySolverBuilder::Attribute<bool>(a);
        KCUDAFastMultipoleFieldSolverBuilder::Attribute<bool>(a);
    }
    KCUDAFastMultipoleFieldSolverBuilder::Attribute<int>("device");
    KCUDAFastMultipoleFieldSolverBuilder::Attribute<bool>("near_field_analytic");
    XParentBuilder::template ComplexElement<KEMField::KCUDAElectricFieldSolver>("cuda_field_solver");
    XParentBuilder::template ComplexElement<KEMField::KCUDAFastMultipoleFieldSolver>(
        "cuda_fast_multipole_field_solver");
    XParentBuilder::template ComplexElement<KEMField::KIntegratingElectrostaticFieldSolverCUDA>(
        "integrating_field_solver");
    return 0;
}

}  // namespace katrin
