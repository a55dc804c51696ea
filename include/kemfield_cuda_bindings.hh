// kemfield_cuda_bindings.hh -- XML bindings of the B200 backend for KEMField's configuration files,
// in the reference's binding framework (Kommon's KComplexElement builders, the way
// KEMField/Source/Bindings/FieldSolvers/Electric/src/KIntegratingElectrostaticFieldSolverBuilder.cc
// and .../ChargeDensitySolvers/Electric/src/KRobinHoodChargeDensitySolverBuilder.cc bind theirs).
//
// Elements (children of the electrostatic boundary field element, registered by
// RegisterKEMCUBuilders<KElectrostaticBoundaryFieldBuilder>() in one source file of the build):
//
//   <cuda_krylov_charge_density_solver tolerance max_iterations mode device/>
//       KCUDAChargeDensitySolver: GMRES on the device; mode = plain | mixed | assembled | assembled_fp64 | fp32
//       | fftm (the fast multipole operator, default tree parameters)
//   <cuda_robin_hood_charge_density_solver tolerance check_sub_interval cache_matrix_elements device/>
//       KCUDARobinHoodChargeDensitySolver (attribute names of the reference's robin_hood element)
//   <cuda_field_solver precision device/>
//       KCUDAElectricFieldSolver; precision = fp64 | mixed | fp32
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
#include "KIntegratingElectrostaticFieldSolver.hh"
#include "kemfield_cuda.hh"

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

template<> inline bool KCUDAChargeDensitySolverBuilder::AddAttribute(KContainer* aContainer)
{
    const std::string& name = aContainer->GetName();
    if (name == "tolerance")
        aContainer->CopyTo(fObject, &KEMField::KCUDAChargeDensitySolver::SetTolerance);
    else if (name == "max_iterations")
        aContainer->CopyTo(fObject, &KEMField::KCUDAChargeDensitySolver::SetMaxIterations);
    else if (name == "device")
        aContainer->CopyTo(fObject, &KEMField::KCUDAChargeDensitySolver::SetDevice);
    else if (name == "mode") {
        try {
            fObject->SetModeName(aContainer->AsString());
        }
        catch (KEMField::KEMSimpleException& e) {
            BINDINGMSG(eWarning) << e.what() << eom;
            return false;
        }
    }
    else
        return false;
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

// Registers the attributes of the four builders and the four elements under the parent builder
// (KElectrostaticBoundaryFieldBuilder in a KEMField build, whose AddElement takes any
// KChargeDensitySolver and KElectricFieldSolver). Call once, e.g.
//   STATICINT sKEMCU = katrin::RegisterKEMCUBuilders<katrin::KElectrostaticBoundaryFieldBuilder>();
template<class XParentBuilder> int RegisterKEMCUBuilders()
{
    KCUDAChargeDensitySolverBuilder::Attribute<double>("tolerance");
    KCUDAChargeDensitySolverBuilder::Attribute<int>("max_iterations");
    KCUDAChargeDensitySolverBuilder::Attribute<std::string>("mode");
    KCUDAChargeDensitySolverBuilder::Attribute<int>("device");
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
    XParentBuilder::template ComplexElement<KEMField::KCUDARobinHoodChargeDensitySolver>(
        "cuda_robin_hood_charge_density_solver");
    XParentBuilder::template ComplexElement<KEMField::KCUDAElectricFieldSolver>("cuda_field_solver");
    XParentBuilder::template ComplexElement<KEMField::KIntegratingElectrostaticFieldSolverCUDA>(
        "integrating_field_solver");
    return 0;
}

}  // namespace katrin
