// Drop-in classes for KEMField's fast multipole method (FFTM) on the B200 backend, against the
// reference's own interfaces; needs the reference's FastMultipole headers on the include path.
//
//   KCUDAFastMultipoleFieldSolver      a KElectricFieldSolver, the device form of
//                                      KElectricFastMultipoleFieldSolver
//                                      (Interface/FieldSolvers/Electric/include/KElectricFastMultipoleFieldSolver.hh:25-66):
//                                      the same KFMElectrostaticParameters (GetParameters()), the
//                                      field and potential of kemcu_fftm_field
//   KCUDAFastMultipoleMatrixGenerator  a KBoundaryMatrixGenerator<double>, the device form of
//                                      KFastMultipoleMatrixGenerator
//                                      (FastMultipole/Utility/include/KFastMultipoleMatrixGenerator.hh:17-128),
//                                      the generator KKrylovChargeDensitySolver::SetMatrixGenerator
//                                      takes: Build() returns a KSquareMatrix whose Multiply is
//                                      kemcu_fftm_matvec
//
// Parameters map one to one (KCUDAFastMultipoleParameters). With use_region_estimation off the
// world cube is the one given; with it on, the library forms the reference's estimate (the
// minimal bounding ball of the element balls, KFMElectrostaticRegionSizeEstimator, in the
// surface container's order), so either way the tree is the reference's. Only the aggressive
// subdivision strategy is built; divisions 2..8 and zeromask 1..3 (kemcu_fftm_configure rejects
// others).
#pragma once

#include "KBoundaryMatrixGenerator.hh"
#include "KFMElectrostaticParameters.hh"
#include "kemfield_cuda.hh"

#include <memory>

namespace KEMField
{

inline kemcu_fftm_params KCUDAFastMultipoleParameters(const KFMElectrostaticParameters& p, bool near_analytic = true)
{
    kemcu_fftm_params q;
    kemcu_fftm_default_params(&q);
    q.degree = (int) p.degree;
    q.top_level_divisions = (int) p.top_level_divisions;
    q.divisions = (int) p.divisions;
    q.zeromask = (int) p.zeromask;
    q.maximum_tree_depth = (int) p.maximum_tree_depth;
    q.insertion_ratio = p.insertion_ratio;
    q.region_expansion_factor = p.region_expansion_factor;
    if (!p.use_region_estimation) {
        q.world_center[0] = p.world_center_x;
        q.world_center[1] = p.world_center_y;
        q.world_center[2] = p.world_center_z;
        q.world_length = p.world_length;
    }
    q.near_analytic = near_analytic ? 1 : 0;
    return q;
}

class KCUDAFastMultipoleFieldSolver : public KElectricFieldSolver
{
  public:
    explicit KCUDAFastMultipoleFieldSolver(int device = 0) : fDevice(device)
    {
        fParameters.degree = 8;  // KElectricFastMultipoleFieldSolver leaves the degree to the caller
    }
    KFMElectrostaticParameters* GetParameters()
    {
        return &fParameters;
    }
    // direct pairs by the analytic integrals (true, as the reference's FFTM field solver) or by
    // the numeric policy of the direct sum
    void SetNearFieldAnalytic(bool choice)
    {
        fNearAnalytic = choice;
    }
    void SetDevice(int device)
    {
        fDevice = device;
    }
    using KElectricFieldSolver::ElectricFieldAndPotential;
    // batched extension: n points P (x, y, z each), out n x 4 (Ex, Ey, Ez, phi)
    void ElectricFieldAndPotential(const double* P, size_t n, double* out) const
    {
        KCUDACheck(Ctx(), kemcu_fftm_field(Ctx(), P, n, out, KEMCU_FIELD_AND_POTENTIAL));
    }
    KCUDASurfaceContainer* DeviceContainer() const
    {
        return fContainer.get();
    }

  private:
    kemcu_ctx* Ctx() const
    {
        if (!fContainer)
            throw KEMSimpleException("kemcu: KCUDAFastMultipoleFieldSolver used before Initialize");
        return fContainer->Context();
    }
    void InitializeCore(KSurfaceContainer& container) override
    {
        fContainer = std::make_unique<KCUDASurfaceContainer>(container, fDevice);
        fContainer->WriteBasisData();
        const kemcu_fftm_params q = KCUDAFastMultipoleParameters(fParameters, fNearAnalytic);
        KCUDACheck(fContainer->Context(), kemcu_fftm_configure(fContainer->Context(), &q));
    }
    void DeinitializeCore() override
    {
        fContainer.reset();
    }
    void One(const KPosition& P, int what, double* o) const
    {
        const double p[3] = {P[0], P[1], P[2]};
        KCUDACheck(Ctx(), kemcu_fftm_field(Ctx(), p, 1, o, what));
    }
    double PotentialCore(const KPosition& P) const override
    {
        double o[4];
        One(P, KEMCU_POTENTIAL, o);
        return o[3];
    }
    KFieldVector ElectricFieldCore(const KPosition& P) const override
    {
        double o[4];
        One(P, KEMCU_FIELD, o);
        return KFieldVector(o[0], o[1], o[2]);
    }
    std::pair<KFieldVector, double> ElectricFieldAndPotentialCore(const KPosition& P) const override
    {
        double o[4];
        One(P, KEMCU_FIELD_AND_POTENTIAL, o);
        return {KFieldVector(o[0], o[1], o[2]), o[3]};
    }

    int fDevice;
    bool fNearAnalytic = true;
    KFMElectrostaticParameters fParameters;
    std::unique_ptr<KCUDASurfaceContainer> fContainer;
};

// The matrix Build() returns: it keeps its own device context (flattened container and tree)
class KCUDAFastMultipoleMatrix : public KSquareMatrix<double>
{
  public:
    KCUDAFastMultipoleMatrix(KSurfaceContainer& container, const kemcu_fftm_params& prm, int device) :
        fContainer(std::make_unique<KCUDASurfaceContainer>(container, device))
    {
        KCUDACheck(fContainer->Context(), kemcu_fftm_configure(fContainer->Context(), &prm));
    }
    unsigned int Dimension() const override
    {
        return fContainer->size();
    }
    // an entry of the operator: the direct boundary integral (the FFTM approximates its products)
    const double& operator()(unsigned int i, unsigned int j) const override
    {
        KCUDACheck(fContainer->Context(), kemcu_matrix_element(fContainer->Context(), i, j, &fEntry));
        return fEntry;
    }
    void Multiply(const KVector<double>& x, KVector<double>& y) const override
    {
        const unsigned n = Dimension();
        fX.resize(n);
        fY.resize(n);
        for (unsigned i = 0; i < n; i++)
            fX[i] = x(i);
        KCUDACheck(fContainer->Context(), kemcu_fftm_matvec(fContainer->Context(), fX.data(), fY.data(), 1));
        for (unsigned i = 0; i < n; i++)
            y[i] = fY[i];
    }
    kemcu_ctx* Context() const
    {
        return fContainer->Context();
    }

  private:
    std::unique_ptr<KCUDASurfaceContainer> fContainer;
    mutable std::vector<double> fX, fY;
    mutable double fEntry = 0.;
};

class KCUDAFastMultipoleMatrixGenerator : public KBoundaryMatrixGenerator<double>
{
  public:
    explicit KCUDAFastMultipoleMatrixGenerator(int device = 0) : fDevice(device) {}
    std::shared_ptr<KSquareMatrix<double>> Build(const KSurfaceContainer& container) const override
    {
        // KCUDASurfaceContainer reads the container (shapes, boundaries); it does not modify it
        auto& c = const_cast<KSurfaceContainer&>(container);
        const kemcu_fftm_params q = KCUDAFastMultipoleParameters(fParameters, true);
        return std::make_shared<KCUDAFastMultipoleMatrix>(c, q, fDevice);
    }
    // the setters of KFastMultipoleMatrixGenerator (KFastMultipoleMatrixGenerator.hh:27-112)
    void SetStrategy(int strategy)
    {
        fParameters.strategy = strategy;
    }
    void SetDegree(unsigned int degree)
    {
        fParameters.degree = degree;
    }
    void SetDivisions(unsigned int divisions)
    {
        fParameters.divisions = divisions;
    }
    void SetInsertionRatio(double r)
    {
        fParameters.insertion_ratio = r;
    }
    void SetMaximumTreeDepth(unsigned int depth)
    {
        fParameters.maximum_tree_depth = depth;
    }
    void SetRegionExpansionFactor(double f)
    {
        fParameters.region_expansion_factor = f;
    }
    void SetTopLevelDivisions(unsigned int d)
    {
        fParameters.top_level_divisions = d;
    }
    void SetUseRegionEstimation(bool choice)
    {
        fParameters.use_region_estimation = choice;
    }
    void SetWorldCenter(const KPosition& c)
    {
        fParameters.world_center_x = c[0];
        fParameters.world_center_y = c[1];
        fParameters.world_center_z = c[2];
    }
    void SetWorldLength(double length)
    {
        fParameters.world_length = length;
    }
    void SetZeromask(unsigned int zeromask)
    {
        fParameters.zeromask = zeromask;
    }
    void SetVerbosity(unsigned int v)
    {
        fParameters.verbosity = v;
    }
    void SetUseCaching(bool choice)
    {
        fParameters.use_caching = choice;
    }
    void SetDevice(int device)
    {
        fDevice = device;
    }
    const KFMElectrostaticParameters& GetParameters() const
    {
        return fParameters;
    }

  private:
    KFMElectrostaticParameters fParameters;
    int fDevice;
};

}  // namespace KEMField
