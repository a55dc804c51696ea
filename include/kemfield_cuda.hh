// kemfield_cuda.hh -- C++ adaptors that plug the B200 backend (include/kemcu.h) into KEMField
// beside its CPU and OpenCL backends, against the reference's unchanged interfaces:
//
//   KCUDASurfaceContainer        flattens a KSurfaceContainer in container order (the matrix
//                                order, KSurfaceContainer.cc:58-72) onto the device and writes
//                                charge densities back into each KElectrostaticBasis, like
//                                KOpenCLSurfaceContainer (KOpenCLSurfaceContainer.cc:10-266)
//   KCUDAIntegratingFieldSolver  Potential / ElectricField / ElectricFieldAndPotential of
//                                KIntegratingFieldSolver (KElectrostaticIntegratingFieldSolver.hh:261-339),
//                                plus a batched ElectricFieldAndPotential over many points; it is
//                                KIntegratingFieldSolver<Integrator, ElectrostaticCUDA>, the
//                                specialisation for the ElectrostaticCUDA Kind, as the OpenCL
//                                plugin specialises ElectrostaticOpenCL
//                                (KOpenCLElectrostaticIntegratingFieldSolver.hh:20)
//   KCUDAElectricFieldSolver     a KElectricFieldSolver (KElectricFieldSolver.hh:19-77), the
//                                object KElectrostaticBoundaryField::SetFieldSolver takes
//                                (KElectrostaticBoundaryField.cc:39-42) beside
//                                KIntegratingElectrostaticFieldSolver; Kassiopeia's
//                                KSElectricKEMField then evaluates its fields on the GPU
//   KCUDABoundaryIntegralMatrix  a KSquareMatrix whose virtual Multiply (KMatrix.hh:87-99) and
//                                operator()(i, j) (KBoundaryIntegralMatrix.hh:31-55) run on the GPU
//   KCUDAChargeDensitySolver     the whole GMRES charge-density solve on the device
//                                (KSimpleIterativeKrylovSolver<double, KGeneralizedMinimalResidual>)
//   KCUDARobinHoodChargeDensitySolver  Robin Hood on the device (KRobinHood.hh:61-104)
//                                both KChargeDensitySolver subclasses that read and write
//                                KEMField's solution cache (KChargeDensitySolver.cc:51-280)
//
// Header-only; include after the reference's KEMField headers and link with -lkemcu and the
// KEMField libraries that hold KChargeDensitySolver and KEMFileInterface. Errors
// surface as KEMSimpleException, as elsewhere in KEMField.
#pragma once

#include "KChargeDensitySolver.hh"
#include "KElectricFieldSolver.hh"
#include "KElectrostaticBasis.hh"
#include "KEMConstants.hh"
#include "KEMSimpleException.hh"
#include "KIntegratingFieldSolverTemplate.hh"
#include "KSquareMatrix.hh"
#include "KSurfaceContainer.hh"
#include "KSurfaceTypes.hh"
#include "kemcu.h"

#include <climits>
#include <memory>
#include <string>
#include <utility>
#include <vector>

namespace KEMField
{

// backend Kind tag, next to ElectrostaticSingleThread (KElectrostaticBoundaryIntegrator.hh:44) and
// ElectrostaticOpenCL (KOpenCLElectrostaticBoundaryIntegrator.hh:24)
class ElectrostaticCUDA;

// The integrator of the CUDA Kind: the device evaluates the reference's numeric policy
// (KEBIFactory::MakeNumeric: cubature bands, RWG near field, analytic wires); what is chosen here
// is only the arithmetic of the cubature nodes (KEMCU_FP64 or KEMCU_MIXED, kemcu_precision).
class KCUDAElectrostaticBoundaryIntegrator
{
  public:
    using Basis = KElectrostaticBasis;
    using Kind = ElectrostaticCUDA;
    explicit KCUDAElectrostaticBoundaryIntegrator(int precision = KEMCU_FP64) : fPrecision(precision) {}
    int Precision() const
    {
        return fPrecision;
    }

  private:
    int fPrecision;
};

inline void KCUDACheck(kemcu_ctx* ctx, int rc)
{
    if (rc != KEMCU_OK)
        throw KEMSimpleException(std::string("kemcu: ") + kemcu_last_error(ctx));
}

class KCUDASurfaceContainer
{
  public:
    explicit KCUDASurfaceContainer(KSurfaceContainer& container, int device = 0) : fContainer(container)
    {
        kemcu_config cfg;
        kemcu_default_config(&cfg);
        cfg.device = device;
        cfg.one_over_four_pi_eps0 = KEMConstants::OneOverFourPiEps0;
        cfg.eps0 = KEMConstants::Eps0;
        const int rc = kemcu_create(&fCtx, &cfg);
        if (rc != KEMCU_OK) {
            const std::string msg = fCtx ? kemcu_last_error(fCtx) : "context creation failed";
            kemcu_destroy(fCtx);
            throw KEMSimpleException("kemcu: " + msg);
        }
        Flatten();
    }
    ~KCUDASurfaceContainer()
    {
        kemcu_destroy(fCtx);
    }
    KCUDASurfaceContainer(const KCUDASurfaceContainer&) = delete;
    KCUDASurfaceContainer& operator=(const KCUDASurfaceContainer&) = delete;

    kemcu_ctx* Context() const
    {
        return fCtx;
    }
    unsigned int size() const
    {
        return fContainer.size();
    }

    // sigma from each KElectrostaticBasis onto the device
    void WriteBasisData()
    {
        std::vector<double> s(size());
        for (unsigned i = 0; i < size(); i++)
            s[i] = Basis(i)->GetSolution();
        KCUDACheck(fCtx, kemcu_set_sigma(fCtx, s.data()));
    }
    // device sigma back into each KElectrostaticBasis (KOpenCLSurfaceContainer::ReadBasisData)
    void ReadBasisData()
    {
        std::vector<double> s(size());
        KCUDACheck(fCtx, kemcu_get_sigma(fCtx, s.data()));
        for (unsigned i = 0; i < size(); i++)
            Basis(i)->GetSolution() = s[i];
    }

  private:
    KElectrostaticBasis* Basis(unsigned i) const
    {
        auto* b = dynamic_cast<KElectrostaticBasis*>(fContainer[i]->GetBasis());
        if (!b)
            throw KEMSimpleException("kemcu: element without an electrostatic basis");
        return b;
    }

    void Flatten()
    {
        const unsigned n = size();
        std::vector<int32_t> shape(n), boundary(n);
        std::vector<double> geom(11 * (size_t) n, 0.), value(n);
        for (unsigned i = 0; i < n; i++) {
            KSurfacePrimitive* s = fContainer[i];
            double* g = &geom[11 * (size_t) i];
            if (auto* t = dynamic_cast<KTriangle*>(s->GetShape())) {
                shape[i] = KEMCU_TRIANGLE;
                Planar(*t, g);
            }
            else if (auto* r = dynamic_cast<KRectangle*>(s->GetShape())) {
                shape[i] = KEMCU_RECTANGLE;
                Planar(*r, g);
            }
            else if (auto* l = dynamic_cast<KLineSegment*>(s->GetShape())) {
                shape[i] = KEMCU_LINE_SEGMENT;
                for (int c = 0; c < 3; c++) {
                    g[c] = l->GetP0()[c];
                    g[3 + c] = l->GetP1()[c];
                }
                g[6] = l->GetDiameter();
            }
            else if (auto* cs = dynamic_cast<KConicSection*>(s->GetShape())) {
                shape[i] = KEMCU_CONIC_SECTION;
                g[0] = cs->GetR0();
                g[1] = cs->GetZ0();
                g[2] = cs->GetR1();
                g[3] = cs->GetZ1();
            }
            else if (auto* rg = dynamic_cast<KRing*>(s->GetShape())) {
                shape[i] = KEMCU_RING;
                g[0] = rg->GetR();
                g[1] = rg->GetZ();
            }
            else
                throw KEMSimpleException("kemcu: only triangles, rectangles, line segments, conic sections and rings "
                                         "are supported");
            if (auto* d = dynamic_cast<KBoundaryType<KElectrostaticBasis, KDirichletBoundary>*>(s->GetBoundary())) {
                boundary[i] = KEMCU_DIRICHLET;
                value[i] = d->GetBoundaryValue();
            }
            else if (auto* nb = dynamic_cast<KBoundaryType<KElectrostaticBasis, KNeumannBoundary>*>(s->GetBoundary())) {
                boundary[i] = KEMCU_NEUMANN;
                value[i] = nb->GetNormalBoundaryFlux();
            }
            else
                throw KEMSimpleException("kemcu: unsupported boundary type");
        }
        KCUDACheck(fCtx, kemcu_set_geometry(fCtx, n, shape.data(), boundary.data(), geom.data(), value.data()));
    }

    template<class S> static void Planar(const S& s, double* g)
    {
        g[0] = s.GetA();
        g[1] = s.GetB();
        for (int c = 0; c < 3; c++) {
            g[2 + c] = s.GetP0()[c];
            g[5 + c] = s.GetN1()[c];
            g[8 + c] = s.GetN2()[c];
        }
    }

    KSurfaceContainer& fContainer;
    kemcu_ctx* fCtx = nullptr;
};

class KCUDAIntegratingFieldSolver
{
  public:
    explicit KCUDAIntegratingFieldSolver(KCUDASurfaceContainer& container, int precision = KEMCU_FP64) :
        fContainer(container),
        fPrecision(precision)
    {}
    double Potential(const KPosition& P) const
    {
        double o[4];
        Eval(&P[0], 1, o, KEMCU_POTENTIAL);
        return o[3];
    }
    KFieldVector ElectricField(const KPosition& P) const
    {
        double o[4];
        Eval(&P[0], 1, o, KEMCU_FIELD);
        return KFieldVector(o[0], o[1], o[2]);
    }
    std::pair<KFieldVector, double> ElectricFieldAndPotential(const KPosition& P) const
    {
        double o[4];
        Eval(&P[0], 1, o, KEMCU_FIELD_AND_POTENTIAL);
        return std::make_pair(KFieldVector(o[0], o[1], o[2]), o[3]);
    }
    // batched extension: P n x 3, out n x 4 (Ex, Ey, Ez, phi)
    void ElectricFieldAndPotential(const double* P, size_t n, double* out) const
    {
        Eval(P, n, out, KEMCU_FIELD_AND_POTENTIAL);
    }

  private:
    void Eval(const double* P, size_t n, double* out, int what) const
    {
        KCUDACheck(fContainer.Context(), kemcu_field(fContainer.Context(), P, n, out, fPrecision, what));
    }
    KCUDASurfaceContainer& fContainer;
    int fPrecision;
};

// KIntegratingFieldSolver<KCUDAElectrostaticBoundaryIntegrator> resolves here through the
// integrator's Kind, as KIntegratingFieldSolver<KOpenCLElectrostaticBoundaryIntegrator> does for
// OpenCL (KIntegratingElectrostaticFieldSolver.cc:44-69)
template<class Integrator>
class KIntegratingFieldSolver<Integrator, ElectrostaticCUDA> : public KCUDAIntegratingFieldSolver
{
  public:
    KIntegratingFieldSolver(KCUDASurfaceContainer& container, const Integrator& integrator) :
        KCUDAIntegratingFieldSolver(container, integrator.Precision())
    {}
};

// The field solver KElectrostaticBoundaryField holds (SetFieldSolver). Initialize, called by the
// boundary field after its charge-density solver has written sigma into every
// KElectrostaticBasis (KElectrostaticBoundaryField.cc:75-93), flattens the container onto the
// device with those charge densities; every field call then runs on the GPU. Deinitialize
// releases the device context.
class KCUDAElectricFieldSolver : public KElectricFieldSolver
{
  public:
    explicit KCUDAElectricFieldSolver(int precision = KEMCU_FP64, int device = 0) :
        fPrecision(precision),
        fDevice(device)
    {}
    // the arithmetic of the cubature nodes: KEMCU_FP64 (default), KEMCU_MIXED or KEMCU_FP32
    void SetPrecision(int precision)
    {
        fPrecision = precision;
    }
    void UseMixedPrecision(bool choice)
    {
        fPrecision = choice ? KEMCU_MIXED : KEMCU_FP64;
    }
    void SetDevice(int device)
    {
        fDevice = device;
    }
    int GetPrecision() const
    {
        return fPrecision;
    }
    int GetDevice() const
    {
        return fDevice;
    }
    // the single-point calls of KElectricFieldSolver stay visible beside the batched ones
    using KElectricFieldSolver::ElectricFieldAndPotential;
    // batched extension: n points P (x, y, z each), out n x 4 (Ex, Ey, Ez, phi); one device call
    void ElectricFieldAndPotential(const double* P, size_t n, double* out) const
    {
        Solver().ElectricFieldAndPotential(P, n, out);
    }
    void ElectricFieldAndPotential(const std::vector<KPosition>& P, std::vector<KFieldVector>& E,
                                   std::vector<double>& phi) const
    {
        std::vector<double> p(3 * P.size()), o(4 * P.size());
        for (size_t i = 0; i < P.size(); i++)
            for (int c = 0; c < 3; c++)
                p[3 * i + c] = P[i][c];
        Solver().ElectricFieldAndPotential(p.data(), P.size(), o.data());
        E.resize(P.size());
        phi.resize(P.size());
        for (size_t i = 0; i < P.size(); i++) {
            E[i] = KFieldVector(o[4 * i], o[4 * i + 1], o[4 * i + 2]);
            phi[i] = o[4 * i + 3];
        }
    }
    KCUDASurfaceContainer* DeviceContainer() const
    {
        return fContainer.get();
    }

  private:
    using Solver_t = KIntegratingFieldSolver<KCUDAElectrostaticBoundaryIntegrator>;
    const Solver_t& Solver() const
    {
        if (!fSolver)
            throw KEMSimpleException("kemcu: KCUDAElectricFieldSolver used before Initialize");
        return *fSolver;
    }
    void InitializeCore(KSurfaceContainer& container) override
    {
        fContainer = std::make_unique<KCUDASurfaceContainer>(container, fDevice);
        fContainer->WriteBasisData();
        fIntegrator = KCUDAElectrostaticBoundaryIntegrator(fPrecision);
        fSolver = std::make_unique<Solver_t>(*fContainer, fIntegrator);
    }
    void DeinitializeCore() override
    {
        fSolver.reset();
        fContainer.reset();
    }
    double PotentialCore(const KPosition& P) const override
    {
        return Solver().Potential(P);
    }
    KFieldVector ElectricFieldCore(const KPosition& P) const override
    {
        return Solver().ElectricField(P);
    }
    std::pair<KFieldVector, double> ElectricFieldAndPotentialCore(const KPosition& P) const override
    {
        return Solver().ElectricFieldAndPotential(P);
    }

    int fPrecision, fDevice;
    KCUDAElectrostaticBoundaryIntegrator fIntegrator;
    std::unique_ptr<KCUDASurfaceContainer> fContainer;
    std::unique_ptr<Solver_t> fSolver;
};

class KCUDABoundaryIntegralMatrix : public KSquareMatrix<double>
{
  public:
    explicit KCUDABoundaryIntegralMatrix(KCUDASurfaceContainer& container, bool assembled = false) :
        fContainer(container),
        fAssembled(assembled)
    {}
    unsigned int Dimension() const override
    {
        return fContainer.size();
    }
    const double& operator()(unsigned int i, unsigned int j) const override
    {
        KCUDACheck(fContainer.Context(), kemcu_matrix_element(fContainer.Context(), i, j, &fEntry));
        return fEntry;
    }
    void Multiply(const KVector<double>& x, KVector<double>& y) const override
    {
        const unsigned n = Dimension();
        std::vector<double> xs(n), ys(n);
        for (unsigned i = 0; i < n; i++)
            xs[i] = x(i);
        KCUDACheck(fContainer.Context(),
                   kemcu_matvec(fContainer.Context(), xs.data(), ys.data(), 1, KEMCU_FP64, fAssembled ? 1 : 0));
        for (unsigned i = 0; i < n; i++)
            y[i] = ys[i];
    }

  private:
    KCUDASurfaceContainer& fContainer;
    bool fAssembled;
    mutable double fEntry = 0.;
};

// The charge-density solvers are KChargeDensitySolver subclasses (KChargeDensitySolver.hh:17-45),
// so KElectrostaticBoundaryField::SetChargeDensitySolver (KElectrostaticBoundaryField.cc:29-32)
// takes them where it takes KKrylovChargeDensitySolver or KRobinHoodChargeDensitySolver.
// Initialize(container) keeps the reference's solution cache protocol
// (KRobinHoodChargeDensitySolver.cc:83-216): FindSolution(tolerance) first, which loads a cached
// solution of the same shape and boundary hashes solved to at least this tolerance (or a
// superposition of such solutions); otherwise the solve runs on the device, sigma is written into
// each KElectrostaticBasis and SaveSolution(tolerance) stores it through KEMFileInterface.
// Solve(KCUDASurfaceContainer&) is the uncached device solve on an existing context.
class KCUDAChargeDensitySolverBase : public KChargeDensitySolver
{
  public:
    KCUDAChargeDensitySolverBase(double tolerance, int device) : fTolerance(tolerance), fDevice(device)
    {
        // the defaults KElectrostaticBoundaryField passes in before Initialize
        // (KElectrostaticBoundaryField.cc:20-21, 79); it overrides them when it drives the solver
        SetHashProperties(20, 1.e-14);
    }
    void SetTolerance(double d)
    {
        fTolerance = d;
    }
    double GetTolerance() const
    {
        return fTolerance;
    }
    void SetDevice(int device)
    {
        fDevice = device;
    }
    // true when the last Initialize took its solution from the cache, without a device solve
    bool SolutionFromCache() const
    {
        return fFromCache;
    }

  protected:
    virtual void DeviceSolve(KCUDASurfaceContainer& container) = 0;
    double fTolerance;
    int fDevice;

  private:
    void InitializeCore(KSurfaceContainer& container) override
    {
        if (container.empty())
            throw KEMSimpleException("kemcu: charge density solver got no electrode elements");
        fFromCache = FindSolution(fTolerance, container);
        if (fFromCache)
            return;
        {
            KCUDASurfaceContainer gpu(container, fDevice);
            DeviceSolve(gpu);
        }
        SaveSolution(fTolerance, container);
    }
    bool fFromCache = false;
};

// the library's default fast multipole parameters (kemcu_fftm_default_params)
inline kemcu_fftm_params KCUDADefaultFastMultipoleParameters()
{
    kemcu_fftm_params p;
    kemcu_fftm_default_params(&p);
    return p;
}

// KKrylovChargeDensitySolver analogue: the whole Krylov solve on the device, GMRES by default
// (KSimpleIterativeKrylovSolver<double, KGeneralizedMinimalResidual>) on the direct operator or
// (mode fftm) on the fast multipole one; with the solver / preconditioner / restart choices of
// krylov_bem_solver (KKrylovChargeDensitySolverOld with KFMElectrostaticFastMultipoleBoundaryValueSolver)
class KCUDAChargeDensitySolver : public KCUDAChargeDensitySolverBase
{
  public:
    KCUDAChargeDensitySolver(double tolerance = 1e-10, int max_iterations = 500, int mode = KEMCU_SOLVE_PLAIN,
                             int device = 0) :
        KCUDAChargeDensitySolverBase(tolerance, device),
        fMaxIterations(max_iterations),
        fMode(mode)
    {
        kemcu_fftm_default_params(&fFftm);
    }
    // the tree of KEMCU_SOLVE_FFTM (GMRES on the fast multipole operator, the device form of
    // KKrylovChargeDensitySolver with KFastMultipoleMatrixGenerator)
    void SetFastMultipoleParameters(const kemcu_fftm_params& prm)
    {
        fFftm = prm;
        fFftmEstimate = prm.world_length <= 0.;
        fFftmWorldLength = prm.world_length;
    }
    kemcu_fftm_params& FastMultipoleParameters()
    {
        return fFftm;
    }
    const kemcu_fftm_params& GetFastMultipoleParameters() const
    {
        return fFftm;
    }
    // the world cube: estimated from the elements (true, the default) or the centre in
    // FastMultipoleParameters().world_center with this side length
    void SetFastMultipoleRegionEstimation(bool choice)
    {
        fFftmEstimate = choice;
    }
    void SetFastMultipoleWorldLength(double length)
    {
        fFftmWorldLength = length;
    }
    void SetMaxIterations(int n)
    {
        fMaxIterations = n;
    }
    void SetMode(int mode)
    {
        fMode = mode;
    }
    int GetMaxIterations() const
    {
        return fMaxIterations;
    }
    int GetMode() const
    {
        return fMode;
    }
    // the solver and preconditioner choices of the reference's Krylov solvers (the attributes
    // solver_name, preconditioner, iterations_between_restarts, preconditioner_tolerance,
    // max_preconditioner_iterations and preconditioner_degree of krylov_bem_solver,
    // KKrylovChargeDensitySolverOldBuilder.hh, and the dispatch of
    // KFMElectrostaticFastMultipoleBoundaryValueSolver.cc:189-233). Plain GMRES without restarts
    // runs kemcu_gmres; any other choice runs kemcu_krylov_solve (for the refinement modes mixed,
    // assembled and fp32 the solver and preconditioner apply to the inner solves).
    void SetSolverName(const std::string& name)
    {
        if (name == "gmres")
            fSolver = KEMCU_KRYLOV_GMRES;
        else if (name == "bicgstab")
            fSolver = KEMCU_KRYLOV_BICGSTAB;
        else
            throw KEMSimpleException("kemcu: unknown Krylov solver <" + name + "> (gmres, bicgstab)");
    }
    // "none", "jacobi", "implicit_krylov" (an inner GMRES on the solver's tree at
    // preconditioner_degree, or on SetPreconditionerMode's operator for a direct system) or
    // "independent_implicit_krylov" (an inner GMRES on the tree of
    // SetPreconditionerFastMultipoleParameters)
    void SetPreconditionerName(const std::string& name)
    {
        if (name == "none")
            fPrecon = KEMCU_PRECON_NONE;
        else if (name == "jacobi")
            fPrecon = KEMCU_PRECON_JACOBI;
        else if (name == "implicit_krylov" || name == "independent_implicit_krylov")
            fPrecon = KEMCU_PRECON_IMPLICIT_KRYLOV;
        else
            throw KEMSimpleException("kemcu: unknown preconditioner <" + name +
                                     "> (none, jacobi, implicit_krylov, independent_implicit_krylov)");
        fIndependent = name == "independent_implicit_krylov";
    }
    void SetIterationsBetweenRestart(unsigned int n)
    {
        fRestart = n >= (unsigned int) INT_MAX ? 0 : (int) n;
    }
    void SetPreconditionerTolerance(double t)
    {
        fPreTolerance = t;
    }
    void SetMaxPreconditionerIterations(unsigned int n)
    {
        fPreMaxIterations = n >= (unsigned int) INT_MAX ? INT_MAX : (int) n;
    }
    // the degree of the implicit_krylov preconditioner's tree (0..15; 0 by default, as the
    // reference's KFMElectrostaticFastMultipoleBoundaryValueSolverConfiguration)
    void SetPreconditionerDegree(unsigned int d)
    {
        fPreDegree = (int) d;
    }
    // the tree of independent_implicit_krylov (preconditioner_electrostatic_parameters); a world
    // length <= 0 estimates the world cube
    void SetPreconditionerFastMultipoleParameters(const kemcu_fftm_params& prm)
    {
        fPreFftm = prm;
    }
    // the operator of the implicit Krylov preconditioner for a direct system (kemcu_solve_mode;
    // default KEMCU_SOLVE_FP32, the FP32 far-field matrix-free operator)
    void SetPreconditionerMode(int mode)
    {
        fPreMode = mode;
    }
    int GetSolver() const
    {
        return fSolver;
    }
    int GetPreconditioner() const
    {
        return fPrecon;
    }
    bool IndependentPreconditioner() const
    {
        return fIndependent;
    }
    int GetIterationsBetweenRestart() const
    {
        return fRestart;
    }
    double GetPreconditionerTolerance() const
    {
        return fPreTolerance;
    }
    int GetMaxPreconditionerIterations() const
    {
        return fPreMaxIterations;
    }
    int GetPreconditionerDegree() const
    {
        return fPreDegree;
    }
    const kemcu_fftm_params& GetPreconditionerFastMultipoleParameters() const
    {
        return fPreFftm;
    }
    // XML form: "plain", "mixed", "assembled", "assembled_fp64", "fp32" or "fftm" (kemcu_solve_mode)
    void SetModeName(const std::string& name)
    {
        if (name == "plain")
            fMode = KEMCU_SOLVE_PLAIN;
        else if (name == "mixed")
            fMode = KEMCU_SOLVE_MIXED;
        else if (name == "assembled")
            fMode = KEMCU_SOLVE_ASSEMBLED;
        else if (name == "assembled_fp64")
            fMode = KEMCU_SOLVE_ASSEMBLED_FP64;
        else if (name == "fp32")
            fMode = KEMCU_SOLVE_FP32;
        else if (name == "fftm")
            fMode = KEMCU_SOLVE_FFTM;
        else
            throw KEMSimpleException("kemcu: unknown solve mode <" + name +
                                     "> (plain, mixed, assembled, assembled_fp64, fp32, fftm)");
    }
    // solves A sigma = b for the boundary values and writes sigma into the container
    kemcu_solve_stats Solve(KCUDASurfaceContainer& container) const
    {
        std::vector<double> x(container.size());
        kemcu_solve_stats st{};
        kemcu_fftm_params q = fFftm;
        q.world_length = fFftmEstimate ? 0. : fFftmWorldLength;
        if (fMode == KEMCU_SOLVE_FFTM)
            KCUDACheck(container.Context(), kemcu_fftm_configure(container.Context(), &q));
        if (fSolver == KEMCU_KRYLOV_GMRES && fPrecon == KEMCU_PRECON_NONE && fRestart == 0) {
            KCUDACheck(container.Context(),
                       kemcu_gmres(container.Context(), nullptr, x.data(), 1, fTolerance, fMaxIterations, fMode, &st));
        }
        else {
            kemcu_krylov_params p;
            kemcu_krylov_default_params(&p);
            p.solver = fSolver;
            p.mode = fMode;
            p.tolerance = fTolerance;
            p.max_iterations = fMaxIterations;
            p.iterations_between_restarts = fRestart;
            p.preconditioner = fPrecon;
            p.preconditioner_tolerance = fPreTolerance;
            p.max_preconditioner_iterations = fPreMaxIterations;
            p.preconditioner_mode = fPreMode;
            if (fPrecon == KEMCU_PRECON_IMPLICIT_KRYLOV && fMode == KEMCU_SOLVE_FFTM) {
                // implicit_krylov: the solver's tree at the preconditioner's degree
                // (KFMElectrostaticFastMultipoleBoundaryValueSolver.cc:731-737); independent: its own
                kemcu_fftm_params pq = q;
                if (fIndependent)
                    pq = fPreFftm;
                else
                    pq.degree = fPreDegree;
                KCUDACheck(container.Context(), kemcu_fftm_configure_preconditioner(container.Context(), &pq));
                p.preconditioner_mode = KEMCU_SOLVE_FFTM;
            }
            KCUDACheck(container.Context(), kemcu_krylov_solve(container.Context(), nullptr, x.data(), 1, &p, &st));
        }
        container.ReadBasisData();
        return st;
    }
    const kemcu_solve_stats& LastStats() const
    {
        return fStats;
    }

  private:
    void DeviceSolve(KCUDASurfaceContainer& container) override
    {
        fStats = Solve(container);
    }
    int fMaxIterations, fMode;
    kemcu_fftm_params fFftm;
    bool fFftmEstimate = true;
    double fFftmWorldLength = 0.;
    int fSolver = KEMCU_KRYLOV_GMRES, fPrecon = KEMCU_PRECON_NONE, fRestart = 0;
    bool fIndependent = false;
    double fPreTolerance = 0.01;
    int fPreMaxIterations = 30, fPreDegree = 0, fPreMode = KEMCU_SOLVE_FP32;
    kemcu_fftm_params fPreFftm = KCUDADefaultFastMultipoleParameters();
    kemcu_solve_stats fStats{};
};

// KRobinHoodChargeDensitySolver analogue (KRobinHood<double>::Solve, KRobinHood.hh:61-104):
// Robin Hood on the device, starting from the charge densities the container holds
class KCUDARobinHoodChargeDensitySolver : public KCUDAChargeDensitySolverBase
{
  public:
    KCUDARobinHoodChargeDensitySolver(double tolerance = 1e-8, int check_interval = 0, bool assembled = false,
                                      int device = 0) :
        KCUDAChargeDensitySolverBase(tolerance, device),
        fCheckInterval(check_interval),
        fAssembled(assembled)
    {}
    // residual check every i corrections; 0 picks the element count
    void SetCheckSubInterval(unsigned int i)
    {
        fCheckInterval = (int) i;
    }
    void CacheMatrixElements(bool choice)
    {
        fAssembled = choice;
    }
    int GetCheckSubInterval() const
    {
        return fCheckInterval;
    }
    bool MatrixElementsCached() const
    {
        return fAssembled;
    }
    kemcu_rh_stats Solve(KCUDASurfaceContainer& container) const
    {
        std::vector<double> x(container.size(), 0.);
        container.WriteBasisData();
        KCUDACheck(container.Context(), kemcu_get_sigma(container.Context(), x.data()));
        kemcu_rh_stats st{};
        KCUDACheck(container.Context(), kemcu_robin_hood(container.Context(), nullptr, x.data(), fTolerance,
                                                         fCheckInterval, 0, fAssembled ? 1 : 0, &st));
        container.ReadBasisData();
        return st;
    }
    const kemcu_rh_stats& LastStats() const
    {
        return fStats;
    }

  private:
    void DeviceSolve(KCUDASurfaceContainer& container) override
    {
        fStats = Solve(container);
    }
    int fCheckInterval;
    bool fAssembled;
    kemcu_rh_stats fStats{};
};

}  // namespace KEMField
