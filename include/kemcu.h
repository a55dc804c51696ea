/*
 * kemcu.h -- C ABI of the B200 (sm_100a) backend for KEMField's electrostatic
 * boundary-element hot path.
 *
 * Plain C: pointers, sizes and status codes only. A context owns one CUDA device and one
 * stream; it is not re-entrant (the reference's solvers are not either, they keep static
 * locals, KBoundaryIntegralMatrix.hh:42-44), but separate contexts may be used from
 * separate threads. All functions return KEMCU_OK (0) or a negative KEMCU_E* code; the
 * message of the last failure is kemcu_last_error(ctx). There is no CPU fallback: a missing
 * or failing GPU is reported, never worked around.
 *
 * Element encoding (the flattened KSurfaceContainer, KSurfaceContainer.cc:36-72; element
 * index = matrix row/column index):
 *   shape[i]    KEMCU_TRIANGLE | KEMCU_RECTANGLE | KEMCU_LINE_SEGMENT, or
 *               KEMCU_CONIC_SECTION | KEMCU_RING (axisymmetric; a context holds either kind,
 *               not both)
 *   boundary[i] KEMCU_DIRICHLET (value = potential, KDirichletBoundary::GetBoundaryValue)
 *               KEMCU_NEUMANN   (value = normal boundary flux, KNeumannBoundary; planar only)
 *   geom[11*i]  triangle / rectangle: A, B, P0(xyz), N1(xyz), N2(xyz)
 *               (KTriangle.hh:125-130, KRectangle.hh:132-137; P1 = P0 + A*N1, P2 = P0 + B*N2)
 *               line segment: P0(xyz), P1(xyz), diameter, 0, 0, 0, 0 (KLineSegment.hh:74-76)
 *               conic section: r0, z0, r1, z1, 0... (KConicSection.hh: P0 = (r0, 0, z0),
 *               P1 = (r1, 0, z1)); ring: r, z, 0... (KRing.hh: P = (r, 0, z)). Their integrals
 *               are KElectrostaticAnalyticConicSectionIntegrator / ...RingIntegrator, FP64
 *               whatever the precision argument; tracking, the adjoint, matrix-free Robin
 *               Hood and the band histogram take planar elements only (KEMCU_EINVAL
 *               otherwise; Robin Hood on the assembled operator takes both).
 * Units are SI; 1/(4 pi eps0) and eps0 come from kemcu_config (KEMConstants, KEMConstants.cc:11-12).
 */
#ifndef KEMCU_H
#define KEMCU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KEMCU_OK 0
#define KEMCU_EINVAL (-1)       /* invalid argument or size */
#define KEMCU_ECUDA (-2)        /* CUDA runtime / launch failure, or no usable device */
#define KEMCU_ENONFINITE (-3)   /* a result contains NaN or Inf */
#define KEMCU_ENOTCONVERGED (-4)/* solver stopped before reaching its tolerance */
#define KEMCU_ETIMEOUT (-5)     /* step/time budget exhausted (tracker) */
#define KEMCU_ENOMEM (-6)       /* device allocation failed or budget exceeded */
#define KEMCU_ESTATE (-7)       /* call out of order (e.g. no geometry set) */

enum kemcu_shape {
    KEMCU_TRIANGLE = 0,
    KEMCU_RECTANGLE = 1,
    KEMCU_LINE_SEGMENT = 2,
    KEMCU_CONIC_SECTION = 3,
    KEMCU_RING = 4
};
enum kemcu_boundary { KEMCU_DIRICHLET = 0, KEMCU_NEUMANN = 1 };
/* arithmetic form of the element integrals */
enum kemcu_precision {
    KEMCU_FP64 = 0,  /* every node in FP64: the plain form */
    KEMCU_MIXED = 1, /* cubature nodes with the FP32-class hardware reciprocal square root
                        refined by one FP64 Newton step (~1e-13 relative); RWG / analytic
                        near field and the compensated accumulation as in FP64 */
    KEMCU_FP32 = 2   /* far field in FP32: the cubature nodes of triangles and rectangles on
                        FP32 FMAs and the FP32 hardware reciprocal square root, relative to the
                        element's FP64 centre distance (~1e-7 relative per element); the RWG /
                        analytic near field, wires, the per-element set-up and the compensated
                        element sums in FP64. Field evaluation and matrix-free matvec only (the
                        tracker, the adjoint and the autotuner take FP64 and MIXED) */
};
/* which quantities a field evaluation produces (out4 = Ex, Ey, Ez, phi) */
enum kemcu_what { KEMCU_FIELD_AND_POTENTIAL = 0, KEMCU_POTENTIAL = 1, KEMCU_FIELD = 2 };
/* charge-density solve strategies */
enum kemcu_solve_mode {
    KEMCU_SOLVE_PLAIN = 0,     /* GMRES, FP64 matrix-free matvec (the reference algorithm) */
    KEMCU_SOLVE_MIXED = 1,     /* iterative refinement: inner GMRES on the MIXED matrix-free
                                  operator, FP64 matrix-free residual and correction */
    KEMCU_SOLVE_ASSEMBLED = 2, /* operator assembled once in HBM (FP64, plus an FP32 copy);
                                  inner GMRES on FP32, FP64 residual (refinement) */
    KEMCU_SOLVE_ASSEMBLED_FP64 = 3, /* GMRES on the assembled FP64 operator alone (no FP32 copy,
                                  no refinement): the plain algorithm with the same assembly,
                                  which separates the gain of assembly from that of precision */
    KEMCU_SOLVE_FP32 = 4,      /* iterative refinement, matrix-free: inner GMRES on the FP32
                                  far-field operator (KEMCU_FP32), FP64 matrix-free residual and
                                  correction; FP64-accurate charge densities */
    KEMCU_SOLVE_FFTM = 5       /* GMRES on the fast multipole operator of kemcu_fftm_configure
                                  (the operator of KKrylovChargeDensitySolver with
                                  KFastMultipoleMatrixGenerator): the residual is the FFTM
                                  operator's, whose entries differ from the direct ones by the
                                  expansion's truncation error */
};

typedef struct kemcu_ctx kemcu_ctx;

typedef struct {
    int device;                    /* CUDA device ordinal */
    double one_over_four_pi_eps0;  /* KEMConstants::OneOverFourPiEps0 (KEMConstants.cc:12) */
    double eps0;                   /* KEMConstants::Eps0 (KEMConstants.cc:11) */
    size_t assembled_budget_bytes; /* device bytes an assembled operator may take; 0 = 70% of free */
    int autotune;                  /* nonzero (default): the first field-and-potential calls of each
                                      precision and size class try the direct-sum kernel's launch
                                      shapes in turn and keep the fastest (kemcu_tune_field) */
} kemcu_config;

typedef struct {
    int iterations;          /* total Krylov iterations (all refinement steps) */
    int outer;               /* refinement steps (1 for KEMCU_SOLVE_PLAIN) */
    int fp64_matvecs;        /* FP64 operator applications */
    int low_matvecs;         /* reduced-precision operator applications */
    double rel_residual;     /* max over RHS of |b - A x| / |b|, A applied in FP64 */
    double rel_residual_estimate; /* GMRES implicit estimate |p_{j+1}| / |b| of the last cycle */
    double seconds;          /* device time of the solve */
} kemcu_solve_stats;

/* per-iteration hook, the analogue of KIterativeSolver visitors (KIterativeSolver.hh:57-134):
   return nonzero to stop the solve (KTimeTerminator-style) */
typedef int (*kemcu_iteration_callback)(void* user, int iteration, double rel_residual_estimate);

typedef struct {
    double sphere_radius;    /* electrode hit when |x| <= sphere_radius (0 disables) */
    double max_radius;       /* track leaves the volume when |x| >= max_radius (0 disables) */
} kemcu_hit_model;

enum kemcu_track_status { KEMCU_TRACK_ACTIVE = 0, KEMCU_TRACK_HIT = 1, KEMCU_TRACK_MAX_STEPS = 2,
                          KEMCU_TRACK_LEFT = 3, KEMCU_TRACK_NONFINITE = 4 };

typedef struct {
    long long steps;         /* RK8 steps taken by all tracks */
    long long field_evals;   /* field evaluations (12 per step: the 13-stage scheme's stage 10 has
                                zero weight everywhere, KSMathRK8.h:139-226, and is not evaluated) */
    int hit, max_steps, left, nonfinite, active;
    double seconds;
} kemcu_track_stats;

/* ---- context (KElectrostaticBoundaryIntegratorPolicy / use_opencl analogue,
        KIntegratingElectrostaticFieldSolver.cc:44-69) ---- */
void kemcu_default_config(kemcu_config* cfg);
int kemcu_create(kemcu_ctx** ctx, const kemcu_config* cfg);
int kemcu_destroy(kemcu_ctx* ctx);
const char* kemcu_last_error(const kemcu_ctx* ctx);
/* device milliseconds of the last call's kernels (0 if none) */
double kemcu_last_kernel_ms(const kemcu_ctx* ctx);

/* ---- geometry (KOpenCLSurfaceContainer analogue, KOpenCLSurfaceContainer.cc:10-204) ---- */
int kemcu_set_geometry(kemcu_ctx* ctx, size_t n, const int32_t* shape, const int32_t* boundary,
                       const double* geom11, const double* value);
size_t kemcu_num_elements(const kemcu_ctx* ctx);
/* charge densities (KElectrostaticBasis::GetSolution, KElectrostaticBasis.hh:22), n values */
int kemcu_set_sigma(kemcu_ctx* ctx, const double* sigma);
int kemcu_get_sigma(kemcu_ctx* ctx, double* sigma);
/* right-hand side b_i = KBoundaryIntegralVector(i) (KBoundaryIntegralVector.hh:60-78) */
int kemcu_rhs(kemcu_ctx* ctx, double* b);

/* ---- direct summation (KIntegratingFieldSolver::{Potential,ElectricField,
        ElectricFieldAndPotential}, KElectrostaticIntegratingFieldSolver.hh:261-339),
        batched over n points: P is n x 3, out4 is n x 4 (Ex, Ey, Ez, phi) ---- */
int kemcu_field(kemcu_ctx* ctx, const double* P, size_t n, double* out4, int precision, int what);
/* same with device pointers, ordered on the context stream, synchronous on return */
int kemcu_field_dev(kemcu_ctx* ctx, const double* dP, size_t n, double* dout4, int precision, int what);

/* ---- direct summation that allocates no device memory (no counterpart in the reference) ----
   For callers that cannot call cudaMalloc while they evaluate fields: a host framework that has
   given all device memory to its own pool allocator, or a loop that must not incur the implicit
   device synchronisation a cudaMalloc / cudaFree can cause while other work runs on the GPU.
   Same result as kemcu_field_dev to rounding: the points are evaluated in the caller's order
   (kemcu_field_dev re-sorts them above 4,096 points) and the element list may be split into
   fewer partial sums, so the summation order can differ. The
   element-split partial sums live in one file-scope device array of
   KEMCU_NOALLOC_SCRATCH_BYTES (8 MiB, held by every GPU that loads the library until the
   process exits); its device address is looked up once per context in kemcu_create. n may be
   at most KEMCU_NOALLOC_MAX_POINTS; larger n returns KEMCU_EINVAL. All calls share the array,
   so calls that overlap on the GPU (several contexts or threads on one device at once) race;
   calls in sequence do not, every call overwrites the part it reads. */
#define KEMCU_NOALLOC_SCRATCH_BYTES (8u << 20)
#define KEMCU_NOALLOC_MAX_POINTS (KEMCU_NOALLOC_SCRATCH_BYTES / 32u)
int kemcu_field_dev_noalloc(kemcu_ctx* ctx, const double* dP, size_t n, double* dout4, int precision, int what);

/* ---- autotuner of the direct sum's launch shape (no counterpart in the reference: the OpenCL
        plugin fixes its work-group size at build time, KOpenCLElectrostaticIntegratingFieldSolver.hh)
   The direct-sum kernel exists in kemcu_field_variant_count() launch shapes (resident CTAs per SM
   its registers are bounded for, element-ring stages: kemcu_field_variant_info); all compute the
   same operations in the same order, so every shape returns the same bits. Per context, precision
   and size class (the bit length of the point count) the library keeps the fastest shape: with
   kemcu_config.autotune set, the first field-and-potential calls of a class each run one shape
   (timed with CUDA events) until all have run; kemcu_tune_field times every shape at once on the
   caller's device points dP (n x 3; dout4 n x 4 receives the field) and records the choice, with
   the K1 time of each shape in ms (kemcu_field_variant_count() values) when ms is not NULL.
   kemcu_field_variant gives the shape chosen for n points (-1: none yet). ---- */
int kemcu_tune_field(kemcu_ctx* ctx, const double* dP, size_t n, double* dout4, int precision, int* variant,
                     float* ms);
int kemcu_field_variant(const kemcu_ctx* ctx, size_t n, int precision, int* variant);
int kemcu_field_variant_info(int variant, int* min_blocks, int* ring_stages);
int kemcu_field_variant_count(void);

/* ---- boundary-integral matrix (KBoundaryIntegralMatrix, KBoundaryIntegralMatrix.hh:16-99) ---- */
/* single entry A(i, j) = BoundaryIntegral(source j, target i) (KBoundaryIntegralMatrix.hh:31-55) */
int kemcu_matrix_element(kemcu_ctx* ctx, size_t i, size_t j, double* a);
/* y = A x for n_rhs right-hand sides (x, y: n_rhs x n), KMatrix::Multiply (KMatrix.hh:87-99);
   assembled != 0 uses (and on first use builds) the assembled operator: its FP64 copy for
   KEMCU_FP64, its FP32 copy for KEMCU_MIXED and KEMCU_FP32 */
int kemcu_matvec(kemcu_ctx* ctx, const double* x, double* y, int n_rhs, int precision, int assembled);

/* ---- charge-density solve (KSimpleIterativeKrylovSolver<double, KGeneralizedMinimalResidual>::Solve,
        KSimpleIterativeKrylovSolver.hh:139-194; KGeneralizedMinimalResidual.hh:178-337) ----
   b: n_rhs x n right-hand sides, or NULL for the boundary values (single RHS);
   x: n_rhs x n solution. For n_rhs == 1 the solution is also stored as the context's sigma. */
int kemcu_gmres(kemcu_ctx* ctx, const double* b, double* x, int n_rhs, double rel_tol, int max_iter, int mode,
                kemcu_solve_stats* stats);
void kemcu_set_iteration_callback(kemcu_ctx* ctx, kemcu_iteration_callback cb, void* user);

/* ---- Robin Hood charge-density solve (KRobinHood<double, KRobinHood_SingleThread>::Solve,
        KRobinHood.hh:61-104; KRobinHood_SingleThread.hh:59-120) ----
   Repeatedly picks the element with the largest |residual| (first index on ties), sets its
   charge density so that this residual vanishes (correction r_k / A(k, k)) and updates the
   residual with column k of the operator. Every check_interval sub-iterations (0 = n, the
   reference default) the relative residual |b - A x|_inf / |b|_inf is evaluated; the solve
   ends when it is <= rel_tol (after finishing that sub-iteration, as the reference does).
   b: n values or NULL for the boundary values; x: n values, in: initial guess (as the
   reference, A x is applied when |x|_inf > 1e-16), out: solution, also stored as the
   context's sigma. assembled != 0 reads the columns from the assembled FP64 operator (built
   on first use), else computes them on the fly. Returns KEMCU_ENOTCONVERGED after
   max_subiterations (0 = unlimited) or when the iteration callback asks to stop (it is
   called after every residual check with the check count and the relative residual). */
typedef struct {
    long long subiterations; /* single-element corrections applied */
    int iterations;          /* residual checks (KIterativeSolver::GetIteration) */
    double rel_residual;     /* |b - A x|_inf / |b|_inf at the last check */
    double seconds;          /* device time of the solve */
} kemcu_rh_stats;
int kemcu_robin_hood(kemcu_ctx* ctx, const double* b, double* x, double rel_tol, int check_interval,
                     long long max_subiterations, int assembled, kemcu_rh_stats* stats);

/* ---- batched exact-trajectory RK8 tracking in the electrostatic field (KSMathRK8::Integrate,
        Kassiopeia/Math/Include/KSMathRK8.h:45-226; KSTrajTermPropagation::Differentiate,
        KSTrajTermPropagation.cxx:25-35) ----
   state: n x 8 (t, s, x, y, z, px, py, pz), updated in place; steps: n step counters
   (in/out, tracks stop at max_steps); status: n kemcu_track_status values (in/out, only
   KEMCU_TRACK_ACTIVE tracks advance). step_budget bounds the steps of this call per track
   (<= 0: no extra bound). momentum_change (n values, in/out, may be NULL): per track, the sum over
   its steps of |p_after - p_before|, added to the values passed in (KSStep::ContinuousMomentumChange,
   which KSRoot sums into KSTrack, KSRootTrajectory.cxx:217-218, KSRoot.cxx:695-705). */
int kemcu_track_rk8(kemcu_ctx* ctx, double* state, int32_t* steps, int32_t* status, size_t n, double dt,
                    int max_steps, int step_budget, double charge, double mass, const kemcu_hit_model* hit,
                    int precision, kemcu_track_stats* stats, double* momentum_change);

/* ---- adjoint: vector-Jacobian product of the direct sum (no reference counterpart) ----
   w: n x 4 weights on (Ex, Ey, Ez, phi) at points P (n x 3); L = sum_p w_p . out_p.
   Outputs (either may be NULL):
   dsigma[N]    = dL/dsigma_j
   dvert[N x 9] = dL/d(P0, P1, P2) of element j, the three defining vertices
                  (triangle: P0, P0 + A N1, P0 + B N2; rectangle: P0, P0 + A N1, P0 + B N2),
                  within the quadrature band each (element, point) pair has; zeros for line
                  segments. precision selects the arithmetic of the dsigma sums. */
int kemcu_field_vjp(kemcu_ctx* ctx, const double* P, size_t n, const double* w, double* dsigma, double* dvert,
                    int precision);

/* ---- diagnostics (no device needed) ----
   nodes and weights of the cubature rules the kernels use, on the canonical element
   node = P0 + s (P1 - P0) + t (P2 - P0) (triangle) or P0 + s A N1 + t B N2 (rectangle):
   which 0..2 = triangle 7/12/33-point (KElectrostaticCubatureTriangleIntegrator.cc:36-268),
   3..5 = rectangle 7/12/33-point (KElectrostaticCubatureRectangleIntegrator.cc:46-290),
   6 = 4-node and 7 = 16-node Gauss-Legendre half rules (x, w, 0) on [-1, 1]
   (KElectrostaticQuadratureLineSegmentIntegrator.hh:47-80).
   out: up to 33 x 3 (s, t, w); returns the node count or KEMCU_EINVAL. */
int kemcu_rule_nodes(int which, double* out);
/* number of this library's own kernel launches on the context since it was created */
unsigned long long kemcu_launch_count(const kemcu_ctx* ctx);
/* quadrature-band histogram over all (element, point) pairs for points P (n x 3):
   counts[shape * 4 + band], band 0 = analytic (RWG / analytic wire), 1 = 33-point / 16-node,
   2 = 12-point / 4-node, 3 = 7-point; the algorithmic work of a field evaluation */
int kemcu_band_histogram(kemcu_ctx* ctx, const double* P, size_t n, long long* counts12);
/* self-test of the device-side timeout path (no counterpart in the reference): a kernel waits
   on a barrier phase that completes only when `complete` is nonzero; otherwise its bounded
   wait gives up after ~2e6 cycles and the call returns KEMCU_ETIMEOUT, as a stalled element
   pipeline would. The context stays usable either way. */
int kemcu_selftest_timeout(kemcu_ctx* ctx, int complete);
/* measured FMA throughput of the context's device, FP64 and FP32 CUDA-core pipes (TFLOP/s,
   2 flops per FMA), from independent dependent-FMA chains */
int kemcu_fma_peak(kemcu_ctx* ctx, double* fp64_tflops, double* fp32_tflops);

/* ---- fast multipole method (FFTM) for the field of planar elements ----
   The reference's fast-multipole field solver (KFMElectrostaticFastMultipoleFieldSolver.cc:47-163
   with the tree of KFMElectrostaticTreeConstructor.hh:44-87): a cubic tree over the world cube
   (root divided top_level_divisions times per dimension, every further level `divisions` times,
   down to level maximum_tree_depth); every element is owned by the deepest cell that contains
   its bounding ball's centre and whose bounding ball, scaled by insertion_ratio, contains the
   element's bounding ball (KFMInsertionCondition.hh:52-78); multipole moments of degree `degree`
   about the owner cells, M2M up, M2L between the cells of each level that are not neighbours
   (within `zeromask` cells) but whose parents are, L2L down; a point is the local expansion of
   its leaf plus the direct sum over the elements owned by the neighbours of its leaf's
   ancestors. Divisions 2..8 and zeromask 1..3; the M2L operators (one per offset of the
   interaction lists, ((2 (zeromask+1) divisions - 1)^3 - (2 zeromask + 1)^3) matrices of
   (degree+1)^4 doubles) must fit in 8 GB. */
typedef struct {
    int degree;                     /* expansion degree p, 0..15 (KFMElectrostaticParameters::degree) */
    int top_level_divisions;        /* divisions of the root per dimension, 1..8 */
    int divisions;                  /* divisions of every further level per dimension, 2..8 (2) */
    int zeromask;                   /* neighbour order: cells within it are summed directly, 1..3 (1) */
    int maximum_tree_depth;         /* level of the leaves, 1..10 */
    double insertion_ratio;         /* insertion condition's ratio (4/3) */
    double region_expansion_factor; /* world cube side over the elements' extent (1.1) */
    double world_center[3];         /* explicit world cube, used when world_length > 0 */
    double world_length;
    int near_analytic;              /* direct pairs by the analytic integrals (1, as the reference's
                                       fast-multipole field solver: KEBIFactory::MakeAnalytic) or
                                       by the numeric policy of kemcu_field (0) */
} kemcu_fftm_params;
void kemcu_fftm_default_params(kemcu_fftm_params* prm);
/* builds the tree for the context's (planar) geometry; the charge densities are read at each
   evaluation. Replaces the previous tree. */
int kemcu_fftm_configure(kemcu_ctx* ctx, const kemcu_fftm_params* prm);
/* field and potential at n points (host or device buffers, out4 as kemcu_field); points outside
   the world cube are summed directly, as the reference falls back to its direct solver
   (KFMElectrostaticFastMultipoleFieldSolver.cc:145-160) */
int kemcu_fftm_field(kemcu_ctx* ctx, const double* P, size_t n, double* out4, int what);
int kemcu_fftm_field_dev(kemcu_ctx* ctx, const double* dP, size_t n, double* dout4, int what);
/* y = A x with the fast multipole operator (KFastMultipoleMatrixGenerator, KFastMultipoleMatrixGenerator.cc:
   23-41): the local expansion of the leaf holding each row's collocation point (potential, or
   field along the normal for a Neumann row) plus the direct entries, by the numeric policy as
   kemcu_matvec, of the elements owned by the neighbours of that leaf's ancestors; x, y n_rhs x n.
   The first product of a tree computes the near part's entries and keeps them on the device (as
   the reference keeps the sparse part of its matrix) when they fit a quarter of the free device
   memory and at most 8 GB; otherwise every product computes them. */
int kemcu_fftm_matvec(kemcu_ctx* ctx, const double* x, double* y, int n_rhs);
/* tree summary: world4 = world cube centre and side; counts = {cells with moments, elements
   owned per level 0..maximum_tree_depth} (counts has room for 2 + maximum_tree_depth ints) */
int kemcu_fftm_info(const kemcu_ctx* ctx, double* world4, int* counts);
/* a second tree whose operator serves as the implicit Krylov preconditioner's matrix
   (KEMCU_SOLVE_FFTM as kemcu_krylov_params.preconditioner_mode): the solver's parameters with
   degree = preconditioner_degree for the reference's "implicit_krylov" (a lower-degree
   operator on the same tree, KFMElectrostaticFastMultipoleBoundaryValueSolver.cc:726-745), or
   the preconditioner_electrostatic_parameters for "independent_implicit_krylov" (:831-848).
   Degree 0..15 (0, the reference's default preconditioner_degree, keeps the monopoles only).
   Replaces the previous preconditioner tree. */
int kemcu_fftm_configure_preconditioner(kemcu_ctx* ctx, const kemcu_fftm_params* prm);

/* ---- Krylov charge-density solves with restarts and right preconditioners: the solver
        dispatch of KKrylovSolverFactory.hh:110-150 and of the fast-multipole boundary-value
        solver (KFMElectrostaticFastMultipoleBoundaryValueSolver.cc:189-233) ----
   GMRES as KGeneralizedMinimalResidual / KPreconditionedGeneralizedMinimalResidual
   (KPreconditionedGeneralizedMinimalResidual.hh: right preconditioning, the preconditioned basis
   kept when the preconditioner is not stationary) and BiCGStab as
   KBiconjugateGradientStabilized / KPreconditionedBiconjugateGradientStabilized; the iteration
   loop of KSimpleIterativeKrylovSolver.hh:139-194 / KPreconditionedIterativeKrylovSolver.hh
   (convergence when the solver's residual norm over |b| is <= tolerance; a restart every
   iterations_between_restarts iterations, KIterativeKrylovRestartCondition.hh, recomputes the
   residual b - A x and starts a new Krylov space from the current solution). Preconditioners:
   Jacobi (KJacobiPreconditioner.hh: 1 / A(i, i)) and implicit Krylov
   (KImplicitKrylovPreconditioner.hh: an inner GMRES from zero on the preconditioner's operator to
   preconditioner_tolerance, at most max_preconditioner_iterations iterations).
   b: n_rhs x n or NULL (boundary values, one RHS); x: n_rhs x n solution from x0 = 0 (also the
   context's sigma for one RHS). Stats: iterations = Krylov iterations, outer = cycles (1 +
   restarts), fp64_matvecs = applications of the system's operator, low_matvecs = of the
   preconditioner's, rel_residual = max over RHS of |b - A x| / |b| recomputed at the end with the
   system's operator, rel_residual_estimate = the solver's own residual norm over |b|. Returns
   KEMCU_ENOTCONVERGED when the solver's residual norm (for the refinement modes the FP64 one) is
   above the tolerance at the end. For the refinement modes, outer counts the refinement steps,
   fp64_matvecs the FP64 products and low_matvecs the inner solves' and the preconditioner's. */
enum kemcu_krylov_solver { KEMCU_KRYLOV_GMRES = 0, KEMCU_KRYLOV_BICGSTAB = 1 };
enum kemcu_preconditioner { KEMCU_PRECON_NONE = 0, KEMCU_PRECON_JACOBI = 1, KEMCU_PRECON_IMPLICIT_KRYLOV = 2 };
typedef struct {
    int solver;                         /* kemcu_krylov_solver ("solver_name": gmres, bicgstab) */
    int mode;                           /* kemcu_solve_mode: KEMCU_SOLVE_PLAIN (FP64 matrix-free),
                                           KEMCU_SOLVE_ASSEMBLED_FP64 or KEMCU_SOLVE_FFTM solve that
                                           operator; KEMCU_SOLVE_MIXED, _ASSEMBLED and _FP32 refine
                                           as kemcu_gmres does (FP64 residuals, corrections from
                                           inner solves on the reduced operator), the solver, its
                                           restarts and the preconditioner applying to the inner
                                           solves */
    double tolerance;                   /* "tolerance" */
    int max_iterations;                 /* "max_iterations" (bounds the GMRES basis kept on the device) */
    int iterations_between_restarts;    /* "iterations_between_restarts"; 0 = never */
    int preconditioner;                 /* kemcu_preconditioner ("preconditioner") */
    int preconditioner_mode;            /* operator of the implicit Krylov preconditioner:
                                           KEMCU_SOLVE_FFTM = the tree of kemcu_fftm_configure_preconditioner;
                                           KEMCU_SOLVE_FP32 / KEMCU_SOLVE_MIXED = the FP32 / MIXED
                                           matrix-free operator; KEMCU_SOLVE_ASSEMBLED = the FP32 copy
                                           of the assembled operator; KEMCU_SOLVE_PLAIN /
                                           KEMCU_SOLVE_ASSEMBLED_FP64 = the FP64 one */
    double preconditioner_tolerance;    /* "preconditioner_tolerance" */
    int max_preconditioner_iterations;  /* "max_preconditioner_iterations" */
} kemcu_krylov_params;
/* gmres, KEMCU_SOLVE_PLAIN, tolerance 1e-8, 500 iterations, no restart, no preconditioner;
   implicit Krylov defaults: KEMCU_SOLVE_FFTM, tolerance 0.01, 30 iterations (the reference's
   example configurations) */
void kemcu_krylov_default_params(kemcu_krylov_params* prm);
int kemcu_krylov_solve(kemcu_ctx* ctx, const double* b, double* x, int n_rhs, const kemcu_krylov_params* prm,
                       kemcu_solve_stats* stats);
/* multipole moments of every element of the context, for unit total charge, about the origins
   (n x 3), as KFMElectrostaticMultipoleCalculatorAnalytic::ConstructExpansion gives them:
   out n x (degree+1)^2 complex (re, im) in the index l(l+1)+m */
int kemcu_fm_moments(kemcu_ctx* ctx, int degree, const double* origins, double* out);
/* potential and field of a local expansion about `origin` (coefficients for m >= 0,
   (degree+1)(degree+2)/2 complex in the index l(l+1)/2+m, the reference's
   KFMElectrostaticLocalCoefficientSet layout) at n points, times 1 / (4 pi eps0), as
   KFMElectrostaticLocalCoefficientFieldCalculator evaluates it; out4 as kemcu_field */
int kemcu_fm_local_field(kemcu_ctx* ctx, int degree, const double* origin, const double* coeff, size_t n,
                         const double* P, double* out4);
/* the translation response of `kind` (0 M2M, 1 M2L, 2 L2L) between two origins, as the
   reference's KFMResponseKernel_3DLaplace* GetResponseFunction gives it: out
   (degree+1)^2 x (degree+1)^2 complex, [target][source]; host arithmetic (no device) */
int kemcu_fm_response(int kind, int degree, const double* source_origin, const double* target_origin, double* out);

#ifdef __cplusplus
}
#endif

#endif /* KEMCU_H */
