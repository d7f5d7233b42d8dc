/* selfgpu.h -- C ABI of libselfgpu, the B200 (sm_100a) DGSEM tendency engine
 * for SELF's 2-D Model2D path.
 *
 * Two groups of entry points:
 *
 *  1. Drop-in replacements for SELF's HIP wrappers.  Same symbol names, same
 *     argument lists and the same "pointer to device pointer" convention that
 *     SELF's Fortran interfaces produce (TYPE(c_ptr) without VALUE arrives as
 *     real**, INTEGER(C_INT),VALUE as int).  `real` is double: these are the
 *     FP64 build (-DDOUBLE_PRECISION) of the reference.  Like the reference
 *     they return void, launch on the legacy default stream and do not
 *     synchronise; a launch failure is recorded and can be read with
 *     selfgpu_last_error().  Layouts are SELF's Fortran column-major layouts
 *     (src/hip/SELF_HIP_Macros.h:20-38 of the reference).
 *
 *  2. Fused entry points (selfgpu_*) that return an int status
 *     (SELFGPU_OK == 0).  They run a whole CalculateTendency or whole
 *     Williamson RK3 steps of LinearShallowWater, ShallowWater or
 *     CompressibleIdealGas2D as one kernel per RK stage, on buffers that the
 *     caller owns (the Fortran hfReal device arrays); only the engine's own
 *     face-trace cache is allocated by the library, inside the handle.
 *
 * Every reference citation below is file:line inside the SELF repository.
 */
#ifndef SELFGPU_H
#define SELFGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- constants */
/* quadrature ids, src/SELF_Constants.f90:78-84 */
#define SELFGPU_GAUSS 1
#define SELFGPU_GAUSS_LOBATTO 2
#define SELFGPU_UNIFORM 5
/* boundary condition ids, src/hip/SELF_HIP_Macros.h:40-49 */
#define SELFGPU_BC_PRESCRIBED 100
#define SELFGPU_BC_RADIATION 101
#define SELFGPU_BC_NONORMALFLOW 102
/* models */
#define SELFGPU_MODEL_LSW 1 /* LinearShallowWater, src/models/SELF_LinearShallowWater.f90 */
#define SELFGPU_MODEL_SW 2  /* ShallowWater,       src/models/SELF_ShallowWater.f90 */
#define SELFGPU_MODEL_CIG 3 /* CompressibleIdealGas2D, src/models/SELF_CompressibleIdealGas2D.f90 */
/* arithmetic forms of the fused path */
#define SELFGPU_FP64 0       /* plain FP64, production build: multiply-add contraction and reciprocal
                                products (within FP64 round-off of the reference CPU path) */
#define SELFGPU_FP32_BULK 1  /* FP32 flux/divergence, FP64 metrics/sources/RK accumulation */
#define SELFGPU_FP64_REF 2   /* plain FP64 with the reference's roundings: no contraction, the
                                reference's divisions and order; equals the FP64 CPU path bit for bit */
/* largest polynomial degree the fused kernels are instantiated for */
#define SELFGPU_MAX_N 7
/* status codes */
#define SELFGPU_OK 0
#define SELFGPU_ERR_ARG 1      /* bad argument (null pointer, size, degree, model) */
#define SELFGPU_ERR_MESH 2     /* malformed sideInfo rejected before launch */
#define SELFGPU_ERR_CUDA 3     /* CUDA launch or runtime error */
#define SELFGPU_ERR_STATE 4    /* handle not fully bound */
#define SELFGPU_ERR_NONFINITE 5/* NaN/Inf found by selfgpu_model2d_check_finite */
#define SELFGPU_ERR_TIMEOUT 6  /* a bounded device wait ran out */

/* Message for the calling thread's most recent error ("" when none). */
const char* selfgpu_last_error(void);

/* ====================================================== 1. drop-in wrappers */

/* -- Lagrange: src/SELF_Lagrange.f90 interfaces, src/hip/SELF_Lagrange.cpp -- */
/* replaces ScalarGridInterp_2D_gpu_wrapper, SELF_Lagrange.cpp:107 */
void ScalarGridInterp_2D_gpu_wrapper(double** iMatrix, double** f, double** fInterp, int N, int M, int nVar,
                                     int nEl);
/* replaces VectorGridInterp_2D_gpu_wrapper, SELF_Lagrange.cpp:140 */
void VectorGridInterp_2D_gpu_wrapper(double** iMatrix, double** f, double** fInterp, int N, int M, int nVar,
                                     int nEl);
/* replaces ScalarBoundaryInterp_2D_gpu_wrapper, SELF_Lagrange.cpp:395 */
void ScalarBoundaryInterp_2D_gpu_wrapper(double** bMatrix, double** f, double** fBound, int N, int nVar,
                                         int nEl);
/* replaces VectorBoundaryInterp_2D_gpu_wrapper, SELF_Lagrange.cpp:424 */
void VectorBoundaryInterp_2D_gpu_wrapper(double** bMatrix, double** f, double** fBound, int N, int nVar,
                                         int nEl);
/* replaces TensorBoundaryInterp_2D_gpu_wrapper, SELF_Lagrange.cpp:483 */
void TensorBoundaryInterp_2D_gpu_wrapper(double** bMatrix, double** f, double** fBound, int N, int nVar,
                                         int nEl);
/* replaces VectorGradient_2D_gpu_wrapper, SELF_Lagrange.cpp:730 */
void VectorGradient_2D_gpu_wrapper(double** dMatrix, double** f, double** df, int N, int nVar, int nEl);
/* replaces VectorDGDivergence_2D_gpu_wrapper, SELF_Lagrange.cpp:827 */
void VectorDGDivergence_2D_gpu_wrapper(double** dgMatrix, double** bMatrix, double** qWeights, double** f,
                                       double** bf, double** df, int N, int nVar, int nEl);

/* -- Data / Geometry: src/hip/SELF_Data.cpp, src/hip/SELF_Geometry.cpp -- */
/* replaces Determinant_Tensor2D_gpu_wrapper, SELF_Data.cpp:74 */
void Determinant_Tensor2D_gpu_wrapper(double** tensor, double** detTensor, int N, int nVar, int nEl);
/* replaces CalculateContravariantBasis_SEMQuad_gpu_wrapper, SELF_Geometry.cpp:96 */
void CalculateContravariantBasis_SEMQuad_gpu_wrapper(double** dxds, double** dsdx, int N, int nEl);
/* replaces AdjustBoundaryContravariantBasis_SEMQuad_gpu_wrapper, SELF_Geometry.cpp:123 */
void AdjustBoundaryContravariantBasis_SEMQuad_gpu_wrapper(double** dsdx, double** J, int N, int nEl);

/* -- MappedData: src/SELF_MappedData.f90:162-600, src/hip/SELF_MappedData.cpp -- */
/* replaces GradientBR_MappedScalar2D_gpu_wrapper, SELF_MappedData.cpp:164 */
void GradientBR_MappedScalar2D_gpu_wrapper(double** scalar, double** avgBoundary, double** dsdx, double** jacobian,
                                           double** nHat, double** nScale, double** gradF, double** dgMatrix,
                                           double** bMatrix, double** qWeights, int N, int nVar, int nEl);
/* replaces GradientSF_MappedScalar2D_gpu_wrapper, SELF_MappedData.cpp:203 */
void GradientSF_MappedScalar2D_gpu_wrapper(double** scalar, double** dsdx, double** jacobian, double** gradF,
                                           double** dMatrix, int N, int nVar, int nEl);
/* replaces JacobianWeight_MappedScalar2D_gpu_wrapper, SELF_MappedData.cpp:223 */
void JacobianWeight_MappedScalar2D_gpu_wrapper(double** scalar, double** jacobian, int N, int nVar, int nEl);
/* replaces ContravariantProjection_MappedVector2D_gpu_wrapper, SELF_MappedData.cpp:422 */
void ContravariantProjection_MappedVector2D_gpu_wrapper(double** vector, double** dsdx, int N, int nVar, int nEl);
/* replaces JacobianWeight_MappedVector2D_gpu_wrapper, SELF_MappedData.cpp:466 */
void JacobianWeight_MappedVector2D_gpu_wrapper(double** vector, double** jacobian, int N, int nVar, int nEl);
/* replaces SideExchange_MappedScalar2D_gpu_wrapper, SELF_MappedData.cpp:943 */
void SideExchange_MappedScalar2D_gpu_wrapper(double** extBoundary, double** boundary, int** sideInfo,
                                             int** elemToRank, int rankId, int offset, int N, int nVar, int nEl);
/* replaces SideExchange_MappedVector2D_gpu_wrapper, SELF_MappedData.cpp:982 */
void SideExchange_MappedVector2D_gpu_wrapper(double** extBoundary, double** boundary, int** sideInfo,
                                             int** elemToRank, int rankId, int offset, int N, int nVar, int nEl);
/* replaces BassiRebaySides_MappedScalar2D_gpu_wrapper, SELF_MappedData.cpp:1255 */
void BassiRebaySides_MappedScalar2D_gpu_wrapper(double** avgBoundary, double** boundary, double** extBoundary,
                                                int N, int nVar, int nEl);

/* -- Model2D: src/SELF_Model2D.f90:73-138, src/hip/SELF_Model2D.cpp -- */
/* replaces UpdateGRK_Model2D_gpu_wrapper, SELF_Model2D.cpp:153 */
void UpdateGRK_Model2D_gpu_wrapper(double** grk, double** solution, double** dSdt, double rk_a, double rk_g,
                                   double dt, int nWork, int N, int nVar, int nEl);
/* replaces UpdateSolution_Model2D_gpu_wrapper, SELF_Model2D.cpp:172 */
void UpdateSolution_Model2D_gpu_wrapper(double** solution, double** dSdt, double dt, int N, int nVar, int nEl);
/* replaces CalculateDSDt_Model2D_gpu_wrapper, SELF_Model2D.cpp:192 */
void CalculateDSDt_Model2D_gpu_wrapper(double** fluxDivergence, double** source, double** dSdt, int N, int nVar,
                                       int nEl);

/* -- LinearShallowWater: src/models/SELF_LinearShallowWater.f90:53-97, models/hip/SELF_LinearShallowWater.cpp -- */
/* replaces SetBoundaryCondition_LinearShallowWater_gpu_wrapper, SELF_LinearShallowWater.cpp:48
 * (follows the CPU reflection (n_y^2 - n_x^2), SELF_LinearShallowWater.f90:336) */
void SetBoundaryCondition_LinearShallowWater_gpu_wrapper(double** solution, double** extBoundary, double** nHat,
                                                         int** sideInfo, int N, int nVar, int nEl);
/* replaces Source_LinearShallowWater_gpu_wrapper, SELF_LinearShallowWater.cpp:73 */
void Source_LinearShallowWater_gpu_wrapper(double** source, double** solution, double** f, int N, int nVar, int nEl);
/* replaces Flux_LinearShallowWater_gpu_wrapper, SELF_LinearShallowWater.cpp:102 */
void Flux_LinearShallowWater_gpu_wrapper(double** flux, double** solution, double** H, double g, int N, int nVar,
                                         int nEl);
/* replaces RiemannSolver_LinearShallowWater_gpu_wrapper, SELF_LinearShallowWater.cpp:141 */
void RiemannSolver_LinearShallowWater_gpu_wrapper(double** flux, double** solution, double** extBoundary, double** H,
                                                  double** nHat, double** nScale, double g, int N, int nVar,
                                                  int nEl);

/* -- ShallowWater (nonlinear).  The reference has no device path for this model
 * (its GPU calls are commented out, src/models/SELF_ShallowWater.f90:293-303,
 * :351-360, :392-399, :463-475); these follow the Fortran interfaces those
 * comments name, extended with the fields the CPU path reads. -- */
/* CPU SetBoundaryCondition_ShallowWater, SELF_ShallowWater.f90:284-343 */
void SetBoundaryCondition_ShallowWater_gpu_wrapper(double** solution, double** extBoundary, double** topoBoundary,
                                                   double** nHat, int** sideInfo, int N, int nVar, int nEl);
/* CPU Source_ShallowWater, SELF_ShallowWater.f90:345-384 */
void Source_ShallowWater_gpu_wrapper(double** source, double** solution, double** gradH, double fCori, double g,
                                     int N, int nVar, int nEl);
/* CPU Flux_ShallowWater, SELF_ShallowWater.f90:386-449 (velocity = PreTendency output) */
void Flux_ShallowWater_gpu_wrapper(double** flux, double** solution, double** velocity, double g, int N, int nVar,
                                   int nEl);
/* CPU RiemannSolver_ShallowWater, SELF_ShallowWater.f90:451-529 */
void RiemannSolver_ShallowWater_gpu_wrapper(double** flux, double** solution, double** extBoundary,
                                            double** velocity, double** extVelocity, double** nHat,
                                            double** nScale, double g, int N, int nVar, int nEl);
/* CPU PreTendency_ShallowWater velocity step, SELF_ShallowWater.f90:190-239 (without the exchange) */
void PreTendency_ShallowWater_gpu_wrapper(double** solution, double** solutionBoundary, double** velocity,
                                          double** velocityBoundary, int N, int nVar, int nEl);

/* -- CompressibleIdealGas2D: src/models/SELF_CompressibleIdealGas2D.f90:149-257,
 *    models/hip/SELF_CompressibleIdealGas2D.cpp.  These follow the CPU
 *    branches (hazards: FP64 sound speed, rhoKE = 0.5(rhoU u + rhoV v)). -- */
/* replaces Source_CompressibleIdealGas2D_gpu_wrapper, SELF_CompressibleIdealGas2D.cpp:28.  The
 * reference wrapper receives no drag field; like the reference device kernel
 * this one applies gravity only.  The fused path applies gravity and drag. */
void Source_CompressibleIdealGas2D_gpu_wrapper(double** source, double** solution, double** environmentalsGradient,
                                               int N, int nVar, int nEl);
/* replaces Flux_CompressibleIdealGas2D_gpu_wrapper, SELF_CompressibleIdealGas2D.cpp:95 */
void Flux_CompressibleIdealGas2D_gpu_wrapper(double** flux, double** solution, double** primitive, int N, int nVar,
                                             int nEl);
/* replaces NaiveLLF_CompressibleIdealGas2D_gpu_wrapper, SELF_CompressibleIdealGas2D.cpp:190 */
void NaiveLLF_CompressibleIdealGas2D_gpu_wrapper(double** flux, double** solution, double** extSolution,
                                                 double** primitive, double** extPrimitive, double** diagnostics,
                                                 double** extDiagnostics, double** nHat, double** nScale, int N,
                                                 int nVar, int nDiag, int nEl);
/* replaces SetBoundaryCondition_CompressibleIdealGas2D_gpu_wrapper, SELF_CompressibleIdealGas2D.cpp:286 */
void SetBoundaryCondition_CompressibleIdealGas2D_gpu_wrapper(
    double** solution, double** extSolution, double** prescribedSolution, double** primitive, double** extPrimitive,
    double** prescribedPrimitive, double** diagnostics, double** extDiagnostics, double** prescribedDiagnostics,
    double** nHat, int** sideInfo, int N, int nVar, int nDiag, int nEl);
/* replaces CalculateDiagnostics_CompressibleIdealGas2D_gpu_wrapper, SELF_CompressibleIdealGas2D.cpp:363 */
void CalculateDiagnostics_CompressibleIdealGas2D_gpu_wrapper(double** solution, double** diagnostics,
                                                             double expansionFactor, double R, int N, int nVar,
                                                             int nDiag, int nEl);
/* replaces ConservativeToPrimitive_CompressibleIdealGas2D_gpu_wrapper, SELF_CompressibleIdealGas2D.cpp:402 */
void ConservativeToPrimitive_CompressibleIdealGas2D_gpu_wrapper(double** solution, double** primitive,
                                                                double expansionFactor, int N, int nVar, int nEl);
/* replaces ConservativeToEntropy_CompressibleIdealGas2D_gpu_wrapper, SELF_CompressibleIdealGas2D.cpp:442 */
void ConservativeToEntropy_CompressibleIdealGas2D_gpu_wrapper(double** solution, double** entropy,
                                                              double expansionFactor, int N, int nVar, int nEl);

/* ========================================================= 2. host set-up */

/* Nodes and weights, src/SELF_Quadrature.f90:59-116 (LegendreQuadrature). */
int selfgpu_legendre_quadrature(int N, int type, double* nodes, double* weights);

/* Lagrange%Init host arrays, src/SELF_Lagrange.f90:521-615.  Layouts:
 * iMatrix(0:N,0:M), dMatrix(0:N,0:N), dgMatrix(0:N,0:N), bMatrix(0:N,0:1). */
int selfgpu_lagrange_init(int N, int controlNodeType, int M, int targetNodeType, double* controlPoints,
                          double* targetPoints, double* bWeights, double* qWeights, double* iMatrix,
                          double* dMatrix, double* dgMatrix, double* bMatrix);

/* Structured nx*ny quadrilateral mesh on [x0,x1]x[y0,y1] (nGeo = 1) in the
 * layout Mesh2D%Read_HOPr produces (src/SELF_Mesh.f90:852-1016):
 * nodeCoords(1:2,0:1,0:1,nEl), globalNodeIDs(0:1,0:1,nEl), sideInfo(1:5,1:4,nEl).
 * Periodic directions connect through bcid = 0; perturbation moves interior
 * nodes by perturbation*h*sin(2 pi x)sin(2 pi y); rotation (optional, nEl
 * entries) relabels an element's corners by quarter turns.  A periodic
 * direction may be one element wide (the element is then its own neighbour
 * across it); rotated elements need two or more there (SELFGPU_ERR_ARG). */
int selfgpu_mesh2d_structured(int nx, int ny, double x0, double x1, double y0, double y1, int periodicX,
                              int periodicY, double perturbation, int bcid, const int* rotation,
                              double* nodeCoords, int* globalNodeIDs, int* sideInfo);

/* Host check of sideInfo (neighbour ids, sides, flips); SELFGPU_ERR_MESH if malformed. */
int selfgpu_validate_side_info(const int* sideInfo, int nEl);

/* SEMQuad%GenerateFromMesh on the device (src/SELF_Geometry.f90:393-552):
 * from device nodeCoords (nGeo = 1) and the model's Lagrange matrices (host
 * pointers: iMatrix of the mesh-to-model interpolant (0:1,0:N), dMatrix,
 * bMatrix) fill the device arrays x(2,P,P,1,nEl), dxds/dsdx (2,2,P,P,1,nEl),
 * J(P,P,1,nEl), dsdxBoundary (2,2,P,1,4,nEl), JBoundary(P,1,4,nEl),
 * nHat(2,P,1,4,nEl), nScale(P,1,4,nEl).  Any output pointer may be NULL
 * except those the later ones depend on internally (handled with scratch). */
int selfgpu_semquad_generate(int N, int nEl, const double* nodeCoords_d, const double* meshToModel_iMatrix,
                             const double* dMatrix, const double* bMatrix, double* x_d, double* dxds_d,
                             double* dsdx_d, double* J_d, double* dsdxBoundary_d, double* JBoundary_d,
                             double* nHat_d, double* nScale_d, void* stream);

/* ========================================================= 3. fused engine */

typedef struct selfgpu_model2d selfgpu_model2d;

/* Create an engine for `model` (SELFGPU_MODEL_*), degree N (1..SELFGPU_MAX_N),
 * nEl elements, arithmetic form SELFGPU_FP64, SELFGPU_FP64_REF or SELFGPU_FP32_BULK, on `stream`
 * (a cudaStream_t, NULL = legacy default stream).  Mirrors Model2D%Init
 * (src/SELF_Model2D.f90:142-178) minus the buffers the caller already owns. */
int selfgpu_model2d_create(selfgpu_model2d** out, int model, int N, int nEl, int form, void* stream);
int selfgpu_model2d_destroy(selfgpu_model2d* m);

/* Operator matrices from Lagrange%Init (host pointers, copied into the handle):
 * dgMatrix(0:N,0:N), bMatrix(0:N,0:1), qWeights(0:N). */
int selfgpu_model2d_set_interp(selfgpu_model2d* m, const double* dgMatrix, const double* bMatrix,
                               const double* qWeights);

/* Geometry (device pointers, caller owned): dsdx interior (2,2,P,P,1,nEl),
 * J interior (P,P,1,nEl), nHat boundary (2,P,1,4,nEl), nScale boundary
 * (P,1,4,nEl), sideInfo (5,4,nEl) on the device and a host copy of it, which
 * is validated here (SELFGPU_ERR_MESH on a malformed record). */
int selfgpu_model2d_set_geometry(selfgpu_model2d* m, const double* dsdx, const double* J, const double* nHat,
                                 const double* nScale, const int* sideInfo_d, const int* sideInfo_h);

/* Model state (device, caller owned): solution interior (P,P,nVar,nEl) and
 * the RK register workSol of the same shape (zero it before the first step;
 * the reference never uploads it, hazard H21).  The SELFGPU_FP32_BULK form
 * keeps its RK register in FP32 in engine memory (zeroed here and by
 * selfgpu_model2d_invalidate) and neither reads nor writes workSol; its
 * solution update uses each stage's FP64 register value before rounding. */
int selfgpu_model2d_set_state(selfgpu_model2d* m, double* solution, double* workSol);

/* Model-specific device fields (caller owned), by name:
 *  LSW: "H" interior (P,P,1,nEl), "H.boundary" (P,1,4,nEl), "fCori" interior
 *  SW : "topography.boundary" (P,1,4,nEl), "gradTopography" (2,P,P,1,nEl),
 *       "topography" (P,P,1,nEl; read by selfgpu_model2d_entropy only)
 *  CIG: "environmentalsGradient" (2,P,P,2,nEl), "environmentals" (P,P,2,nEl),
 *       "prescribedSolution.boundary", "prescribedPrimitive.boundary",
 *       "prescribedDiagnostics.boundary" (P,4,4,nEl each)
 *  any: "elementDt" (nEl) -- a time step per element, used by
 *       selfgpu_model2d_rk3 instead of its dt argument (ensembles of
 *       independent instances batched into one handle)
 * A field never set reads as zero. */
int selfgpu_model2d_set_field(selfgpu_model2d* m, const char* name, const double* ptr);

/* Scalar parameters: g and fCori (LSW/SW), expansion factor Cp/Cv and R (CIG). */
int selfgpu_model2d_set_params(selfgpu_model2d* m, double g, double fCori, double expansionFactor, double R);

/* Declare that the solution was written outside the engine (SetSolution and
 * the like): the next tendency or step rebuilds the face-trace cache from it. */
int selfgpu_model2d_invalidate(selfgpu_model2d* m);

/* One CalculateTendency_Model2D (src/SELF_Model2D.f90:816-859): dSdt (device,
 * (P,P,nVar,nEl)) = source - weak-form flux divergence, solution unchanged. */
int selfgpu_model2d_tendency(selfgpu_model2d* m, double* dSdt);

/* nSteps Williamson low-storage RK3 steps of size dt
 * (LowStorageRK3_timeIntegrator, src/SELF_Model.f90:704-732, stepped by
 * count): per stage one fused kernel does tendency + UpdateGRK3.  Steps are
 * replayed from a captured CUDA graph after the first call. */
int selfgpu_model2d_rk3(selfgpu_model2d* m, double dt, int nSteps);

/* Wait for the engine's stream; returns the first pending CUDA error. */
int selfgpu_model2d_sync(selfgpu_model2d* m);

/* CalculateEntropy of the bound model on the device, returned on the host
 * (the stream is synchronised): LSW src/models/SELF_LinearShallowWater.f90:171-216,
 * SW src/models/SELF_ShallowWater.f90:149-188 (reads the interior field
 * "topography"), CIG src/models/SELF_CompressibleIdealGas2D.f90:782-823 (p
 * formed from the current solution; the reference reads the primitive field
 * of its last PreTendency).  Per-element sums in the reference's node order,
 * then a fixed-order tree over the elements. */
int selfgpu_model2d_entropy(selfgpu_model2d* m, double* entropy);

/* Integral_MappedScalar2D (src/SELF_MappedData.f90:1270-1311): the sum of
 * f(i,j,iVar,e) J(i,j,e) w_i w_j over the mesh for a device field interior
 * (P,P,nVar,nEl) and device J (P,P,1,nEl), host qWeights (0:N); the result on
 * the host (the stream is synchronised).  The reference integrates variable 4
 * (hard-coded); iVar (1-based) chooses it here. */
int selfgpu_integral_mapped_scalar2d(const double* interior, int iVar, int nVar, const double* J,
                                     const double* qWeights, int N, int nEl, double* result, void* stream);

/* Scan the solution for NaN/Inf on the device (SELFGPU_ERR_NONFINITE if any). */
int selfgpu_model2d_check_finite(selfgpu_model2d* m);

/* Number of kernel launches the engine has issued (for accounting), and how
 * many of them ran the persistent bulk-copy kernel. */
long long selfgpu_model2d_launch_count(const selfgpu_model2d* m);
long long selfgpu_model2d_persistent_launch_count(const selfgpu_model2d* m);

/* Kernel choice: persistent = 1 (default) uses the warp-specialised kernel
 * that streams elements through shared memory with bulk asynchronous copies
 * wherever it applies (even P, 16-byte aligned buffers); 0 forces the
 * one-CTA-per-element-group kernel. */
int selfgpu_model2d_set_kernel(selfgpu_model2d* m, int persistent);

/* Opt-in (enable = 1): selfgpu_model2d_rk3 runs all 3 nSteps RK stages as
 * ONE cooperative launch (k_fused_steps: the per-element stage body, then a
 * grid barrier before the next stage reads the traces other CTAs wrote) when
 * the mesh's element groups fit one wave of resident CTAs -- small,
 * launch-latency bound meshes such as the 10x10 gravity-wave release.  Larger
 * meshes, a bound closure or halo fall back to graph-replayed steps.  The
 * barrier waits are bounded like the persistent kernel's (set_wait_limit;
 * SELFGPU_ERR_TIMEOUT from sync). */
int selfgpu_model2d_set_multistep(selfgpu_model2d* m, int enable);

/* enable = 1 (the default for the SELFGPU_FP64 and SELFGPU_FP32_BULK forms;
 * 0 for SELFGPU_FP64_REF): selfgpu_model2d_rk3 runs all 3 nSteps RK stages in
 * ONE cooperative launch of the persistent bulk-copy kernel (one CTA per SM)
 * where it applies: N = 7, no closure, no halo, and a mesh that gives every
 * consumer group three to 24 elements per stage (4 440 to 35 520 elements
 * on 148 SMs for FP64 CompressibleIdealGas2D, 5 328 to 42 624 for the
 * production FP64 ShallowWater models, 6 216 to 49 728 in the FP32-bulk form;
 * on larger meshes the saved per-launch costs are too small to measure).
 * Each group runs the same elements in every stage and copies the next
 * stage's first elements ahead across the stage boundary; a stage-end
 * counter orders only the neighbour-trace reads (bounded waits as in
 * set_wait_limit; SELFGPU_ERR_TIMEOUT from sync).  Results equal the
 * stage-by-stage launches bit for bit.  Elsewhere rk3 falls back to them. */
int selfgpu_model2d_set_multistage(selfgpu_model2d* m, int enable);

/* Explicit launch configuration (what the autotuner picks): persistent 0/1
 * and the persistent kernel's consumer-group cap (0 = as many as fit). */
int selfgpu_model2d_set_launch(selfgpu_model2d* m, int persistent, int groups);

/* Ensembles: n handles (each ready to step; typically one per degree of an
 * uneven batch, every element carrying its instance's dt) advanced together.
 * selfgpu_ensemble_rk3 runs nSteps RK3 steps of every handle as ONE CUDA
 * graph launch per step on the ensemble's stream (NULL at create: its own);
 * the graph has one branch per handle, so the handles' stage kernels run
 * concurrently.  Results equal selfgpu_model2d_rk3 on each handle bit for
 * bit.  Work issued earlier on the handles' streams runs first, and later
 * work on them waits for the steps.  The handles must outlive the ensemble. */
typedef struct selfgpu_ensemble selfgpu_ensemble;
int selfgpu_ensemble_create(selfgpu_model2d* const* handles, int n, void* stream, selfgpu_ensemble** out);
int selfgpu_ensemble_rk3(selfgpu_ensemble* e, double dt, int nSteps);
int selfgpu_ensemble_destroy(selfgpu_ensemble* e);

/* Autotuner: times the per-element-group kernel and the persistent kernel at
 * every consumer-group count that fits (elements in flight per CTA, each with
 * its double-buffered staging tile) on RK-stage launches over this handle's
 * own data (a zero step on scratch copies of the solution and RK register;
 * the state is not modified), keeps the fastest, and reports it (persistent
 * 0/1, group count, microseconds per stage).  Allocates scratch memory. */
int selfgpu_model2d_autotune(selfgpu_model2d* m, int* persistent, int* groups, float* usPerStage);

/* Failure detection.  Every wait inside the persistent kernel is bounded; a
 * wait that runs out sets an error word, the kernel stops and returns, and the
 * next selfgpu_model2d_sync() returns SELFGPU_ERR_TIMEOUT.  set_wait_limit
 * sets the bound in SM clock cycles (default 4e9, about 2 s).  inject_stall
 * (for tests of this path) with enable = 1 makes the next launches register
 * one element's copies without issuing them, so its consumers' wait runs
 * out; with enable = 2 one group of a multi-stage launch (set_multistage)
 * never announces the end of its stages, so the others' stage-end waits run
 * out. */
int selfgpu_model2d_set_wait_limit(selfgpu_model2d* m, long long cycles);
int selfgpu_model2d_inject_stall(selfgpu_model2d* m, int enable);

/* ========================================= 4. tendency without allocation */

/* Size of the fixed device array behind selfgpu_cig2d_tendency_noalloc. */
#define SELFGPU_NOALLOC_SCRATCH_BYTES (16 * 1024 * 1024)

/* No counterpart in the reference: an added entry point for callers that may
 * not allocate device memory (a host code that owns every device buffer and
 * forbids the library to allocate, a process under a fixed device-memory cap,
 * a call inside a solver step that must not stall or fail on cudaMalloc).
 * It computes the CompressibleIdealGas2D tendency dSdt bit for bit as
 * selfgpu_model2d_tendency does for a SELFGPU_FP64_REF CIG handle with no
 * gravity, drag or prescribed-boundary fields, from caller-owned device
 * arrays in SELF's layouts (solution (P,P,4,nEl), dsdx, J, nHat, nScale,
 * sideInfo on the device plus a host copy of sideInfo for validation) and
 * host copies of dgMatrix, bMatrix and qWeights.  Sides must be periodic /
 * interior (bcid 0) or NONORMALFLOW walls; any other physical side is
 * rejected with SELFGPU_ERR_ARG.  There is no gravity or drag term (so g
 * plays no part) and R only enters a diagnostic the tendency does not use.
 * It calls no allocator: its face-trace scratch is a file-scope device array
 * of SELFGPU_NOALLOC_SCRATCH_BYTES; inputs needing more (above 7281 elements
 * at N = 7, 14563 at N = 3) are rejected with SELFGPU_ERR_ARG.  CUDA loads
 * device code lazily, so the first call on a device reserves the array there
 * (and looks up its address), and the device holds it until the process
 * exits: make that first call during set-up, before any stream capture.  All
 * calls on a device share the array: calls that overlap on the GPU race. */
int selfgpu_cig2d_tendency_noalloc(const double* solution, double* dSdt, const double* dsdx, const double* J,
                                   const double* nHat, const double* nScale, const int* sideInfo_d,
                                   const int* sideInfo_h, const double* dgMatrix, const double* bMatrix,
                                   const double* qWeights, double expansionFactor, int N, int nEl, void* stream);

/* ==================================== 5. shock closure (artificial viscosity) */

/* No counterpart in the reference's tendency: an artificial-viscosity closure
 * for CompressibleIdealGas2D built from the reference's operators
 * (BassiRebaySides + GradientBR, src/SELF_MappedData.f90:919-1078; the
 * Advection2D diffusive fluxes, src/models/hip/SELF_Advection2D.cpp:66-175)
 * with one viscosity per element.  With a closure set, every tendency / RK
 * stage adds div(nu_e grad q) through BR1.  nu_e is formed at the first
 * stage of each RK step (and at every tendency evaluation) and held over the
 * step's other two stages; the gradient is formed at every stage.
 *   mode 1: nu_e from the modal-decay indicator of the density (Persson &
 *           Peraire): a(s) ramps from 0 at s0 - kappa to 1 at s0 + kappa,
 *           s = log10 of the energy fraction in the highest modes;
 *   mode 2: a from the closure MLP (selfgpu_model2d_set_mlp; N >= 5), the
 *           indicator as fallback for features outside the training range;
 *   mode 0: off.
 * nu_e = a * c * h_e / N * max(|u| + c_sound), h_e = sqrt(element area).
 * controlPoints: the P quadrature nodes (Lagrange%controlPoints). */
#define SELFGPU_CLOSURE_OFF 0
#define SELFGPU_CLOSURE_INDICATOR 1
#define SELFGPU_CLOSURE_MLP 2
#define SELFGPU_MLP_WEIGHTS 2208 /* bf16: W1 (32 x 36, row-major), W2 (32 x 32), w3 (32) */
#define SELFGPU_MLP_PARAMS 137   /* float: b1 (32), b2 (32), b3, feature minima (36), maxima (36) */
int selfgpu_model2d_set_closure(selfgpu_model2d* m, int mode, double c, double s0, double kappa,
                                const double* controlPoints);

/* Closure MLP 36 -> 32 -> 32 -> 1 (ReLU, output clamped to [0, 1]): bfloat16
 * weights (raw 16-bit patterns) and float biases / feature ranges, host arrays. */
int selfgpu_model2d_set_mlp(selfgpu_model2d* m, const uint16_t* weights, const float* params);

/* Copies (on the engine's stream) the element viscosity last formed (nEl
 * doubles), the activation applied and the indicator's activation (nEl floats
 * each; the latter written in mode 2) into caller-owned device arrays (each
 * may be NULL), and returns on the host (counts[2], may be NULL) the MLP
 * fallbacks and the MLP evaluations since the last reset.  In mode 2 the
 * indicator screens: elements more than one decade below the activation ramp
 * get a = 0 without an MLP evaluation. */
int selfgpu_model2d_closure_state(selfgpu_model2d* m, double* nu, float* activation, float* indicatorActivation,
                                  int* counts, int resetCounts);

/* Modal transform T(k,i) = w_i sqrt((2k+1)/2) L_k(x_i) (P x P, k fastest). */
int selfgpu_modal_matrix(int N, const double* controlPoints, const double* qWeights, double* T);

/* Training-data harvest: per element of a device CIG state (P,P,4,nEl), the
 * indicator activation of the density and the 36 closure features (36, nEl),
 * float32 device outputs (either may be NULL; features need N >= 5). */
int selfgpu_cig2d_closure_features(const double* solution, int N, int nEl, const double* controlPoints,
                                   const double* qWeights, double s0, double kappa, float* activation,
                                   float* features, void* stream);

/* Training of the closure MLP on device samples features (36, n) and labels
 * (n): minibatch Adam on float32 master weights with the forward pass on
 * bfloat16-rounded weights (quantisation-aware), squared error on the
 * clamped output.  params (host, in/out) holds the float32 masters in the
 * order W1 (32x36), b1 (32), W2 (32x32), b2 (32), w3 (32), b3 (1): 2273
 * floats.  lossPerEpoch (host, epochs floats) may be NULL. */
#define SELFGPU_MLP_MASTER 2273
int selfgpu_mlp_train(const float* features, const float* labels, int n, int epochs, int batch, float lr,
                      unsigned long long seed, float* params, float* lossPerEpoch, void* stream);

/* Inference of the closure MLP over n device feature vectors (36, n) into
 * out (n floats), with the device-side weights layout of set_mlp (host arrays). */
int selfgpu_mlp_infer(const float* features, int n, const uint16_t* weights, const float* params, float* out,
                      void* stream);

/* ====================================================== 6. checkpoint files */

/* Checkpoint / pickup files with the dataset paths, Fortran-order shapes and
 * attributes of Write_Model2D / Read_Model2D (src/SELF_Model2D.f90:861-1099:
 * /quadrature/{xi,weights,dgmatrix,dmatrix,bmatrix}, /state/interior/solution,
 * /state/boundary/solution, /mesh/interior/x, /mesh/boundary/x, attribute N)
 * in a plain binary container instead of HDF5.  Arrays are copied from /
 * to host memory (onDevice = 0) or device memory (onDevice = 1).  dims[] is
 * in Fortran order (first fastest); the last dimension is the element index
 * for per-element data, and selfgpu_ckpt_get can read one rank's element
 * slab of it (Read_Model2D with MPI, :1070-1080). */
#define SELFGPU_DT_F64 1
#define SELFGPU_DT_I32 2
#define SELFGPU_DT_F32 3
typedef struct selfgpu_ckpt selfgpu_ckpt;
int selfgpu_ckpt_open(selfgpu_ckpt** out, const char* path, int write);
int selfgpu_ckpt_put(selfgpu_ckpt* c, const char* name, const void* data, int dtype, int ndims, const long long* dims,
                     int onDevice);
int selfgpu_ckpt_put_attr(selfgpu_ckpt* c, const char* name, double value);
int selfgpu_ckpt_info(selfgpu_ckpt* c, const char* name, int* dtype, int* ndims, long long* dims);
int selfgpu_ckpt_get(selfgpu_ckpt* c, const char* name, void* data, long long capacityBytes, long long elemOffset,
                     long long nElem, int onDevice);
int selfgpu_ckpt_get_attr(selfgpu_ckpt* c, const char* name, double* value);
int selfgpu_ckpt_close(selfgpu_ckpt* c);

/* TimeStamp(time, 's') (src/SELF_SupportRoutines.f90:856-924): "DDDDHHMMSSmmm"
 * into out (14 bytes with the terminator); the default pickup name is
 * solution.<stamp>.ckpt. */
int selfgpu_time_stamp(double time, char* out);

/* ============================================ 7. multi-rank decomposition */

/* DomainDecomp (src/SELF_Mesh.f90:2159-2177): contiguous element ranges,
 * offsetElem[d] = first element (0-based) of rank d, offsetElem[nDomains] =
 * nElems.  ElemToRank (:2179-2215): the rank holding the 1-based elemID. */
int selfgpu_domain_decomp(int nElems, int nDomains, int* offsetElem);
int selfgpu_elem_to_rank(int nDomains, const int* offsetElem, int elemID, int* domain);

/* Halo plan of one rank (the B200 form of MPIExchangeAsync + ApplyFlip,
 * src/SELF_MappedData.f90:3323-3443): the rank's sideInfo (5,4,nLocal) with
 * each off-rank neighbour renumbered to a halo element nLocal+1..nLocal+nHalo
 * (the fused kernels then apply flips themselves), the number of shared
 * faces per peer rank, and per face (concatenated in peer order, shared faces
 * sorted by their lower global (element, side)) the trace-cache block this
 * rank sends (side + 4 * element) and the halo block it receives.
 * sendBlocks / recvBlocks: room for 4 * nLocal ints. */
int selfgpu_halo_plan(const int* sideInfoGlobal, int nElGlobal, int nDomains, const int* offsetElem, int rank,
                      int* sideInfoLocal, int* nHalo, int* peerCount, int* sendBlocks, int* recvBlocks);

/* Engine side of a decomposed run.  set_halo (before set_geometry) sizes the
 * trace caches for nEl + nHalo elements.  Per RK stage the host then runs:
 * prologue (after setting the solution) or stage m, and between them the
 * exchange: pack the send blocks of the caches the next stage reads
 * (selfgpu_model2d_caches: face traces, and for ShallowWater the stage-lagged
 * velocity traces), move them to the peers (NCCL send/recv or any transport),
 * unpack into the halo blocks.  The shock closure is single-rank. */
int selfgpu_model2d_set_halo(selfgpu_model2d* m, int nHalo);
int selfgpu_model2d_prologue(selfgpu_model2d* m);
int selfgpu_model2d_stage(selfgpu_model2d* m, double dt, int stage);
int selfgpu_model2d_caches(selfgpu_model2d* m, void** traces, int* traceBlockBytes, void** velocity,
                           int* velocityBlockBytes);
/* packed[k] = cache block blocks[k] / cache block blocks[k] = packed[k]
 * (device arrays; blockBytes a multiple of 4; blocks on the device). */
int selfgpu_pack_blocks(const void* cache, const int* blocks, int n, int blockBytes, void* packed, void* stream);
int selfgpu_unpack_blocks(const void* packed, const int* blocks, int n, int blockBytes, void* cache, void* stream);

/* ============================================ 8. HIP runtime memory shim */

/* The five HIP runtime entry points SELF's Fortran memory layer reaches
 * through hipfort's bind(c) interfaces (src/SELF_Memory.f90:11-12 USE
 * hipfort), implemented on the CUDA runtime so that layer runs unchanged
 * without ROCm/HIP: link hipfort's interface modules against libselfgpu
 * instead of the HIP runtime (never both in one process).  Return value:
 * hipError_t (0 = hipSuccess; 1 invalid value, 2 out of memory, 100 no
 * device, 101 invalid device, 999 any other failure). */
/* replaces hipMalloc as bound by hipfort: Alloc_hfReal_r1 etc., src/SELF_Memory.f90:362 */
int hipMalloc(void** ptr, size_t sizeBytes);
/* replaces hipFree: Free_hfReal_r1 etc., src/SELF_Memory.f90:767-777 */
int hipFree(void* ptr);
/* replaces hipMemcpy: UpdateHost/UpdateDevice, src/SELF_Memory.f90:988-1033, :1295-1306;
 * kind = hipMemcpyKind (0 host-host, 1 host-device, 2 device-host, 3 device-device, 4 default) */
int hipMemcpy(void* dst, const void* src, size_t sizeBytes, int kind);
/* replaces hipGetDeviceCount: GPUAvailable, src/SELF_Memory.f90:336-350; src/SELF_Mesh.f90:2043 */
int hipGetDeviceCount(int* count);
/* replaces hipSetDevice: rank-to-GPU binding, src/SELF_Mesh.f90:2050 */
int hipSetDevice(int deviceId);

#ifdef __cplusplus
}
#endif
#endif /* SELFGPU_H */
