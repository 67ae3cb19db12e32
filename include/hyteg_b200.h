/*
 * C ABI of the B200 matrix-free P1 geometric-multigrid path.
 *
 * Each entry point replaces one call of the reference's operator/solver API
 * (paths relative to the reference project root, se-sic/hyteg-VaRA):
 *
 *   hyb_storage_create            SetupPrimitiveStorage(meshInfo, nproc) +
 *                                 setMeshBoundaryFlagsOnBoundary(1,0,true) + PrimitiveStorage
 *                                 (src/hyteg/primitivestorage/SetupPrimitiveStorage.hpp:52,136)
 *   hyb_storage_create_cuboid     MeshInfo::meshCuboid (src/hyteg/mesh/MeshGenCuboid.cpp:34-160)
 *   hyb_storage_create_spherical_shell  MeshInfo::meshSphericalShell with SHELLMESH_CLASSIC
 *                                 (src/hyteg/mesh/MeshGenSphericalShell.cpp:577-900): the same
 *                                 vertices, cells and cell order
 *   hyb_function_create           P1Function<V>(name, storage, minLevel, maxLevel)
 *                                 (src/hyteg/p1functionspace/P1Function.hpp:26-27)
 *   hyb_function_interpolate_const  VertexDoFFunction::interpolate(constant, level, flag)
 *   hyb_function_assign / _add    VertexDoFFunction::assign / add (VertexDoFFunction.cpp:1076-1098, 1357+)
 *   hyb_function_dot              VertexDoFFunction::dotGlobal (VertexDoFFunction.cpp:1669-1740)
 *   hyb_function_copy_convert     P1Function<float> <-> P1Function<double> copy (mixed precision)
 *   hyb_operator_create_laplace   P1ConstantLaplaceOperator (P1ConstantOperator.cpp:603-655 stencil assembly)
 *   hyb_operator_create_divkgrad  P1ElementwiseOperator<forms::p1_div_k_grad_affine_q3>
 *                                 (src/hyteg/elementwiseoperators/P1ElementwiseOperator.cpp:64-302)
 *   hyb_operator_create_blend_divkgrad  P1ElementwiseBlendingDivKGradOperator
 *                                 (src/hyteg/elementwiseoperators/P1ElementwiseOperator.hpp:349, form
 *                                 p1_div_k_grad_blending_q3) with IcosahedralShellMap::setMap
 *                                 (src/hyteg/geometry/IcosahedralShellMap.hpp:225-250)
 *   hyb_operator_apply            Operator::apply(src, dst, level, flag, updateType) (P1Operator.hpp:196)
 *   hyb_operator_smooth_sor       SORSmoothable::smooth_sor(dst, rhs, relax, level, flag) (P1Operator.hpp:343-422)
 *   hyb_operator_smooth_sor_backwards  SORBackwardsSmoothable::smooth_sor_backwards (P1Operator.hpp:424-431)
 *   hyb_operator_smooth_sor_reference_order  smooth_sor / smooth_sor_backwards in the reference's
 *                                 own V -> E -> F -> C lexicographic order (P1Operator.hpp:352-431)
 *   hyb_operator_smooth_jac       WeightedJacobiSmoothable::smooth_jac (P1Operator.hpp:424-440)
 *   hyb_prolongate                P1toP1LinearProlongation::prolongate / prolongateAndAdd
 *                                 (src/hyteg/gridtransferoperators/P1toP1LinearProlongation.cpp:194-410)
 *   hyb_restrict                  P1toP1LinearRestriction::restrict (P1toP1LinearRestriction.cpp:168-345)
 *   hyb_cg_solve                  CGSolver::solve (src/hyteg/solvers/CGSolver.hpp:66-135)
 *   hyb_gmg_create / hyb_gmg_solve  GeometricMultigridSolver ctor / solve (GeometricMultigridSolver.hpp:42-235)
 *   hyb_gmg_set_cycle_type        the CycleType argument of the GeometricMultigridSolver ctor (V or W)
 *   hyb_gmg_setup_chebyshev       ChebyshevSmoother::setupCoefficients (ChebyshevSmoother.hpp)
 *   hyb_operator_estimate_spectral_radius  chebyshev::estimateRadius (ChebyshevSmoother.hpp)
 *   hyb_gmg_solve_fmg             FullMultigridSolver::solve (src/hyteg/solvers/FullMultigridSolver.hpp)
 *   hyb_storage_create_from_gmsh  MeshInfo::fromGmshFile (src/hyteg/mesh/MeshGenFromGmshFile.cpp)
 *
 *   hyb_server_*                  no reference counterpart (the reference runs one solve per
 *                                 MPI job): a continuous-batching loop that serves many
 *                                 GeometricMultigridSolver solves on one GPU
 *
 * Conventions: plain pointers and sizes; every call that enqueues GPU work
 * takes a cudaStream_t passed as void* (NULL = legacy default stream) and is
 * asynchronous unless documented as blocking. Every call returns an hyb_status;
 * hyb_last_error() describes the last failure of the calling thread. Flags are
 * the reference's DoFType bits and UpdateType values.
 */
#ifndef HYTEG_B200_H
#define HYTEG_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum
{
   HYB_OK          = 0,
   HYB_EINVAL      = 1, /* invalid argument (reference: WALBERLA_CHECK abort) */
   HYB_ENOMEM      = 2, /* device allocation failed */
   HYB_EUNSUPPORTED = 3, /* operation not available for this object (reference: std::runtime_error) */
   HYB_EDEVICE     = 4, /* CUDA runtime error */
   HYB_ETIMEOUT    = 5, /* iteration budget exhausted without convergence */
   HYB_ENOTCONVERGED = 6
} hyb_status;

/* DoFType (src/hyteg/types/types.hpp:35-44) */
#define HYB_INNER 1
#define HYB_DIRICHLET 2
#define HYB_NEUMANN 4
#define HYB_FREESLIP 8
#define HYB_ALL 15
/* UpdateType */
#define HYB_REPLACE 0
#define HYB_ADD 1
/* value types */
#define HYB_F64 0
#define HYB_F32 1
/* smoothers of the V-cycle: SORSmoother, WeightedJacobiSmoother, SymmetricSORSmoother
 * (src/hyteg/solvers/SymmetricSORSmoother.hpp: a forward, then a backward sweep) */
#define HYB_SMOOTHER_SOR 0
#define HYB_SMOOTHER_JACOBI 1
#define HYB_SMOOTHER_SYMMETRIC_SOR 2
/* ChebyshevSmoother (src/hyteg/solvers/ChebyshevSmoother.hpp): x += p(D^-1 A) D^-1 (b - A x),
 * coefficients from hyb_gmg_setup_chebyshev before the first solve */
#define HYB_SMOOTHER_CHEBYSHEV 3
/* SORSmoother / SymmetricSORSmoother with the reference's own sweep order
 * (hyb_operator_smooth_sor_reference_order) instead of the multicolour order */
#define HYB_SMOOTHER_SOR_REFERENCE_ORDER 4
#define HYB_SMOOTHER_SYMMETRIC_SOR_REFERENCE_ORDER 5
/* multigrid cycle types (GeometricMultigridSolver.hpp CycleType) */
#define HYB_CYCLE_V 0
#define HYB_CYCLE_W 1

typedef struct hyb_storage_s  hyb_storage;
typedef struct hyb_function_s hyb_function;
typedef struct hyb_operator_s hyb_operator;
typedef struct hyb_gmg_s      hyb_gmg;

const char* hyb_last_error( void );
/* number of kernels this library has enqueued so far (a CUDA-graph replay counts the
 * kernels it holds); instrumentation in the spirit of the reference's timing tree */
long long   hyb_kernel_launch_count( void );

/* ---- storage (macro-mesh + level hierarchy metadata on the device) ---- */
int     hyb_storage_create( const double* coords, int64_t num_vertices, const int64_t* tets, int64_t num_tets,
                            int max_level, hyb_storage** out );
/* MeshInfo::fromGmshFile (src/hyteg/mesh/MeshGenFromGmshFile.cpp): a Gmsh 2.2 ASCII file,
 * vertices in file-id order, tetrahedra in the reference's cell order */
int     hyb_storage_create_from_gmsh( const char* path, int max_level, hyb_storage** out );
/* thick spherical shell, the reference's SHELLMESH_CLASSIC meshing: the icosahedron's ten
 * diamonds refined by arc midpoints into ntan x ntan nodes (ntan - 1 a power of two) on nrad
 * equidistant radii in [rmin, rmax], every grid cell between two radii split into six
 * tetrahedra; vertex ids and cell order as MeshInfo::meshSphericalShell numbers them */
int     hyb_storage_create_spherical_shell( int ntan, int nrad, double rmin, double rmax, int max_level, hyb_storage** out );
int     hyb_storage_create_cuboid( int nx, int ny, int nz, const double* lo3, const double* hi3, int max_level,
                                   hyb_storage** out );
int     hyb_storage_destroy( hyb_storage* s );
/* counts[0..3] = macro-vertices, -edges, -faces, -cells */
int     hyb_storage_counts( const hyb_storage* s, int64_t* counts4 );
int64_t hyb_storage_num_dofs( const hyb_storage* s, int level );
/* mesh as stored (coords: num_vertices x 3, tets: num_tets x 4) */
int     hyb_storage_mesh( const hyb_storage* s, double* coords, int64_t* tets );
/* coordinates (num_dofs x 3) of the micro-vertices of a level in the canonical DoF order
 * (vertexdof::macrocell::coordinateFromIndex, VertexDoFMacroCell.hpp:68-75), for
 * host-side interpolation of right-hand sides and coefficients */
int     hyb_storage_dof_coords( const hyb_storage* s, int level, double* xyz );
/* multicolour SOR: number of colours and the per-macro-vertex labels */
int     hyb_storage_colouring( const hyb_storage* s, int* num_colours, int* labels );

/* ---- P1 functions ---- */
int hyb_function_create( hyb_storage* s, int min_level, int max_level, int dtype, hyb_function** out );
int hyb_function_destroy( hyb_function* f );
/* host <-> device in the canonical DoF order (hyb_storage_num_dofs values of the
 * function's dtype); blocking with respect to the host buffer */
int hyb_function_upload( hyb_function* f, int level, const void* host_dofs, void* stream );
int hyb_function_download( hyb_function* f, int level, void* host_dofs, void* stream );
/* same, with the canonical DoF vector already in device memory */
int hyb_function_upload_device( hyb_function* f, int level, const void* device_dofs, void* stream );
int hyb_function_download_device( hyb_function* f, int level, void* device_dofs, void* stream );
int hyb_function_interpolate_const( hyb_function* f, int level, double value, int flag, void* stream );
/* Seeded synthetic input on the device (no reference counterpart: the reference's
 * benchmarks interpolate analytic right-hand sides): every DoF gets a value in [-1, 1)
 * from a SplitMix64 hash of its position on the lattice of spacing 1/lattice and of the
 * seed, so replicas and repeated calls agree bit for bit and the values do not depend
 * on the mesh partition. */
int hyb_function_fill_uniform_random( hyb_function* f, int level, uint64_t seed, double lattice, void* stream );
/* f = sum_i scalars[i] * srcs[i]   (n <= 3)  /  f += sum_i ... */
int hyb_function_assign( hyb_function* f, int level, int n, const double* scalars, hyb_function* const* srcs, int flag,
                         void* stream );
int hyb_function_add( hyb_function* f, int level, int n, const double* scalars, hyb_function* const* srcs, int flag,
                      void* stream );
/* blocking: returns the dot product over the DoFs whose BC is in flag */
int hyb_function_dot( hyb_function* a, hyb_function* b, int level, int flag, double* out, void* stream );
int hyb_function_copy_convert( hyb_function* dst, hyb_function* src, int level, void* stream );
/* Same dot product as hyb_function_dot, for callers that cannot allocate device memory
 * while they run (a serving loop bound to a fixed HBM budget, a host framework that owns
 * the allocator). No counterpart in the reference. It allocates nothing: its scratch is
 * a 1 MiB file-scope device array that every GPU loading this library holds until exit,
 * so problems needing more than 131072 partial sums ((closure size / 256, rounded up) x
 * #macro-cells) are rejected with HYB_EINVAL. Asynchronous on `stream`; the result is
 * written to the device double `out_device`. The first call on a device looks up the
 * array's device address with that device current; make that first call before any
 * stream capture. All calls share the array and it keeps the last call's contents:
 * calls that overlap on the GPU (other streams, other host threads) race, and so do
 * CUDA graphs captured from this call: their partial sums go to the same array, so such
 * a graph must not run concurrently with another call or graph of this entry point.
 * The functions and out_device must live on the current device (HYB_EINVAL otherwise);
 * the looked-up address is cached, so do not call this after a cudaDeviceReset. */
int hyb_function_dot_noalloc( hyb_function* a, hyb_function* b, int level, int flag, double* out_device, void* stream );

/* ---- operators ---- */
int hyb_operator_create_laplace( hyb_storage* s, int min_level, int max_level, hyb_operator** out );
/* nodal_k[l - min_level] = coefficient values at the micro-vertices of level l in the
 * canonical DoF order; the element coefficient is the P1 interpolant integrated by the
 * reference form's 5-point rule */
int hyb_operator_create_divkgrad( hyb_storage* s, int min_level, int max_level, const double* const* nodal_k,
                                  hyb_operator** out );
/* the coefficient as a callback k(x) evaluated at every micro-vertex of every level */
int hyb_operator_create_divkgrad_callback( hyb_storage* s, int min_level, int max_level,
                                           double ( *k )( const double* xyz, void* ctx ), void* ctx,
                                           hyb_operator** out );
/* the coefficient k(x) = exp( radial (1 - |x|) + sigma sqrt(2/modes) sum_m cos( w_m . x + phase_m ) )
 * (a radial profile times the exponential of random Fourier features of a Gaussian random
 * field; w is modes x 3, phase has modes entries), evaluated on the device at every
 * micro-vertex of every level; blocking */
int hyb_operator_create_divkgrad_rff( hyb_storage* s, int min_level, int max_level, const double* w,
                                      const double* phase, int modes, double sigma, double radial, hyb_operator** out );
/* P1ElementwiseOperator< p1_div_k_grad_affine_q3 > with its coefficient callback as the
 * reference evaluates it (p1_div_k_grad_affine_q3.cpp:179+, per level from
 * P1ElementwiseOperator.cpp:64-221): k at the 5 quadrature points of every micro-tet on every
 * level, where the nodal operators above take the level's P1 interpolant. The factors
 * 24 sum_q w_q k(x_q) are computed once per level on the device and kept (6 values per
 * closure point and cell, FP64 and FP32), so an application reads one factor per incident
 * micro-tet. kind 1: k = tanh(2 (x - 1/2)) + 2 (ElementwiseDivKGradCGConvergenceTest's
 * coefficient; w, phase, modes, sigma, radial ignored); kind 2: the random-feature field of
 * hyb_operator_create_divkgrad_rff. Every smoother, CG and GMG accept it; blocking */
int hyb_operator_create_divkgrad_quadrature( hyb_storage* s, int min_level, int max_level, int kind, const double* w,
                                             const double* phase, int modes, double sigma, double radial,
                                             hyb_operator** out );
/* The same with any coefficient callback k(x) (P1ElementwiseOperator< p1_div_k_grad_affine_q3 >
 * with form(callback)): k is called on the host at the 5 quadrature points of every micro-tet
 * of every level (and at every micro-vertex, for the nodal values); blocking */
int hyb_operator_create_divkgrad_callback_quadrature( hyb_storage* s, int min_level, int max_level,
                                                      double ( *k )( const double* xyz, void* ctx ), void* ctx,
                                                      hyb_operator** out );
/* the curved-shell operator: every macro-cell of a spherical-shell mesh gets its
 * IcosahedralShellMap, and the element matrices of p1_div_k_grad_blending_q3 (5-point rule,
 * map Jacobian at the quadrature points) are integrated on the device per row, with
 * k(y) = exp( alpha (1 - |y|) ) at the mapped points (alpha = 0: the Laplacian). Levels
 * up to 7; apply, residual, (symmetric/backward) SOR, weighted Jacobi, the inverse
 * diagonal (Chebyshev smoother, spectral radius estimate), CG and GMG; an error when a cell
 * has no shell map */
int hyb_operator_create_blend_divkgrad( hyb_storage* s, int min_level, int max_level, double alpha,
                                        hyb_operator** out );
int hyb_operator_destroy( hyb_operator* op );
int hyb_operator_apply( hyb_operator* op, hyb_function* src, hyb_function* dst, int level, int flag, int update,
                        void* stream );
/* r = b - A x on flag (fused residual) */
int hyb_operator_residual( hyb_operator* op, hyb_function* x, hyb_function* b, hyb_function* r, int level, int flag,
                           void* stream );
/* one multicolour SOR sweep (colours in increasing order) */
int hyb_operator_smooth_sor( hyb_operator* op, hyb_function* dst, hyb_function* rhs, double relax, int level, int flag,
                             void* stream );
/* one backward multicolour SOR sweep: the passes of hyb_operator_smooth_sor in reverse
 * order (interior colours 3..0, then the surface colours m-1..0) */
int hyb_operator_smooth_sor_backwards( hyb_operator* op, hyb_function* dst, hyb_function* rhs, double relax, int level,
                                       int flag, void* stream );
/* one SOR sweep in the reference's order (P1Operator.hpp:352-431): macro-vertices, -edges,
 * -faces, then -cells (backwards != 0: cells, faces, edges, vertices), each primitive
 * lexicographic (backwards: reversed) and reading its own closure's current values and every
 * other DoF as it was when the sweep (backwards: the stage) began; stencil and coefficient
 * operators (not the blending operator). The call keeps the sweep's start-of-stage copy and
 * the face couplings in scratch buffers of the storage: calls on one storage must not
 * overlap in time (a GMG solver with a reference-order smoother has its own) */
int hyb_operator_smooth_sor_reference_order( hyb_operator* op, hyb_function* dst, hyb_function* rhs, double relax,
                                             int level, int flag, int backwards, void* stream );
/* dst = src + relax * diag(A)^-1 (rhs - A src) */
int hyb_operator_smooth_jac( hyb_operator* op, hyb_function* dst, hyb_function* rhs, hyb_function* src, double relax,
                             int level, int flag, void* stream );
/* partial stencil of one macro-cell and class mask (15 weights, repository offset order) */
int hyb_operator_cell_stencil( const hyb_operator* op, int level, int cell, int mask, double* out15 );

/* ---- grid transfer (in place on a multi-level function) ---- */
int hyb_prolongate( hyb_function* f, int source_level, int flag, int update, void* stream );
int hyb_restrict( hyb_function* f, int source_level, int flag, void* stream );

/* ---- solvers ---- */
/* blocking; iterations and convergence (1) / budget exhausted (2) reported */
int hyb_cg_solve( hyb_operator* op, hyb_function* x, hyb_function* b, int level, double tol, int max_iter,
                  int* iterations, int* converged, void* stream );
int hyb_gmg_create( hyb_storage* s, hyb_operator* op, int min_level, int max_level, int pre_smooth, int post_smooth,
                    double relax, int smoother, double coarse_tol, int coarse_max_iter, hyb_gmg** out );
int hyb_gmg_destroy( hyb_gmg* g );
/* HYB_CYCLE_V (default) or HYB_CYCLE_W: with W the coarse-grid correction recurses twice
 * (GeometricMultigridSolver.hpp:201-204); applies to every later solve of this solver */
int hyb_gmg_set_cycle_type( hyb_gmg* g, int cycle_type );
/* Stage timers in the shape of the reference's timing tree (the WcTimingTree that
 * GeometricMultigridSolver.hpp:129-233 starts and stops): "Geometric Multigrid Solver" per
 * V-cycle, with children "Level l" (started twice per cycle: before and after the coarse
 * correction), and under those "Smoother", "Restriction", "Prolongation" and, on the
 * coarsest level, "Coarse Grid Solver". The residual sits in its level's own time, as in
 * the reference. The times come from CUDA events recorded on the solve's stream. While
 * timing is on, solves run launch by launch, without CUDA graphs or the one-block program
 * kernel, so every level has its own nodes; off (the default) costs nothing. */
int hyb_gmg_set_timing( hyb_gmg* g, int enable );
/* The accumulated tree as JSON, {"<name>": {"total": s, "average": s, "min": s, "max": s,
 * "count": n, "children": {...}}, ...}. Waits for the recorded events. *length receives the
 * size without the terminating NUL; buf may be NULL to ask for it, else capacity must
 * exceed it (HYB_EINVAL otherwise). */
int hyb_gmg_timing_json( hyb_gmg* g, char* buf, size_t capacity, size_t* length );
/* clears the accumulated times (no timer may be open) */
int hyb_gmg_timing_reset( hyb_gmg* g );
/* ChebyshevSmoother::setupCoefficients(order, lowerBound, upperBound) (ChebyshevSmoother.hpp:98-188):
 * order 1..5, eigenvalue interval [lower, upper] of D^-1 A (the reference's
 * setupCoefficients(order, rho) uses [0.3 rho, 1.2 rho]) */
int hyb_gmg_setup_chebyshev( hyb_gmg* g, int order, double lower, double upper );
/* the coefficients w_0 .. w_{order-1} those calls use */
int hyb_chebyshev_coefficients( int order, double lower, double upper, double* out );
/* chebyshev::estimateRadius (ChebyshevSmoother.hpp:252-262): power iteration on D^-1 A with
 * flag All (SpectrumEstimation.hpp:57-81); x (FP64) is the start vector and is overwritten,
 * tmp (FP64) is scratch; blocking */
int hyb_operator_estimate_spectral_radius( hyb_operator* op, hyb_function* x, hyb_function* tmp, int level,
                                           int iterations, double* radius );
/* one V-cycle on level (GeometricMultigridSolver::solve); b's coarser levels are scratch */
int hyb_gmg_solve( hyb_gmg* g, hyb_function* x, hyb_function* b, int level, void* stream );
/* blocking: cycles until ||b - Ax|| / ||b|| <= rel_tol (Inner|Neumann DoFs) or max_cycles.
 * precision 64: plain FP64 V-cycles; 32: FP32 V-cycles on the residual equation inside
 * FP64 iterative refinement (FP64 residual, update and coarse solve).
 * history[0..cycles] (optional) receives the relative residuals. */
/* FullMultigridSolver::solve (src/hyteg/solvers/FullMultigridSolver.hpp:51-75) with linear
 * FMG prolongation: for l = min_level .. level, cycles_per_level V-cycles on l, then
 * x(l+1) = P x(l) on inner and Neumann DoFs. As in the reference, b must hold the
 * right-hand side on every level, x's coarsest level is the start of the coarse solve, and
 * the V-cycles use b's levels below the current one as scratch. Captured as one CUDA graph
 * per (x, b, level, cycles_per_level); asynchronous. */
int hyb_gmg_solve_fmg( hyb_gmg* g, hyb_function* x, hyb_function* b, int level, int cycles_per_level, void* stream );
int hyb_gmg_solve_to_tolerance( hyb_gmg* g, hyb_function* x, hyb_function* b, int level, double rel_tol,
                                int max_cycles, int precision, double* history, int* cycles, void* stream );

/* ---- serving loop ----
 * Poisson solves -div(k grad u) = f, u = 0 on the boundary, on the unit cube split into
 * nx x ny x nz macro-cubes of 6 macro-tets each, arrive at stated times. The server
 * admits a request when an active slot and its device footprint (hyb_server_footprint)
 * fit the byte budget, keeps each admitted hierarchy resident (an idle hierarchy of the
 * same shape is reused; idle ones are evicted least recently used when memory is needed),
 * and runs every admitted solve on its own stream as one captured CUDA graph that
 * iterates V-cycles (FP64) or refinement steps (FP32 V-cycle in FP64 refinement) with
 * the stopping test on the device, so the solves in flight overlap on the GPU and the
 * host touches a solve only at its start and end. Hierarchies of at most 65536 closure
 * points on their finest level run whole V-cycles in one thread block. New requests
 * join as slots and memory free up. HYB_SERVE_HOST_LOOP=1 steps the solves from the host
 * instead (one graph launch and one residual read per cycle). Each solve is V(3,3) with multicolour SOR (omega 1) and a level-0 FP64 CG
 * coarse solve to 1e-12; f is hyb_function_fill_uniform_random( seed, lattice =
 * lcm(nx,ny,nz) 2^level ) and, for the lognormal coefficient, k is exp of the random
 * field of hyb_rff_features( seed, 0.2, 64 ) with sigma 1 (the radial coefficient: the same
 * field with sigma 0.5 times exp(5 (1 - |x|))). Spherical-shell requests (mesh
 * HYB_MESH_SHELL) use the lattice 2^20 for f. Results do not depend on which other
 * requests share the GPU. */
typedef struct hyb_server_s hyb_server;

enum
{
   HYB_COEFF_CONSTANT  = 0, /* k = 1 (P1ConstantLaplaceOperator) */
   HYB_COEFF_LOGNORMAL = 1, /* k = exp(g), g a Gaussian random field (P1ElementwiseOperator) */
   HYB_COEFF_RADIAL    = 2  /* k = exp(5 (1 - |x|)) exp(0.5 g): the shell benchmark's coefficient */
};
enum
{
   HYB_MESH_CUBOID = 0, /* unit cube split into nx x ny x nz macro-cubes */
   HYB_MESH_SHELL  = 1  /* spherical shell, radii 0.55..1: ntan = nx, nrad = ny (nz unused) */
};

typedef struct hyb_request
{
   int      nx, ny, nz;   /* macro-cubes per direction (shell: ntan, nrad, unused) */
   int      level;        /* refinement level of the solve */
   int      coefficient;  /* HYB_COEFF_* */
   int      precision;    /* 64: FP64 V-cycles; 32: FP32 V-cycles in FP64 iterative refinement */
   uint64_t seed;         /* right-hand side and coefficient seed */
   double   rel_tol;      /* stop when ||b - A x|| / ||b|| <= rel_tol */
   int      max_cycles;   /* give up (HYB_ENOTCONVERGED) after this many cycles */
   int      mesh;         /* HYB_MESH_*; zero-initialised requests are cuboids */
} hyb_request;

typedef struct hyb_request_result
{
   int    status;          /* HYB_OK; HYB_ENOMEM if it can never fit the budget; HYB_ENOTCONVERGED; ... */
   int    cycles;          /* V-cycles (FP64) or refinement steps (mixed) run */
   double rel_residual;    /* final FP64 ||b - A x|| / ||b|| over inner and Neumann DoFs */
   double arrival_s;       /* host clock, seconds from the start of the hyb_server_run call */
   double admit_s;
   double done_s;          /* the result (and the solution, if requested) is on the host */
   size_t footprint_bytes; /* device bytes held by the hierarchy that served the request */
} hyb_request_result;

/* Host only (no device call): budget_bytes bounds the device memory of all resident
 * hierarchies and meshes; at most max_active solves run at a time; meshes are built up
 * to max_level. */
int hyb_server_create( size_t budget_bytes, int max_active, int max_level, hyb_server** out );
int hyb_server_destroy( hyb_server* s );
/* device bytes that the request's resident hierarchy takes (host only) */
int hyb_server_footprint( const hyb_server* s, const hyb_request* r, size_t* bytes );
/* Queue a request arriving arrival_s seconds after the start of the next hyb_server_run.
 * solution_host, if not NULL, receives the solution on the request's level in the
 * canonical DoF order (hyb_storage_num_dofs doubles). Invalid requests are refused with
 * HYB_EINVAL and requests larger than the whole budget with HYB_ENOMEM; neither is queued. */
int hyb_server_submit( hyb_server* s, const hyb_request* r, double arrival_s, double* solution_host, int* id );
/* Serve the queued requests until all are done or time_limit_s has passed (then the
 * unfinished ones end with HYB_ETIMEOUT); blocking. */
int hyb_server_run( hyb_server* s, double time_limit_s );
int hyb_server_result( const hyb_server* s, int id, hyb_request_result* out );
/* peak device bytes held by the server, hierarchies built, graphs captured */
int hyb_server_stats( const hyb_server* s, size_t* peak_bytes, int* hierarchies_built, int* graphs_captured );
/* Launches of the batched whole-solve kernel and the solves they carried. Hierarchies whose
 * whole V-cycle fits the one-block program kernel (at most 65536 closure points on the
 * finest level) are solved together: the small requests admitted in one round of the loop
 * go into ONE kernel launch, a thread block per solve, which runs each solve from its
 * start residual to its tolerance on the device (HYB_SERVE_BATCH=0 solves them one
 * device-iterated graph each instead). No reference counterpart (the reference runs one
 * solve per job). */
int hyb_server_batch_stats( const hyb_server* s, int* batches, int* batched_solves );
/* device bytes of the meshes the server holds (storage, Laplace operator, row tables),
 * which are never evicted and are not part of a request's footprint */
int hyb_server_mesh_bytes( const hyb_server* s, size_t* bytes );
/* The random Fourier features the server draws for a lognormal request of this seed:
 * w (modes x 3) ~ N(0, 1/corr_len^2), phase (modes) ~ U[0, 2 pi), from a SplitMix64
 * stream and the Box-Muller transform (host only). */
int hyb_rff_features( uint64_t seed, double corr_len, int modes, double* w, double* phase );

#ifdef __cplusplus
}
#endif

#endif /* HYTEG_B200_H */
