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
 *   hyb_function_create           P1Function<V>(name, storage, minLevel, maxLevel)
 *                                 (src/hyteg/p1functionspace/P1Function.hpp:26-27)
 *   hyb_function_interpolate_const  VertexDoFFunction::interpolate(constant, level, flag)
 *   hyb_function_assign / _add    VertexDoFFunction::assign / add (VertexDoFFunction.cpp:1076-1098, 1357+)
 *   hyb_function_dot              VertexDoFFunction::dotGlobal (VertexDoFFunction.cpp:1669-1740)
 *   hyb_function_copy_convert     P1Function<float> <-> P1Function<double> copy (mixed precision)
 *   hyb_operator_create_laplace   P1ConstantLaplaceOperator (P1ConstantOperator.cpp:603-655 stencil assembly)
 *   hyb_operator_create_divkgrad  P1ElementwiseOperator<forms::p1_div_k_grad_affine_q3>
 *                                 (src/hyteg/elementwiseoperators/P1ElementwiseOperator.cpp:64-302)
 *   hyb_operator_apply            Operator::apply(src, dst, level, flag, updateType) (P1Operator.hpp:196)
 *   hyb_operator_smooth_sor       SORSmoothable::smooth_sor(dst, rhs, relax, level, flag) (P1Operator.hpp:343-422)
 *   hyb_operator_smooth_jac       WeightedJacobiSmoothable::smooth_jac (P1Operator.hpp:424-440)
 *   hyb_prolongate                P1toP1LinearProlongation::prolongate / prolongateAndAdd
 *                                 (src/hyteg/gridtransferoperators/P1toP1LinearProlongation.cpp:194-410)
 *   hyb_restrict                  P1toP1LinearRestriction::restrict (P1toP1LinearRestriction.cpp:168-345)
 *   hyb_cg_solve                  CGSolver::solve (src/hyteg/solvers/CGSolver.hpp:66-135)
 *   hyb_gmg_create / hyb_gmg_solve  GeometricMultigridSolver ctor / solve (GeometricMultigridSolver.hpp:42-235)
 *
 * Conventions: plain pointers and sizes; every call that enqueues GPU work
 * takes a cudaStream_t passed as void* (NULL = legacy default stream) and is
 * asynchronous unless documented as blocking. Every call returns an hyb_status;
 * hyb_last_error() describes the last failure of the calling thread. Flags are
 * the reference's DoFType bits and UpdateType values.
 */
#ifndef HYTEG_B200_H
#define HYTEG_B200_H

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
/* smoothers of the V-cycle */
#define HYB_SMOOTHER_SOR 0
#define HYB_SMOOTHER_JACOBI 1

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
 * calls that overlap on the GPU (other streams, other host threads) race. */
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
int hyb_operator_destroy( hyb_operator* op );
int hyb_operator_apply( hyb_operator* op, hyb_function* src, hyb_function* dst, int level, int flag, int update,
                        void* stream );
/* r = b - A x on flag (fused residual) */
int hyb_operator_residual( hyb_operator* op, hyb_function* x, hyb_function* b, hyb_function* r, int level, int flag,
                           void* stream );
/* one multicolour SOR sweep (colours in increasing order) */
int hyb_operator_smooth_sor( hyb_operator* op, hyb_function* dst, hyb_function* rhs, double relax, int level, int flag,
                             void* stream );
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
/* one V-cycle on level (GeometricMultigridSolver::solve); b's coarser levels are scratch */
int hyb_gmg_solve( hyb_gmg* g, hyb_function* x, hyb_function* b, int level, void* stream );
/* blocking: cycles until ||b - Ax|| / ||b|| <= rel_tol (Inner|Neumann DoFs) or max_cycles.
 * precision 64: plain FP64 V-cycles; 32: FP32 V-cycles on the residual equation inside
 * FP64 iterative refinement (FP64 residual, update and coarse solve).
 * history[0..cycles] (optional) receives the relative residuals. */
int hyb_gmg_solve_to_tolerance( hyb_gmg* g, hyb_function* x, hyb_function* b, int level, double rel_tol,
                                int max_cycles, int precision, double* history, int* cycles, void* stream );

#ifdef __cplusplus
}
#endif

#endif /* HYTEG_B200_H */
