// CPU oracle for the HyTeG P1 matrix-free geometric-multigrid path.
//
// TEST INFRASTRUCTURE ONLY. Only tests/, __graft_entry__.smoke() and the
// cpu_baseline / reference arm of bench.py may load this library, and only as
// the checker or the timed CPU baseline. The product path never calls it.
//
// It is a plain, sequential-semantics restatement of the reference algorithm on
// a global DoF vector (one value per micro-vertex). Every entry point cites the
// reference function it follows (paths relative to the reference project root).
//
// Canonical DoF order of one level (shared with the product's upload/download):
//   [macro-vertices in mesh order]
//   [macro-edges (sorted vertex pairs, lexicographic), interior points i=1..N-1,
//    i = micro-weight of the larger-id vertex]
//   [macro-faces (sorted vertex triples, lexicographic), interior points (i,j),
//    i/j = micro-weights of the 2nd/3rd vertex, j outer, i inner]
//   [macro-cells in mesh order, interior points in tet-linear order (x fastest)]
// with N = 2^level. This is the reference's per-primitive logical numbering
// (src/hyteg/p1functionspace/VertexDoFIndexing.hpp, MeshInfo edge/face keys).
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

// DoFType bit flags (src/hyteg/types/types.hpp:35-44)
#define ORC_INNER 1
#define ORC_DIRICHLET 2
#define ORC_NEUMANN 4
#define ORC_FREESLIP 8
#define ORC_ALL 15

void*   orc_create( const double* coords, int64_t nv, const int64_t* tets, int64_t nt, int maxLevel );
void    orc_destroy( void* h );
int64_t orc_num_dofs( void* h, int level );
void    orc_dof_coords( void* h, int level, double* xyz );
void    orc_dof_info( void* h, int level, uint8_t* kind, uint8_t* bc );
// closure point (tet-linear index, reference cell layout) -> canonical DoF of one macro-cell
void    orc_cell_closure_map( void* h, int level, int cell, int32_t* out );
int64_t orc_num_prims( void* h, int kind );

// operators: 0 = constant P1 Laplace; then div-k-grad with nodal k per level
int  orc_op_laplace( void* h );
int  orc_op_divkgrad( void* h, const double* const* nodalK );
// P1ElementwiseMassOperator (exact P1 mass matrix |T| (1 + delta_ij) / 20 per micro-tet)
int  orc_op_mass( void* h );
// P1ElementwiseOperator< p1_div_k_grad_affine_q3 > with the coefficient evaluated as the form's
// callback at every micro-tet's quadrature points on every level (the reference's assembly):
// kind 1 tanh(2 (x - 1/2)) + 2; kind 2 exp(radial (1 - |x|) + sigma sqrt(2/M) sum cos(w.x + phase))
int  orc_op_divkgrad_callback( void* h, int kind, const double* w, const double* phase, int modes, double sigma,
                               double radial );
// P1ElementwiseBlendingDivKGradOperator (p1_div_k_grad_blending_q3) on the macro-cells'
// IcosahedralShellMaps with k(y) = exp( alpha (1 - |y|) ) of the mapped point; -1 if a cell
// cannot be classified as a shell cell
int  orc_op_blend_div_k_grad( void* h, double alpha );
// the shell map of a cell at a computational point: F (3) and DF (3x3, row-major)
int  orc_shell_map_eval( void* h, int cell, const double* x, double* Fx, double* DF );
// the blended element matrix (4x4, row-major) of the micro-tet X (4 vertices x 3) in a cell
int  orc_blend_element_matrix( void* h, int cell, const double* X12, double alpha, double* out16 );
// p1_div_k_grad_affine_q3::integrateAll (tetrahedron) restated: X12 the 4 vertices, the
// coefficient the P1 interpolant of the nodal values k4 (kind 0) or tanh(2 (x - 1/2)) + 2 of
// ElementwiseDivKGradCGConvergenceTest (kind 1) at the rule's points
int  orc_divkgrad_element_matrix( const double* X12, int kind, const double* k4, double* out16 );
// OpenMP threads of the oracle's parallel loops (n > 0 sets them); the count in effect
int  orc_set_threads( int n );
void orc_cell_stencil( void* h, int op, int level, int cell, int mask, double* out15 );

void   orc_apply( void* h, int op, int level, const double* src, double* dst, int flag, int add );
// (A src)[dofs[i]] for the listed DoFs only (every flag), for spot checks on large levels
void   orc_apply_rows( void* h, int op, int level, const double* src, const int64_t* dofs, int64_t n, double* out );
// backwards != 0: smooth_sor_backwards (P1Operator.hpp:424-431)
void   orc_sor_ref( void* h, int op, int level, double* x, const double* b, double relax, int flag, int backwards );
// One or more stages of that sweep: bit 0 macro-vertices, 1 macro-edges, 2 macro-faces,
// 3 macro-cells (15 = orc_sor_ref).
void   orc_sor_ref_stages( void* h, int op, int level, double* x, const double* b, double relax, int flag,
                           int backwards, int stages );
void   orc_sor_colored( void* h, int op, int level, double* x, const double* b, double relax, int flag,
                        const int* labels, int m, int backwards );
void   orc_jacobi( void* h, int op, int level, double* x, const double* b, double relax, int flag );
void   orc_prolongate( void* h, int coarseLevel, const double* coarse, double* fine, int flag, int add );
void   orc_restrict( void* h, int fineLevel, const double* fine, double* coarse, int flag );
double orc_dot( void* h, int level, const double* a, const double* b, int flag );
// ChebyshevSmoother: power-basis coefficients of order 1..5 for the eigenvalue interval
// [lower, upper] of D^-1 A (setupCoefficients), the smoother step, diag(A)^-1, and
// chebyshev::estimateRadius (power iteration on D^-1 A, flag All; x = start vector)
void   orc_chebyshev_coefficients( int order, double lower, double upper, double* out );
void   orc_set_chebyshev( void* h, int order, double lower, double upper );
void   orc_smooth_chebyshev( void* h, int op, int level, double* x, const double* b );
void   orc_inv_diag( void* h, int op, int level, double* out );
double orc_spectral_radius( void* h, int op, int level, int iterations, double* x );
int    orc_cg( void* h, int op, int level, double* x, const double* b, double tol, int maxIter );

// V-cycle GMG (src/hyteg/solvers/GeometricMultigridSolver.hpp:127-235).
// smoother: 0 = reference-order SOR, 1 = multicolour SOR (labels, m), 2 = weighted Jacobi,
// 3 = reference-order symmetric SOR, 4 = multicolour symmetric SOR (SymmetricSORSmoother),
// 5 = Chebyshev (ChebyshevSmoother, coefficients from orc_set_chebyshev).
// cycleType: 0 = V-cycle, 1 = W-cycle.
// precision: 64 = plain FP64 cycles; 32 = FP32 inner V-cycles inside FP64 iterative refinement.
// Runs until ||b-Ax||/||b|| <= relTol (Inner|Neumann DoFs) or maxCycles; history[k] =
// relative residual after cycle k (history[0] = initial). Returns cycles done.
int orc_gmg_solve( void* h, int op, int minLevel, int maxLevel, double* x, const double* b, int pre, int post,
                   double relax, int smoother, const int* labels, int m, double coarseTol, int maxCycles,
                   double relTol, int precision, double* history, int cycleType );

#ifdef __cplusplus
}
#endif
