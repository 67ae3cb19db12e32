// Header-only C++ façade over the C ABI (hyteg_b200.h) with the reference's class
// names and call signatures, so code written against HyTeG's P1 multigrid path
// (src/hyteg/p1functionspace, src/hyteg/gridtransferoperators, src/hyteg/solvers)
// ports by changing includes:
//
//   auto storage = std::make_shared< hyteg::PrimitiveStorage >( coords, tets, maxLevel );
//   hyteg::P1Function< double > u( "u", storage, minLevel, maxLevel ), f( "f", storage, minLevel, maxLevel );
//   hyteg::P1ConstantLaplaceOperator A( storage, minLevel, maxLevel );
//   hyteg::GeometricMultigridSolver< hyteg::P1ConstantLaplaceOperator > gmg( storage, A, minLevel, maxLevel, 3, 3 );
//   gmg.solve( A, u, f, maxLevel );
//
// Failures raise std::runtime_error (the reference aborts via WALBERLA_CHECK or
// throws std::runtime_error, e.g. SORSmoother.hpp:49).
#pragma once

#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "hyteg_b200.h"

namespace hyteg {

enum DoFType : int
{
   None              = 0,
   Inner             = HYB_INNER,
   DirichletBoundary = HYB_DIRICHLET,
   NeumannBoundary   = HYB_NEUMANN,
   FreeslipBoundary  = HYB_FREESLIP,
   All               = HYB_ALL
};
inline DoFType operator|( DoFType a, DoFType b ) { return DoFType( int( a ) | int( b ) ); }

enum UpdateType : int
{
   Replace = HYB_REPLACE,
   Add     = HYB_ADD
};

inline void hybCheck( int code )
{
   if ( code != HYB_OK )
      throw std::runtime_error( std::string( "hyteg_b200: " ) + hyb_last_error() );
}

class PrimitiveStorage
{
 public:
   PrimitiveStorage( const std::vector< double >& coords, const std::vector< int64_t >& tets, int maxLevel )
   {
      hybCheck( hyb_storage_create( coords.data(), int64_t( coords.size() / 3 ), tets.data(), int64_t( tets.size() / 4 ),
                                    maxLevel, &h_ ) );
   }
   // MeshInfo::meshCuboid on [lo, hi]
   PrimitiveStorage( int nx, int ny, int nz, const double lo[3], const double hi[3], int maxLevel )
   {
      hybCheck( hyb_storage_create_cuboid( nx, ny, nz, lo, hi, maxLevel, &h_ ) );
   }
   // MeshInfo::fromGmshFile: a Gmsh 2.2 ASCII tetrahedral mesh
   PrimitiveStorage( const std::string& gmshFile, int maxLevel )
   {
      hybCheck( hyb_storage_create_from_gmsh( gmshFile.c_str(), maxLevel, &h_ ) );
   }
   // MeshInfo::meshSphericalShell( ntan, nrad, rmin, rmax ), affine macro-tets
   PrimitiveStorage( int ntan, int nrad, double rmin, double rmax, int maxLevel )
   {
      hybCheck( hyb_storage_create_spherical_shell( ntan, nrad, rmin, rmax, maxLevel, &h_ ) );
   }
   ~PrimitiveStorage() { hyb_storage_destroy( h_ ); }
   PrimitiveStorage( const PrimitiveStorage& )            = delete;
   PrimitiveStorage& operator=( const PrimitiveStorage& ) = delete;

   hyb_storage* handle() const { return h_; }
   int64_t      numberOfDoFs( int level ) const { return hyb_storage_num_dofs( h_, level ); }
   std::vector< double > dofCoordinates( int level ) const
   {
      std::vector< double > xyz( size_t( numberOfDoFs( level ) ) * 3 );
      hybCheck( hyb_storage_dof_coords( h_, level, xyz.data() ) );
      return xyz;
   }

 private:
   hyb_storage* h_ = nullptr;
};

template < typename ValueType >
class P1Function
{
   static_assert( std::is_same< ValueType, double >::value || std::is_same< ValueType, float >::value,
                  "P1Function<double> or P1Function<float>" );

 public:
   using valueType = ValueType;

   P1Function( const std::string& name, const std::shared_ptr< PrimitiveStorage >& storage, int minLevel, int maxLevel )
   : name_( name )
   , storage_( storage )
   {
      hybCheck( hyb_function_create( storage->handle(), minLevel, maxLevel,
                                     std::is_same< ValueType, double >::value ? HYB_F64 : HYB_F32, &h_ ) );
   }
   ~P1Function() { hyb_function_destroy( h_ ); }
   P1Function( const P1Function& )            = delete;
   P1Function& operator=( const P1Function& ) = delete;

   hyb_function*                            handle() const { return h_; }
   const std::string&                       getFunctionName() const { return name_; }
   const std::shared_ptr< PrimitiveStorage >& getStorage() const { return storage_; }

   void interpolate( ValueType constant, int level, DoFType flag = All ) const
   {
      hybCheck( hyb_function_interpolate_const( h_, level, double( constant ), flag, nullptr ) );
   }
   void assign( const std::vector< ValueType >& scalars, const std::vector< const P1Function* >& functions, int level,
                DoFType flag = All ) const
   {
      lincomb( scalars, functions, level, flag, false );
   }
   void add( const std::vector< ValueType >& scalars, const std::vector< const P1Function* >& functions, int level,
             DoFType flag = All ) const
   {
      lincomb( scalars, functions, level, flag, true );
   }
   ValueType dotGlobal( const P1Function& rhs, int level, DoFType flag = All ) const
   {
      double r = 0;
      hybCheck( hyb_function_dot( h_, rhs.h_, level, flag, &r, nullptr ) );
      return ValueType( r );
   }
   template < typename Other >
   void copyFrom( const P1Function< Other >& other, int level ) const
   {
      hybCheck( hyb_function_copy_convert( h_, other.handle(), level, nullptr ) );
   }
   // canonical DoF order (vertices, edges, faces, cell interiors)
   void setValues( const std::vector< ValueType >& v, int level ) const
   {
      hybCheck( hyb_function_upload( h_, level, v.data(), nullptr ) );
   }
   std::vector< ValueType > getValues( int level ) const
   {
      std::vector< ValueType > v( size_t( storage_->numberOfDoFs( level ) ) );
      hybCheck( hyb_function_download( h_, level, v.data(), nullptr ) );
      return v;
   }

 private:
   void lincomb( const std::vector< ValueType >& sc, const std::vector< const P1Function* >& fs, int level, DoFType flag,
                 bool add ) const
   {
      if ( sc.size() != fs.size() || fs.size() > 3 )
         throw std::invalid_argument( "assign/add take matching scalar and function lists of at most 3" );
      std::vector< double >        s( sc.begin(), sc.end() );
      std::vector< hyb_function* > h;
      for ( auto* f : fs )
         h.push_back( f->handle() );
      hybCheck( add ? hyb_function_add( h_, level, int( h.size() ), s.data(), h.data(), flag, nullptr ) :
                      hyb_function_assign( h_, level, int( h.size() ), s.data(), h.data(), flag, nullptr ) );
   }

   std::string                         name_;
   std::shared_ptr< PrimitiveStorage > storage_;
   hyb_function*                       h_ = nullptr;
};

// Operators (Operator<P1Function,P1Function> + SORSmoothable + WeightedJacobiSmoothable)
class P1OperatorBase
{
 public:
   virtual ~P1OperatorBase() { hyb_operator_destroy( h_ ); }
   hyb_operator* handle() const { return h_; }

   template < typename V >
   void apply( const P1Function< V >& src, const P1Function< V >& dst, int level, DoFType flag,
               UpdateType updateType = Replace ) const
   {
      hybCheck( hyb_operator_apply( h_, src.handle(), dst.handle(), level, flag, updateType, nullptr ) );
   }
   template < typename V >
   void smooth_sor( const P1Function< V >& dst, const P1Function< V >& rhs, V relax, int level, DoFType flag ) const
   {
      hybCheck( hyb_operator_smooth_sor( h_, dst.handle(), rhs.handle(), double( relax ), level, flag, nullptr ) );
   }
   template < typename V >
   void smooth_sor_backwards( const P1Function< V >& dst, const P1Function< V >& rhs, V relax, int level, DoFType flag ) const
   {
      hybCheck( hyb_operator_smooth_sor_backwards( h_, dst.handle(), rhs.handle(), double( relax ), level, flag, nullptr ) );
   }
   // smooth_sor / smooth_sor_backwards in the reference's own staged lexicographic order
   // (macro-vertices, -edges, -faces, -cells) instead of the multicolour order
   template < typename V >
   void smooth_sor_reference_order( const P1Function< V >& dst, const P1Function< V >& rhs, V relax, int level,
                                    DoFType flag, bool backwards = false ) const
   {
      hybCheck( hyb_operator_smooth_sor_reference_order( h_, dst.handle(), rhs.handle(), double( relax ), level, flag,
                                                         backwards ? 1 : 0, nullptr ) );
   }
   template < typename V >
   void smooth_gs( const P1Function< V >& dst, const P1Function< V >& rhs, int level, DoFType flag ) const
   {
      smooth_sor( dst, rhs, V( 1 ), level, flag );
   }
   template < typename V >
   void smooth_gs_backwards( const P1Function< V >& dst, const P1Function< V >& rhs, int level, DoFType flag ) const
   {
      smooth_sor_backwards( dst, rhs, V( 1 ), level, flag );
   }
   // chebyshev::estimateRadius (power iteration on D^-1 A); x is the start vector
   double estimateSpectralRadius( const P1Function< double >& x, const P1Function< double >& tmp, int level,
                                  int iterations ) const
   {
      double r = 0;
      hybCheck( hyb_operator_estimate_spectral_radius( h_, x.handle(), tmp.handle(), level, iterations, &r ) );
      return r;
   }
   template < typename V >
   void smooth_jac( const P1Function< V >& dst, const P1Function< V >& rhs, const P1Function< V >& src, V relax, int level,
                    DoFType flag ) const
   {
      hybCheck( hyb_operator_smooth_jac( h_, dst.handle(), rhs.handle(), src.handle(), double( relax ), level, flag, nullptr ) );
   }

 protected:
   hyb_operator* h_ = nullptr;
};

class P1ConstantLaplaceOperator : public P1OperatorBase
{
 public:
   using srcType = P1Function< double >;
   P1ConstantLaplaceOperator( const std::shared_ptr< PrimitiveStorage >& storage, int minLevel, int maxLevel )
   {
      hybCheck( hyb_operator_create_laplace( storage->handle(), minLevel, maxLevel, &h_ ) );
   }
};

// P1ElementwiseOperator< forms::p1_div_k_grad_affine_q3 > with the coefficient as a callback
/// Where the coefficient callback is evaluated: at every micro-vertex (its P1 interpolant
/// integrated exactly; the fast default), or at the 5 quadrature points of every micro-tet as
/// the reference's p1_div_k_grad_affine_q3 form does (the reference's element matrices).
enum class CoefficientAt
{
   Vertices,
   QuadraturePoints
};

class P1ElementwiseDivKGradOperator : public P1OperatorBase
{
 public:
   using srcType = P1Function< double >;
   P1ElementwiseDivKGradOperator( const std::shared_ptr< PrimitiveStorage >& storage, int minLevel, int maxLevel,
                                  double ( *k )( const double* xyz, void* ctx ), void* ctx = nullptr,
                                  CoefficientAt at = CoefficientAt::Vertices )
   {
      if ( at == CoefficientAt::QuadraturePoints )
         hybCheck( hyb_operator_create_divkgrad_callback_quadrature( storage->handle(), minLevel, maxLevel, k, ctx, &h_ ) );
      else
         hybCheck( hyb_operator_create_divkgrad_callback( storage->handle(), minLevel, maxLevel, k, ctx, &h_ ) );
   }
};

/// P1ElementwiseBlendingDivKGradOperator on a spherical-shell storage whose cells carry the
/// IcosahedralShellMap (the reference sets it with IcosahedralShellMap::setMap); the
/// coefficient is k(y) = exp( alpha (1 - |y|) ) at the mapped quadrature points, alpha = 0
/// gives the shell's Laplacian. Levels up to 7.
class P1ElementwiseBlendingDivKGradOperator : public P1OperatorBase
{
 public:
   using srcType = P1Function< double >;
   P1ElementwiseBlendingDivKGradOperator( const std::shared_ptr< PrimitiveStorage >& storage, int minLevel, int maxLevel,
                                          double alpha = 0.0 )
   {
      hybCheck( hyb_operator_create_blend_divkgrad( storage->handle(), minLevel, maxLevel, alpha, &h_ ) );
   }
};

template < typename V = double >
class P1toP1LinearProlongation
{
 public:
   void prolongate( const P1Function< V >& f, int sourceLevel, DoFType flag ) const
   {
      hybCheck( hyb_prolongate( f.handle(), sourceLevel, flag, HYB_REPLACE, nullptr ) );
   }
   void prolongateAndAdd( const P1Function< V >& f, int sourceLevel, DoFType flag ) const
   {
      hybCheck( hyb_prolongate( f.handle(), sourceLevel, flag, HYB_ADD, nullptr ) );
   }
};

template < typename V = double >
class P1toP1LinearRestriction
{
 public:
   void restrict( const P1Function< V >& f, int sourceLevel, DoFType flag ) const
   {
      hybCheck( hyb_restrict( f.handle(), sourceLevel, flag, nullptr ) );
   }
};

template < typename OperatorType >
class CGSolver
{
 public:
   CGSolver( const std::shared_ptr< PrimitiveStorage >&, int, int, int maxIter = 100000, double tolerance = 1e-16 )
   : maxIter_( maxIter )
   , tol_( tolerance )
   {}
   void solve( const OperatorType& A, const P1Function< double >& x, const P1Function< double >& b, int level )
   {
      int it = 0, conv = 0;
      hybCheck( hyb_cg_solve( A.handle(), x.handle(), b.handle(), level, tol_, maxIter_, &it, &conv, nullptr ) );
      iterations_ = it;
   }
   int iterations() const { return iterations_; }

 private:
   int    maxIter_;
   double tol_;
   int    iterations_ = 0;
};

enum class CycleType
{
   VCYCLE = HYB_CYCLE_V,
   WCYCLE = HYB_CYCLE_W
};

// V- or W-cycle with SOR smoothing (SORSmoother, relax; HYB_SMOOTHER_SYMMETRIC_SOR for
// SymmetricSORSmoother, HYB_SMOOTHER_JACOBI for WeightedJacobiSmoother;
// HYB_SMOOTHER_SOR_REFERENCE_ORDER and HYB_SMOOTHER_SYMMETRIC_SOR_REFERENCE_ORDER for the two
// SOR smoothers in the reference's sweep order) and an FP64 CG coarse solve.
template < typename OperatorType >
class GeometricMultigridSolver
{
 public:
   GeometricMultigridSolver( const std::shared_ptr< PrimitiveStorage >& storage, const OperatorType& A, int minLevel,
                             int maxLevel, int preSmoothSteps = 3, int postSmoothSteps = 3, double sorRelax = 1.0,
                             double coarseTolerance = 1e-12, int coarseMaxIter = 10000, CycleType cycleType = CycleType::VCYCLE,
                             int smoother = HYB_SMOOTHER_SOR )
   {
      hybCheck( hyb_gmg_create( storage->handle(), A.handle(), minLevel, maxLevel, preSmoothSteps, postSmoothSteps, sorRelax,
                                smoother, coarseTolerance, coarseMaxIter, &h_ ) );
      if ( cycleType != CycleType::VCYCLE )
         hybCheck( hyb_gmg_set_cycle_type( h_, int( cycleType ) ) );
   }
   ~GeometricMultigridSolver() { hyb_gmg_destroy( h_ ); }
   GeometricMultigridSolver( const GeometricMultigridSolver& )            = delete;
   GeometricMultigridSolver& operator=( const GeometricMultigridSolver& ) = delete;

   // one cycle (GeometricMultigridSolver::solve); the coarser levels of b are scratch
   void solve( const OperatorType&, const P1Function< double >& x, const P1Function< double >& b, int level )
   {
      hybCheck( hyb_gmg_solve( h_, x.handle(), b.handle(), level, nullptr ) );
   }
   // FullMultigridSolver::solve with cyclesPerLevel cycles per level; b is needed on every level
   void solveFullMultigrid( const P1Function< double >& x, const P1Function< double >& b, int level, int cyclesPerLevel = 1 )
   {
      hybCheck( hyb_gmg_solve_fmg( h_, x.handle(), b.handle(), level, cyclesPerLevel, nullptr ) );
   }
   // ChebyshevSmoother::setupCoefficients(order, spectralRadius) for a solver created with
   // HYB_SMOOTHER_CHEBYSHEV
   void setupChebyshev( int order, double spectralRadius )
   {
      hybCheck( hyb_gmg_setup_chebyshev( h_, order, 0.3 * spectralRadius, 1.2 * spectralRadius ) );
   }
   // cycles until ||b - Ax|| / ||b|| <= relTol; precision 64 (FP64) or 32 (FP32 inner cycles)
   std::vector< double > solveToTolerance( const P1Function< double >& x, const P1Function< double >& b, int level,
                                           double relTol, int maxCycles = 100, int precision = 64 )
   {
      std::vector< double > hist( size_t( maxCycles ) + 1 );
      int                   cyc = 0;
      hybCheck( hyb_gmg_solve_to_tolerance( h_, x.handle(), b.handle(), level, relTol, maxCycles, precision, hist.data(), &cyc,
                                            nullptr ) );
      hist.resize( size_t( cyc ) + 1 );
      return hist;
   }

 private:
   hyb_gmg* h_ = nullptr;
};

} // namespace hyteg
