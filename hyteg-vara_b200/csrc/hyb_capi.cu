// Host engine and C ABI of the B200 P1 multigrid path (declarations and the
// reference interface each entry point replaces: include/hyteg_b200.h). One translation
// unit: hyb_storage.inl (storage, functions, operators), hyb_launch.inl (launchers, row
// tables, CG), hyb_gmg.inl (multigrid, program kernel, graphs), the C ABI below, and
// hyb_server.inl (serving loop).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../include/hyteg_b200.h"
#include "hyb_kernels.cuh"
#include "hyb_program.cuh"
#include "topology.hpp"

namespace hyb {

thread_local std::string g_lastError;

struct Error : std::runtime_error
{
   int code;
   Error( int c, const std::string& m ) : std::runtime_error( m ), code( c ) {}
};

#define HYB_CUDA( call )                                                                                              \
   do                                                                                                                 \
   {                                                                                                                  \
      cudaError_t e_ = ( call );                                                                                      \
      if ( e_ != cudaSuccess )                                                                                        \
         throw Error( e_ == cudaErrorMemoryAllocation ? HYB_ENOMEM : HYB_EDEVICE,                                     \
                      std::string( #call ) + ": " + cudaGetErrorString( e_ ) );                                       \
   } while ( 0 )

// Kernels enqueued by this library (graph replays add the kernel nodes they hold).
std::atomic< long long > g_launches{ 0 };

#define HYB_CHECK_LAUNCH()                                                                                            \
   do                                                                                                                 \
   {                                                                                                                  \
      HYB_CUDA( cudaGetLastError() );                                                                                 \
      g_launches.fetch_add( 1, std::memory_order_relaxed );                                                          \
   } while ( 0 )

// Device bytes currently held by this library's buffers and functions (footprint accounting).
std::atomic< long long > g_deviceBytes{ 0 };

inline void require( bool c, const std::string& msg )
{
   if ( !c )
      throw Error( HYB_EINVAL, msg );
}

// Launch with programmatic stream serialization (the kernels' prologue waits for the
// predecessor): consecutive kernels of a stream or a captured graph overlap their launch
// latency with the predecessor's tail.
template < typename... KArgs, typename... Args >
void pdlLaunch( void ( *kernel )( KArgs... ), dim3 grid, dim3 block, size_t smem, cudaStream_t stream, Args&&... args )
{
   cudaLaunchConfig_t  c{};
   cudaLaunchAttribute a{};
   a.id                                         = cudaLaunchAttributeProgrammaticStreamSerialization;
   a.val.programmaticStreamSerializationAllowed = 1;
   c.gridDim                                    = grid;
   c.blockDim                                   = block;
   c.dynamicSmemBytes                           = smem;
   c.stream                                     = stream;
   c.attrs                                      = &a;
   c.numAttrs                                   = 1;
   HYB_CUDA( cudaLaunchKernelEx( &c, kernel, std::forward< Args >( args )... ) );
}

template < typename T >
struct DevBuf
{
   T*     p = nullptr;
   size_t n = 0;
   DevBuf() = default;
   DevBuf( const DevBuf& ) = delete;
   DevBuf& operator=( const DevBuf& ) = delete;
   ~DevBuf() { release(); }
   void release()
   {
      if ( p )
      {
         cudaFree( p );
         g_deviceBytes.fetch_sub( (long long) ( n * sizeof( T ) ) );
      }
      p = nullptr;
      n = 0;
   }
   void alloc( size_t count )
   {
      release();
      if ( count == 0 )
         count = 1;
      HYB_CUDA( cudaMalloc( &p, count * sizeof( T ) ) );
      n = count;
      g_deviceBytes.fetch_add( (long long) ( n * sizeof( T ) ) );
   }
   void upload( const std::vector< T >& v )
   {
      alloc( v.size() );
      if ( !v.empty() )
         HYB_CUDA( cudaMemcpy( p, v.data(), v.size() * sizeof( T ), cudaMemcpyHostToDevice ) );
   }
};

inline cudaStream_t S( void* s ) { return reinterpret_cast< cudaStream_t >( s ); }

#include "hyb_storage.inl"
#include "hyb_launch.inl"
#include "hyb_gmg.inl"

} // namespace hyb

// ===========================================================================
// C ABI
// ===========================================================================
using namespace hyb;

struct hyb_storage_s : Storage
{};
struct hyb_function_s : Function
{};
struct hyb_operator_s : Operator
{};
struct hyb_gmg_s : Gmg
{};

#define HYB_API_BEGIN try {
#define HYB_API_END                                                                                                   \
   return HYB_OK;                                                                                                     \
   }                                                                                                                  \
   catch ( const Error& e )                                                                                           \
   {                                                                                                                  \
      g_lastError = e.what();                                                                                         \
      return e.code;                                                                                                  \
   }                                                                                                                  \
   catch ( const std::invalid_argument& e )                                                                           \
   {                                                                                                                  \
      g_lastError = e.what();                                                                                         \
      return HYB_EINVAL;                                                                                              \
   }                                                                                                                  \
   catch ( const std::exception& e )                                                                                  \
   {                                                                                                                  \
      g_lastError = e.what();                                                                                         \
      return HYB_EUNSUPPORTED;                                                                                        \
   }

static Storage*  ST( hyb_storage* s ) { return static_cast< Storage* >( s ); }
static Function* FN( hyb_function* f ) { return static_cast< Function* >( f ); }
static Operator* OP( hyb_operator* o ) { return static_cast< Operator* >( o ); }

static void sameStorage( const Function* a, const Function* b )
{
   require( a && b && a->st == b->st, "functions belong to different storages" );
}

extern "C" {

const char* hyb_last_error( void ) { return g_lastError.c_str(); }

long long hyb_kernel_launch_count( void ) { return g_launches.load(); }

int hyb_storage_create( const double* coords, int64_t nv, const int64_t* tets, int64_t nt, int maxLevel, hyb_storage** out )
{
   HYB_API_BEGIN
   require( coords && tets && out && nv >= 4 && nt >= 1, "invalid mesh arguments" );
   std::vector< std::array< double, 3 > > V( nv );
   for ( int64_t i = 0; i < nv; ++i )
      V[i] = { coords[3 * i], coords[3 * i + 1], coords[3 * i + 2] };
   std::vector< std::array< int, 4 > > T( nt );
   for ( int64_t i = 0; i < nt; ++i )
      for ( int k = 0; k < 4; ++k )
         T[i][k] = int( tets[4 * i + k] );
   auto s = std::make_unique< hyb_storage_s >();
   buildStorage( *s, V, T, maxLevel );
   *out = s.release();
   HYB_API_END
}

int hyb_storage_create_from_gmsh( const char* path, int maxLevel, hyb_storage** out )
{
   HYB_API_BEGIN
   require( path && out, "null argument" );
   std::vector< std::array< double, 3 > > V;
   std::vector< std::array< int, 4 > >    T;
   readGmsh( path, V, T );
   auto s = std::make_unique< hyb_storage_s >();
   buildStorage( *s, V, T, maxLevel );
   *out = s.release();
   HYB_API_END
}

int hyb_storage_create_spherical_shell( int ntan, int nrad, double rmin, double rmax, int maxLevel, hyb_storage** out )
{
   HYB_API_BEGIN
   require( out, "null argument" );
   std::vector< std::array< double, 3 > > V;
   std::vector< std::array< int, 4 > >    T;
   meshSphericalShell( ntan, nrad, rmin, rmax, V, T );
   auto s = std::make_unique< hyb_storage_s >();
   buildStorage( *s, V, T, maxLevel );
   *out = s.release();
   HYB_API_END
}

int hyb_storage_create_cuboid( int nx, int ny, int nz, const double* lo, const double* hi, int maxLevel, hyb_storage** out )
{
   HYB_API_BEGIN
   require( lo && hi && out, "null argument" );
   std::vector< std::array< double, 3 > > V;
   std::vector< std::array< int, 4 > >    T;
   meshCuboid( nx, ny, nz, lo, hi, V, T );
   auto s = std::make_unique< hyb_storage_s >();
   buildStorage( *s, V, T, maxLevel );
   *out = s.release();
   HYB_API_END
}

int hyb_storage_destroy( hyb_storage* s )
{
   HYB_API_BEGIN
   delete static_cast< hyb_storage_s* >( s );
   HYB_API_END
}

int hyb_storage_counts( const hyb_storage* s, int64_t* c )
{
   HYB_API_BEGIN
   require( s && c, "null argument" );
   const auto& tp = s->topo;
   c[0] = int64_t( tp.V.size() );
   c[1] = int64_t( tp.E.size() );
   c[2] = int64_t( tp.F.size() );
   c[3] = int64_t( tp.T.size() );
   HYB_API_END
}

int64_t hyb_storage_num_dofs( const hyb_storage* s, int level )
{
   if ( !s || level < 0 || level > s->maxLevel )
      return -1;
   return s->topo.numDofs( level );
}

int hyb_storage_mesh( const hyb_storage* s, double* coords, int64_t* tets )
{
   HYB_API_BEGIN
   require( s && coords && tets, "null argument" );
   for ( size_t i = 0; i < s->topo.V.size(); ++i )
      for ( int d = 0; d < 3; ++d )
         coords[3 * i + d] = s->topo.V[i][d];
   for ( size_t i = 0; i < s->topo.T.size(); ++i )
      for ( int k = 0; k < 4; ++k )
         tets[4 * i + k] = s->topo.T[i][k];
   HYB_API_END
}

int hyb_storage_colouring( const hyb_storage* s, int* m, int* labels )
{
   HYB_API_BEGIN
   require( s && m, "null argument" );
   *m = s->topo.colours;
   if ( labels )
      std::copy( s->topo.labels.begin(), s->topo.labels.end(), labels );
   HYB_API_END
}

int hyb_function_create( hyb_storage* s, int minL, int maxL, int dtype, hyb_function** out )
{
   HYB_API_BEGIN
   require( s && out, "null argument" );
   Function* f = makeFunction( ST( s ), minL, maxL, dtype );
   // re-home into the ABI type (same layout, no extra members)
   *out = reinterpret_cast< hyb_function* >( f );
   HYB_API_END
}

int hyb_function_destroy( hyb_function* f )
{
   HYB_API_BEGIN
   delete FN( f );
   HYB_API_END
}

static void checkLevel( const Function* f, int l ) { (void) f->at( l ); }

int hyb_function_upload( hyb_function* fh, int level, const void* host, void* stream )
{
   HYB_API_BEGIN
   Function* f = FN( fh );
   require( f && host, "null argument" );
   checkLevel( f, level );
   const size_t n   = size_t( f->st->topo.numDofs( level ) ) * f->elem();
   char*        tmp = f->st->stage( n );
   HYB_CUDA( cudaMemcpyAsync( tmp, host, n, cudaMemcpyHostToDevice, S( stream ) ) );
   if ( f->dtype == HYB_F64 )
      launchFromDofs< double >( *f->st, level, f->ptr< double >( level ), reinterpret_cast< double* >( tmp ), S( stream ) );
   else
      launchFromDofs< float >( *f->st, level, f->ptr< float >( level ), reinterpret_cast< float* >( tmp ), S( stream ) );
   HYB_CUDA( cudaStreamSynchronize( S( stream ) ) );
   HYB_API_END
}

int hyb_function_download( hyb_function* fh, int level, void* host, void* stream )
{
   HYB_API_BEGIN
   Function* f = FN( fh );
   require( f && host, "null argument" );
   checkLevel( f, level );
   const size_t n   = size_t( f->st->topo.numDofs( level ) ) * f->elem();
   char*        tmp = f->st->stage( n );
   if ( f->dtype == HYB_F64 )
      launchToDofs< double >( *f->st, level, f->ptr< double >( level ), reinterpret_cast< double* >( tmp ), S( stream ) );
   else
      launchToDofs< float >( *f->st, level, f->ptr< float >( level ), reinterpret_cast< float* >( tmp ), S( stream ) );
   HYB_CUDA( cudaMemcpyAsync( host, tmp, n, cudaMemcpyDeviceToHost, S( stream ) ) );
   HYB_CUDA( cudaStreamSynchronize( S( stream ) ) );
   HYB_API_END
}

int hyb_function_upload_device( hyb_function* fh, int level, const void* dev, void* stream )
{
   HYB_API_BEGIN
   Function* f = FN( fh );
   require( f && dev, "null argument" );
   checkLevel( f, level );
   if ( f->dtype == HYB_F64 )
      launchFromDofs< double >( *f->st, level, f->ptr< double >( level ), static_cast< const double* >( dev ), S( stream ) );
   else
      launchFromDofs< float >( *f->st, level, f->ptr< float >( level ), static_cast< const float* >( dev ), S( stream ) );
   HYB_API_END
}

int hyb_function_download_device( hyb_function* fh, int level, void* dev, void* stream )
{
   HYB_API_BEGIN
   Function* f = FN( fh );
   require( f && dev, "null argument" );
   checkLevel( f, level );
   if ( f->dtype == HYB_F64 )
      launchToDofs< double >( *f->st, level, f->ptr< double >( level ), static_cast< double* >( dev ), S( stream ) );
   else
      launchToDofs< float >( *f->st, level, f->ptr< float >( level ), static_cast< float* >( dev ), S( stream ) );
   HYB_API_END
}

int hyb_function_interpolate_const( hyb_function* fh, int level, double value, int flag, void* stream )
{
   HYB_API_BEGIN
   Function* f = FN( fh );
   require( f, "null argument" );
   checkLevel( f, level );
   const auto& L = f->st->L( level );
   if ( value == 0.0 && flag == HYB_ALL )
      HYB_CUDA( cudaMemsetAsync( f->at( level ), 0, f->levelBytes( level ), S( stream ) ) );
   else if ( f->dtype == HYB_F64 )
      k_fill< double ><<< dim3( L.slabBlocks, f->st->td.nC ), 256, 0, S( stream ) >>>( f->st->td, L.dev,
                                                                                      f->ptr< double >( level ), value, flag );
   else
      k_fill< float ><<< dim3( L.slabBlocks, f->st->td.nC ), 256, 0, S( stream ) >>>( f->st->td, L.dev,
                                                                                     f->ptr< float >( level ), float( value ),
                                                                                     flag );
   HYB_CHECK_LAUNCH();
   HYB_API_END
}

int hyb_function_fill_uniform_random( hyb_function* fh, int level, uint64_t seed, double lattice, void* stream )
{
   HYB_API_BEGIN
   Function* f = FN( fh );
   require( f, "null argument" );
   require( lattice > 0.0, "lattice must be positive" );
   checkLevel( f, level );
   const Storage& st = *f->st;
   const auto&    L  = st.L( level );
   if ( f->dtype == HYB_F64 )
      k_fill_uniform_hash< double ><<< dim3( L.slabBlocks, st.td.nC ), 256, 0, S( stream ) >>>(
          st.td, L.dev, st.cellCoords.p, st.cellOrder.p, f->ptr< double >( level ), seed, lattice );
   else
      k_fill_uniform_hash< float ><<< dim3( L.slabBlocks, st.td.nC ), 256, 0, S( stream ) >>>(
          st.td, L.dev, st.cellCoords.p, st.cellOrder.p, f->ptr< float >( level ), seed, lattice );
   HYB_CHECK_LAUNCH();
   HYB_API_END
}

static int lincombApi( hyb_function* fh, int level, int n, const double* sc, hyb_function* const* srcs, int flag,
                       void* stream, bool add )
{
   HYB_API_BEGIN
   Function* f = FN( fh );
   require( f && ( n == 0 || ( sc && srcs ) ), "null argument" );
   require( n >= 0 && n <= 3, "at most three source functions" );
   checkLevel( f, level );
   for ( int i = 0; i < n; ++i )
   {
      sameStorage( f, FN( srcs[i] ) );
      require( FN( srcs[i] )->dtype == f->dtype, "source and destination dtypes differ" );
      checkLevel( FN( srcs[i] ), level );
   }
   if ( f->dtype == HYB_F64 )
   {
      const double* p[3] = { nullptr, nullptr, nullptr };
      for ( int i = 0; i < n; ++i )
         p[i] = FN( srcs[i] )->ptr< double >( level );
      launchLincomb< double >( *f->st, level, f->ptr< double >( level ), n, sc, p, add, flag, S( stream ) );
   }
   else
   {
      const float* p[3] = { nullptr, nullptr, nullptr };
      for ( int i = 0; i < n; ++i )
         p[i] = FN( srcs[i] )->ptr< float >( level );
      launchLincomb< float >( *f->st, level, f->ptr< float >( level ), n, sc, p, add, flag, S( stream ) );
   }
   HYB_API_END
}

int hyb_function_assign( hyb_function* f, int level, int n, const double* sc, hyb_function* const* srcs, int flag,
                         void* stream )
{
   return lincombApi( f, level, n, sc, srcs, flag, stream, false );
}

int hyb_function_add( hyb_function* f, int level, int n, const double* sc, hyb_function* const* srcs, int flag, void* stream )
{
   return lincombApi( f, level, n, sc, srcs, flag, stream, true );
}

int hyb_function_dot( hyb_function* ah, hyb_function* bh, int level, int flag, double* out, void* stream )
{
   HYB_API_BEGIN
   Function *a = FN( ah ), *b = FN( bh );
   require( out, "null argument" );
   sameStorage( a, b );
   require( a->dtype == b->dtype, "dtypes differ" );
   checkLevel( a, level );
   checkLevel( b, level );
   if ( a->dtype == HYB_F64 )
      launchDot< double >( *a->st, level, a->ptr< double >( level ), b->ptr< double >( level ), flag, 1, S( stream ) );
   else
      launchDot< float >( *a->st, level, a->ptr< float >( level ), b->ptr< float >( level ), flag, 1, S( stream ) );
   HYB_CUDA( cudaMemcpyAsync( a->st->hostScalar, a->st->scalars.p + 1, sizeof( double ), cudaMemcpyDeviceToHost, S( stream ) ) );
   HYB_CUDA( cudaStreamSynchronize( S( stream ) ) );
   *out = a->st->hostScalar[0];
   HYB_API_END
}

int hyb_function_copy_convert( hyb_function* dh, hyb_function* sh, int level, void* stream )
{
   HYB_API_BEGIN
   Function *d = FN( dh ), *s = FN( sh );
   sameStorage( d, s );
   checkLevel( d, level );
   checkLevel( s, level );
   if ( d->dtype == HYB_F64 && s->dtype == HYB_F32 )
      launchConvert< double, float >( *d->st, level, d->ptr< double >( level ), s->ptr< float >( level ), S( stream ) );
   else if ( d->dtype == HYB_F32 && s->dtype == HYB_F64 )
      launchConvert< float, double >( *d->st, level, d->ptr< float >( level ), s->ptr< double >( level ), S( stream ) );
   else
      HYB_CUDA( cudaMemcpyAsync( d->at( level ), s->at( level ), d->levelBytes( level ), cudaMemcpyDeviceToDevice,
                                 S( stream ) ) );
   HYB_API_END
}

int hyb_operator_create_laplace( hyb_storage* s, int minL, int maxL, hyb_operator** out )
{
   HYB_API_BEGIN
   require( s && out, "null argument" );
   *out = reinterpret_cast< hyb_operator* >( makeLaplace( ST( s ), minL, maxL ) );
   HYB_API_END
}

int hyb_operator_create_divkgrad( hyb_storage* s, int minL, int maxL, const double* const* nodal, hyb_operator** out )
{
   HYB_API_BEGIN
   require( s && out && nodal, "null argument" );
   std::vector< std::vector< double > > k;
   for ( int l = minL; l <= maxL; ++l )
   {
      require( nodal[l - minL] != nullptr, "missing nodal coefficient level" );
      const int64_t n = ST( s )->topo.numDofs( l );
      k.emplace_back( nodal[l - minL], nodal[l - minL] + n );
   }
   *out = reinterpret_cast< hyb_operator* >( makeDivKGrad( ST( s ), minL, maxL, k ) );
   HYB_API_END
}

int hyb_operator_create_divkgrad_callback( hyb_storage* s, int minL, int maxL, double ( *kfun )( const double*, void* ),
                                           void* ctx, hyb_operator** out )
{
   HYB_API_BEGIN
   require( s && out && kfun, "null argument" );
   require( minL >= 0 && minL <= maxL && maxL <= ST( s )->maxLevel, "invalid level range" );
   const Topology& tp = ST( s )->topo;
   std::vector< std::vector< double > > k;
   for ( int l = minL; l <= maxL; ++l )
   {
      std::vector< double > xyz;
      dofCoords( tp, l, xyz );
      std::vector< double > kv( xyz.size() / 3 );
      for ( size_t i = 0; i < kv.size(); ++i )
         kv[i] = kfun( &xyz[3 * i], ctx );
      k.push_back( std::move( kv ) );
   }
   *out = reinterpret_cast< hyb_operator* >( makeDivKGrad( ST( s ), minL, maxL, k ) );
   HYB_API_END
}

int hyb_operator_create_divkgrad_callback_quadrature( hyb_storage* s, int minL, int maxL,
                                                      double ( *kfun )( const double*, void* ), void* ctx,
                                                      hyb_operator** out )
{
   HYB_API_BEGIN
   require( s && out && kfun, "null argument" );
   require( minL >= 0 && minL <= maxL && maxL <= ST( s )->maxLevel, "invalid level range" );
   *out = reinterpret_cast< hyb_operator* >( makeDivKGradCallbackQuadrature( ST( s ), minL, maxL, kfun, ctx ) );
   HYB_API_END
}

int hyb_operator_create_divkgrad_quadrature( hyb_storage* s, int minL, int maxL, int kind, const double* w,
                                             const double* phase, int modes, double sigma, double radial,
                                             hyb_operator** out )
{
   HYB_API_BEGIN
   require( s && out, "null argument" );
   require( kind == 1 || kind == 2, "coefficient kind must be 1 (tanh) or 2 (random features)" );
   if ( kind == 2 )
   {
      require( w && phase, "null argument" );
      require( modes > 0 && modes <= 4096, "modes must be in [1, 4096]" );
   }
   *out = reinterpret_cast< hyb_operator* >(
       makeDivKGradQuadrature( ST( s ), minL, maxL, kind, w, phase, modes, sigma, radial ) );
   HYB_API_END
}

int hyb_operator_create_divkgrad_rff( hyb_storage* s, int minL, int maxL, const double* w, const double* phase,
                                      int modes, double sigma, double radial, hyb_operator** out )
{
   HYB_API_BEGIN
   require( s && w && phase && out, "null argument" );
   require( modes > 0 && modes <= 4096, "modes must be in [1, 4096]" );
   *out = reinterpret_cast< hyb_operator* >( makeDivKGradRff( ST( s ), minL, maxL, w, phase, modes, sigma, radial ) );
   HYB_API_END
}

int hyb_operator_create_blend_divkgrad( hyb_storage* s, int minL, int maxL, double alpha, hyb_operator** out )
{
   HYB_API_BEGIN
   require( s && out, "null argument" );
   *out = reinterpret_cast< hyb_operator* >( makeBlendDivKGrad( ST( s ), minL, maxL, alpha ) );
   HYB_API_END
}

int hyb_storage_dof_coords( const hyb_storage* s, int level, double* xyz )
{
   HYB_API_BEGIN
   require( s && xyz, "null argument" );
   require( level >= 0 && level <= s->maxLevel, "level out of range" );
   std::vector< double > v;
   dofCoords( s->topo, level, v );
   std::copy( v.begin(), v.end(), xyz );
   HYB_API_END
}

int hyb_operator_destroy( hyb_operator* op )
{
   HYB_API_BEGIN
   delete OP( op );
   HYB_API_END
}

static void checkOpFn( const Operator* op, const Function* f, int level )
{
   require( op && f, "null argument" );
   require( op->st == f->st, "operator and function belong to different storages" );
   require( level >= op->minL && level <= op->maxL, "level outside the operator's level range" );
   checkLevel( f, level );
}

int hyb_operator_apply( hyb_operator* oh, hyb_function* sh, hyb_function* dh, int level, int flag, int update, void* stream )
{
   HYB_API_BEGIN
   Operator* op = OP( oh );
   Function *src = FN( sh ), *dst = FN( dh );
   checkOpFn( op, src, level );
   checkOpFn( op, dst, level );
   require( src != dst, "apply needs distinct src and dst (reference: WALBERLA_ASSERT_NOT_IDENTICAL)" );
   require( src->dtype == dst->dtype, "dtypes differ" );
   require( update == HYB_REPLACE || update == HYB_ADD, "invalid update type" );
   const int mode = update == HYB_ADD ? kAdd : kReplace;
   if ( src->dtype == HYB_F64 )
      launchApply< double >( *op, level, src->ptr< double >( level ), dst->ptr< double >( level ), nullptr, flag, mode, S( stream ) );
   else
      launchApply< float >( *op, level, src->ptr< float >( level ), dst->ptr< float >( level ), nullptr, flag, mode, S( stream ) );
   HYB_API_END
}

int hyb_operator_residual( hyb_operator* oh, hyb_function* xh, hyb_function* bh, hyb_function* rh, int level, int flag,
                           void* stream )
{
   HYB_API_BEGIN
   Operator* op = OP( oh );
   Function *x = FN( xh ), *b = FN( bh ), *r = FN( rh );
   checkOpFn( op, x, level );
   checkOpFn( op, b, level );
   checkOpFn( op, r, level );
   require( x != r && b != r, "residual needs a separate output function" );
   require( x->dtype == b->dtype && x->dtype == r->dtype, "dtypes differ" );
   if ( x->dtype == HYB_F64 )
      launchApply< double >( *op, level, x->ptr< double >( level ), r->ptr< double >( level ), b->ptr< double >( level ), flag,
                             kResidual, S( stream ) );
   else
      launchApply< float >( *op, level, x->ptr< float >( level ), r->ptr< float >( level ), b->ptr< float >( level ), flag,
                            kResidual, S( stream ) );
   HYB_API_END
}

int hyb_operator_smooth_sor( hyb_operator* oh, hyb_function* dh, hyb_function* rh, double relax, int level, int flag,
                             void* stream )
{
   HYB_API_BEGIN
   Operator* op = OP( oh );
   Function *u = FN( dh ), *b = FN( rh );
   checkOpFn( op, u, level );
   checkOpFn( op, b, level );
   require( u != b, "smooth_sor needs distinct dst and rhs" );
   require( u->dtype == b->dtype, "dtypes differ" );
   if ( u->dtype == HYB_F64 )
      launchSor< double >( *op, level, u->ptr< double >( level ), b->ptr< double >( level ), relax, flag, S( stream ) );
   else
      launchSor< float >( *op, level, u->ptr< float >( level ), b->ptr< float >( level ), float( relax ), flag, S( stream ) );
   HYB_API_END
}

int hyb_operator_smooth_sor_backwards( hyb_operator* oh, hyb_function* dh, hyb_function* rh, double relax, int level,
                                       int flag, void* stream )
{
   HYB_API_BEGIN
   Operator* op = OP( oh );
   Function *u = FN( dh ), *b = FN( rh );
   checkOpFn( op, u, level );
   checkOpFn( op, b, level );
   require( u != b, "smooth_sor_backwards needs distinct dst and rhs" );
   require( u->dtype == b->dtype, "dtypes differ" );
   if ( u->dtype == HYB_F64 )
      launchSor< double >( *op, level, u->ptr< double >( level ), b->ptr< double >( level ), relax, flag, S( stream ), true );
   else
      launchSor< float >( *op, level, u->ptr< float >( level ), b->ptr< float >( level ), float( relax ), flag, S( stream ),
                          true );
   HYB_API_END
}

int hyb_operator_smooth_sor_reference_order( hyb_operator* oh, hyb_function* dh, hyb_function* rh, double relax,
                                             int level, int flag, int backwards, void* stream )
{
   HYB_API_BEGIN
   Operator* op = OP( oh );
   Function *u = FN( dh ), *b = FN( rh );
   checkOpFn( op, u, level );
   checkOpFn( op, b, level );
   require( u != b, "smooth_sor_reference_order needs distinct dst and rhs" );
   require( u->dtype == b->dtype, "dtypes differ" );
   if ( u->dtype == HYB_F64 )
      launchSorReference< double >( *op, level, u->ptr< double >( level ), b->ptr< double >( level ), relax, flag,
                                    op->st->snapScratch< double >( level ),
                                    op->st->sorCoefScratch< double >( sorRefCoefElems( *op->st, level ) ), S( stream ),
                                    backwards != 0 );
   else
      launchSorReference< float >( *op, level, u->ptr< float >( level ), b->ptr< float >( level ), float( relax ), flag,
                                   op->st->snapScratch< float >( level ),
                                   op->st->sorCoefScratch< float >( sorRefCoefElems( *op->st, level ) ), S( stream ),
                                   backwards != 0 );
   HYB_API_END
}

int hyb_operator_smooth_jac( hyb_operator* oh, hyb_function* dh, hyb_function* rh, hyb_function* sh, double relax, int level,
                             int flag, void* stream )
{
   HYB_API_BEGIN
   Operator* op = OP( oh );
   Function *d = FN( dh ), *b = FN( rh ), *s = FN( sh );
   checkOpFn( op, d, level );
   checkOpFn( op, b, level );
   checkOpFn( op, s, level );
   require( d != s, "smooth_jac needs distinct dst and src" );
   require( d->dtype == b->dtype && d->dtype == s->dtype, "dtypes differ" );
   if ( d->dtype == HYB_F64 )
      launchJacobi< double >( *op, level, s->ptr< double >( level ), d->ptr< double >( level ), b->ptr< double >( level ), relax,
                              flag, S( stream ) );
   else
      launchJacobi< float >( *op, level, s->ptr< float >( level ), d->ptr< float >( level ), b->ptr< float >( level ),
                             float( relax ), flag, S( stream ) );
   HYB_API_END
}

int hyb_operator_cell_stencil( const hyb_operator* oh, int level, int cell, int mask, double* out15 )
{
   HYB_API_BEGIN
   const Operator* op = reinterpret_cast< const Operator* >( oh );
   require( op && out15, "null argument" );
   require( !op->variable && !op->blend, "stencils are stored for constant-coefficient operators only" );
   require( level >= op->minL && level <= op->maxL && cell >= 0 && cell < op->st->td.nC && mask >= 0 && mask < 16,
            "index out of range" );
   const auto& st = op->stHost[level - op->minL];
   std::copy( st.begin() + ( size_t( cell ) * 16 + mask ) * 15, st.begin() + ( size_t( cell ) * 16 + mask ) * 15 + 15, out15 );
   HYB_API_END
}

int hyb_prolongate( hyb_function* fh, int src, int flag, int update, void* stream )
{
   HYB_API_BEGIN
   Function* f = FN( fh );
   require( f, "null argument" );
   checkLevel( f, src );
   checkLevel( f, src + 1 );
   require( update == HYB_REPLACE || update == HYB_ADD, "invalid update type" );
   if ( f->dtype == HYB_F64 )
      launchProlongate< double >( *f->st, src, f->ptr< double >( src ), f->ptr< double >( src + 1 ), flag, update == HYB_ADD,
                                  S( stream ) );
   else
      launchProlongate< float >( *f->st, src, f->ptr< float >( src ), f->ptr< float >( src + 1 ), flag, update == HYB_ADD,
                                 S( stream ) );
   HYB_API_END
}

int hyb_restrict( hyb_function* fh, int src, int flag, void* stream )
{
   HYB_API_BEGIN
   Function* f = FN( fh );
   require( f, "null argument" );
   checkLevel( f, src );
   checkLevel( f, src - 1 );
   if ( f->dtype == HYB_F64 )
      launchRestrict< double >( *f->st, src, f->ptr< double >( src ), f->ptr< double >( src - 1 ), flag, S( stream ) );
   else
      launchRestrict< float >( *f->st, src, f->ptr< float >( src ), f->ptr< float >( src - 1 ), flag, S( stream ) );
   HYB_API_END
}

int hyb_cg_solve( hyb_operator* oh, hyb_function* xh, hyb_function* bh, int level, double tol, int maxIter, int* iters,
                  int* converged, void* stream )
{
   HYB_API_BEGIN
   Operator* op = OP( oh );
   Function *x = FN( xh ), *b = FN( bh );
   checkOpFn( op, x, level );
   checkOpFn( op, b, level );
   require( x->dtype == HYB_F64 && b->dtype == HYB_F64, "the CG solver runs in FP64" );
   require( maxIter >= 0, "max_iter must be non-negative" );
   CgScratch cs;
   launchCg( *op, level, x->ptr< double >( level ), b->ptr< double >( level ), cs, tol, maxIter, S( stream ) );
   int st[2] = { 0, 0 };
   HYB_CUDA( cudaMemcpyAsync( st, cs.status.p, 2 * sizeof( int ), cudaMemcpyDeviceToHost, S( stream ) ) );
   HYB_CUDA( cudaStreamSynchronize( S( stream ) ) );
   if ( iters )
      *iters = st[0];
   if ( converged )
      *converged = st[1];
   HYB_API_END
}

int hyb_gmg_create( hyb_storage* s, hyb_operator* oh, int minL, int maxL, int pre, int post, double relax, int smoother,
                    double coarseTol, int coarseMaxIter, hyb_gmg** out )
{
   HYB_API_BEGIN
   Operator* op = OP( oh );
   require( s && op && out, "null argument" );
   require( op->st == ST( s ), "operator belongs to another storage" );
   require( minL >= op->minL && maxL <= op->maxL && minL <= maxL, "GMG levels outside the operator's level range" );
   require( pre >= 0 && post >= 0, "smoothing steps must be non-negative" );
   require( smoother == HYB_SMOOTHER_SOR || smoother == HYB_SMOOTHER_JACOBI || smoother == HYB_SMOOTHER_SYMMETRIC_SOR ||
                smoother == HYB_SMOOTHER_CHEBYSHEV || smoother == HYB_SMOOTHER_SOR_REFERENCE_ORDER ||
                smoother == HYB_SMOOTHER_SYMMETRIC_SOR_REFERENCE_ORDER,
            "unknown smoother" );
   auto g = std::make_unique< hyb_gmg_s >();
   initGmg( *g, ST( s ), op, minL, maxL, pre, post, relax, smoother, coarseTol, coarseMaxIter );
   *out = g.release();
   HYB_API_END
}

int hyb_gmg_destroy( hyb_gmg* g )
{
   HYB_API_BEGIN
   delete static_cast< hyb_gmg_s* >( g );
   HYB_API_END
}

int hyb_gmg_set_timing( hyb_gmg* gh, int enable )
{
   HYB_API_BEGIN
   Gmg* g = static_cast< Gmg* >( static_cast< hyb_gmg_s* >( gh ) );
   require( g != nullptr, "null argument" );
   g->timing = enable != 0;
   HYB_API_END
}

int hyb_gmg_timing_reset( hyb_gmg* gh )
{
   HYB_API_BEGIN
   Gmg* g = static_cast< Gmg* >( static_cast< hyb_gmg_s* >( gh ) );
   require( g != nullptr, "null argument" );
   g->tt.reset();
   HYB_API_END
}

int hyb_gmg_timing_json( hyb_gmg* gh, char* buf, size_t capacity, size_t* length )
{
   HYB_API_BEGIN
   Gmg* g = static_cast< Gmg* >( static_cast< hyb_gmg_s* >( gh ) );
   require( g != nullptr && length != nullptr, "null argument" );
   g->tt.collect();
   std::string out;
   TimingTree::json( g->tt.root, out );
   *length = out.size();
   if ( buf )
   {
      require( capacity > out.size(), "buffer too small for the timing tree (length holds the size needed)" );
      std::memcpy( buf, out.c_str(), out.size() + 1 );
   }
   HYB_API_END
}

int hyb_gmg_set_cycle_type( hyb_gmg* gh, int cycleType )
{
   HYB_API_BEGIN
   Gmg* g = static_cast< Gmg* >( static_cast< hyb_gmg_s* >( gh ) );
   require( g != nullptr, "null argument" );
   require( cycleType == HYB_CYCLE_V || cycleType == HYB_CYCLE_W, "unknown cycle type" );
   if ( cycleType == g->cycleType )
      return HYB_OK;
   // the recorded graphs and coarse-level programs encode the old cycle; drop them once
   // no work that uses them is in flight
   HYB_CUDA( cudaDeviceSynchronize() );
   for ( auto& gr : g->graphs )
      cudaGraphExecDestroy( gr.exec );
   for ( auto& gr : g->loops )
      cudaGraphExecDestroy( gr.exec );
   g->graphs.clear();
   g->loops.clear();
   g->programs.clear();
   g->solvePrograms.clear();
   g->cycleType = cycleType;
   HYB_API_END
}

int hyb_chebyshev_coefficients( int order, double lower, double upper, double* out )
{
   HYB_API_BEGIN
   require( out, "null argument" );
   const auto w = chebyshevCoefficients( order, lower, upper );
   std::copy( w.begin(), w.end(), out );
   HYB_API_END
}

int hyb_gmg_setup_chebyshev( hyb_gmg* gh, int order, double lower, double upper )
{
   HYB_API_BEGIN
   Gmg* g = gh;
   require( g != nullptr, "null argument" );
   require( g->smoother == HYB_SMOOTHER_CHEBYSHEV, "the solver was not created with the Chebyshev smoother" );
   g->cheb = chebyshevCoefficients( order, lower, upper );
   // captured graphs hold the old coefficients
   HYB_CUDA( cudaDeviceSynchronize() );
   for ( auto& gr : g->graphs )
      cudaGraphExecDestroy( gr.exec );
   g->graphs.clear();
   HYB_API_END
}

int hyb_operator_estimate_spectral_radius( hyb_operator* oh, hyb_function* xh, hyb_function* th, int level, int iterations,
                                           double* radius )
{
   HYB_API_BEGIN
   Operator* op = OP( oh );
   Function *x = FN( xh ), *t = FN( th );
   require( radius && iterations >= 1, "null argument or no iteration" );
   checkOpFn( op, x, level );
   checkOpFn( op, t, level );
   require( x != t && x->dtype == HYB_F64 && t->dtype == HYB_F64, "two distinct FP64 functions are needed" );
   Storage&          s   = *op->st;
   const long long   n   = (long long) s.td.nC * s.L( level ).dev.stride;
   std::unique_ptr< Function > inv( makeFunction( &s, level, level, HYB_F64 ) );
   std::unique_ptr< Function > zero( makeFunction( &s, level, level, HYB_F64 ) );
   launchInvDiag< double >( *op, level, zero->ptr< double >( level ), inv->ptr< double >( level ), nullptr );
   double*       xp = x->ptr< double >( level );
   double*       tp = t->ptr< double >( level );
   const double* ip = inv->ptr< double >( level );
   auto dot = [&]( const double* a, const double* b ) {
      launchDot< double >( s, level, a, b, HYB_ALL, 1, nullptr );
      HYB_CUDA( cudaMemcpy( s.hostScalar, s.scalars.p + 1, sizeof( double ), cudaMemcpyDeviceToHost ) );
      return s.hostScalar[0];
   };
   // scale the slab: every replica and the zero padding alike
   auto scale = [&]( double* dst, const double* src, double a ) {
      const int g = int( std::max< long long >( 1, std::min< long long >( ( n + 255 ) / 256, (long long) s.numSMs * 8 ) ) );
      k_scale_copy<<< g, 256 >>>( n, src, dst, a );
      HYB_CHECK_LAUNCH();
   };
   // D^-1 A on All (chebyshev::InvDiagOperatorWrapper::apply)
   auto invDiagA = [&]( const double* src, double* dst ) {
      launchApply< double >( *op, level, src, dst, nullptr, HYB_ALL, kReplace, nullptr );
      const int g = int( std::max< long long >( 1, std::min< long long >( ( n + 255 ) / 256, (long long) s.numSMs * 8 ) ) );
      k_mul<<< g, 256 >>>( n, ip, dst );
      HYB_CHECK_LAUNCH();
   };
   // estimateSpectralRadiusWithPowerIteration (SpectrumEstimation.hpp:57-81)
   double norm = std::sqrt( dot( xp, xp ) );
   scale( xp, xp, 1.0 / norm );
   invDiagA( xp, tp );
   double r = 0;
   for ( int it = 1; it <= iterations; ++it )
   {
      norm = std::sqrt( dot( tp, tp ) );
      scale( xp, tp, 1.0 / norm );
      invDiagA( xp, tp );
      r = dot( xp, tp );
   }
   HYB_CUDA( cudaDeviceSynchronize() );
   *radius = r;
   HYB_API_END
}

static void checkGmg( Gmg* g, Function* x, Function* b, int level )
{
   require( g && x && b, "null argument" );
   require( x->st == g->st && b->st == g->st, "functions belong to another storage" );
   require( x->dtype == HYB_F64 && b->dtype == HYB_F64, "GMG functions are FP64 (the FP32 hierarchy is internal)" );
   require( level > g->minL - 1 && level <= g->maxL, "level outside the GMG level range" );
   require( x->minL <= g->minL && b->minL <= g->minL && x->maxL >= level && b->maxL >= level,
            "x and b must span the GMG levels" );
}

int hyb_gmg_solve( hyb_gmg* gh, hyb_function* xh, hyb_function* bh, int level, void* stream )
{
   HYB_API_BEGIN
   Gmg*      g = gh;
   Function *x = FN( xh ), *b = FN( bh );
   checkGmg( g, x, b, level );
   runGraph( *g, *x, *b, level, 0, S( stream ) );
   HYB_API_END
}

int hyb_gmg_solve_fmg( hyb_gmg* gh, hyb_function* xh, hyb_function* bh, int level, int cyclesPerLevel, void* stream )
{
   HYB_API_BEGIN
   Gmg*      g = gh;
   Function *x = FN( xh ), *b = FN( bh );
   checkGmg( g, x, b, level );
   require( cyclesPerLevel >= 1 && cyclesPerLevel <= 8, "cycles per level must be in [1, 8]" );
   runGraph( *g, *x, *b, level, kFmg64 + cyclesPerLevel, S( stream ) );
   HYB_API_END
}

int hyb_gmg_solve_to_tolerance( hyb_gmg* gh, hyb_function* xh, hyb_function* bh, int level, double relTol, int maxCycles,
                                int precision, double* history, int* cycles, void* stream )
{
   HYB_API_BEGIN
   Gmg*      g = gh;
   Function *x = FN( xh ), *b = FN( bh );
   checkGmg( g, x, b, level );
   require( precision == 64 || precision == 32, "precision must be 64 or 32" );
   require( maxCycles >= 0, "max_cycles must be non-negative" );
   cudaStream_t s = S( stream );
   Storage&     st = *g->st;
   if ( precision == 32 )
      ensureMixed( *g );
   // ||b|| and the initial residual
   launchDot< double >( st, level, b->ptr< double >( level ), b->ptr< double >( level ), kGmgFlag, g->partial.p,
                        g->scalars.p + 1, s );
   runGraph( *g, *x, *b, level, precision == 64 ? kNorm64 : kNormMixed, s );
   HYB_CUDA( cudaMemcpyAsync( g->hostScalar, g->scalars.p, 2 * sizeof( double ), cudaMemcpyDeviceToHost, s ) );
   HYB_CUDA( cudaStreamSynchronize( s ) );
   const double nb  = std::sqrt( g->hostScalar[1] ) > 0 ? std::sqrt( g->hostScalar[1] ) : 1.0;
   double       rel = std::sqrt( g->hostScalar[0] ) / nb;
   if ( history )
      history[0] = rel;
   int cyc = 0;
   while ( cyc < maxCycles && rel > relTol )
   {
      runGraph( *g, *x, *b, level, precision == 64 ? kCycle64Norm : kMixedStep, s );
      HYB_CUDA( cudaMemcpyAsync( g->hostScalar, g->scalars.p, sizeof( double ), cudaMemcpyDeviceToHost, s ) );
      HYB_CUDA( cudaStreamSynchronize( s ) );
      rel = std::sqrt( g->hostScalar[0] ) / nb;
      ++cyc;
      if ( history )
         history[cyc] = rel;
      if ( !std::isfinite( rel ) )
         throw Error( HYB_ENOTCONVERGED, "residual is not finite: the iteration diverged" );
   }
   if ( cycles )
      *cycles = cyc;
   HYB_API_END
}

} // extern "C"

// ===========================================================================
// Dot product that allocates nothing
// ===========================================================================
// For callers that cannot allocate device memory while they run: a serving loop that
// admitted its solves against a fixed HBM budget, or a host framework that owns the
// device allocator and forbids allocations behind its back. The first pass writes one
// partial sum per thread block into a file-scope device array instead of a buffer the
// library allocates; the caller passes the inputs and a device pointer for the result.
namespace hyb {

// 131072 partial sums = 1 MiB. Every GPU that loads this library holds the array until
// the process exits. A call needs (closure size / 256, rounded up) x (#macro-cells)
// slots; larger problems are rejected.
constexpr int kNoAllocSlots = 131072;
static __device__ __align__( 256 ) double g_noAllocPartial[kNoAllocSlots];

// In host code the array's name is only a host-side stand-in, not a device address: the
// address is looked up once per device, with that device current, and cached for the
// rest of the process. A cudaDeviceReset (or anything else that destroys the device's
// primary context) invalidates the cached address; do not call the entry point after one.
double* noAllocScratch()
{
   static std::mutex mu;
   static double*    addr[256] = {};
   int               dev       = 0;
   HYB_CUDA( cudaGetDevice( &dev ) );
   require( dev >= 0 && dev < 256, "device ordinal out of range" );
   std::lock_guard< std::mutex > lock( mu );
   if ( !addr[dev] )
   {
      void* p = nullptr;
      HYB_CUDA( cudaGetSymbolAddress( &p, g_noAllocPartial ) );
      addr[dev] = static_cast< double* >( p );
   }
   return addr[dev];
}

} // namespace hyb

extern "C" {

int hyb_function_dot_noalloc( hyb_function* ah, hyb_function* bh, int level, int flag, double* out_device, void* stream )
{
   HYB_API_BEGIN
   Function *a = FN( ah ), *b = FN( bh );
   require( out_device, "null result pointer" );
   sameStorage( a, b );
   {
      // the scratch array used is the current device's: the functions and the result must
      // live there too (a host pointer would only fail later, asynchronously)
      int dev = 0;
      HYB_CUDA( cudaGetDevice( &dev ) );
      require( dev == a->st->device, "the functions live on device " + std::to_string( a->st->device ) +
                                         ", the current device is " + std::to_string( dev ) );
      cudaPointerAttributes pa{};
      HYB_CUDA( cudaPointerGetAttributes( &pa, out_device ) );
      require( ( pa.type == cudaMemoryTypeDevice || pa.type == cudaMemoryTypeManaged ) && pa.device == dev,
               "out_device must be device (or managed) memory of the current device" );
   }
   require( a->dtype == b->dtype, "dtypes differ" );
   checkLevel( a, level );
   checkLevel( b, level );
   const Storage& st    = *a->st;
   const auto&    L     = st.L( level );
   const long     slots = long( L.slabBlocks ) * st.td.nC;
   require( slots <= kNoAllocSlots, "problem too large for the no-allocation dot product: needs " +
                                        std::to_string( slots ) + " scratch slots, the maximum is " +
                                        std::to_string( kNoAllocSlots ) );
   double* scratch = noAllocScratch();
   // every slot the reduction reads is rewritten by the first pass, so nothing is cleared
   if ( a->dtype == HYB_F64 )
      k_dot_partial< double ><<< dim3( L.slabBlocks, st.td.nC ), 256, 0, S( stream ) >>>(
          st.td, L.dev, a->ptr< double >( level ), b->ptr< double >( level ), flag, scratch, nullptr );
   else
      k_dot_partial< float ><<< dim3( L.slabBlocks, st.td.nC ), 256, 0, S( stream ) >>>(
          st.td, L.dev, a->ptr< float >( level ), b->ptr< float >( level ), flag, scratch, nullptr );
   HYB_CHECK_LAUNCH();
   k_reduce_final<<< 1, 1024, 0, S( stream ) >>>( scratch, int( slots ), out_device );
   HYB_CHECK_LAUNCH();
   HYB_API_END
}

} // extern "C"

// ===========================================================================
// Serving loop
// ===========================================================================
#include "hyb_server.inl"
