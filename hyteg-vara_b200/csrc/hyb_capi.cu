// Host engine and C ABI of the B200 P1 multigrid path (declarations and the
// reference interface each entry point replaces: include/hyteg_b200.h).
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

// ---------------------------------------------------------------------------
// Storage
// ---------------------------------------------------------------------------
// Row tables of a small level (SlabRow, any operator of the storage): the surface lanes of each SOR
// colour, the interior points of each interior colour (cell-major), and all DoFs (the
// surface lanes of the full lists, then every interior point) for residuals and CG.
struct RowTables
{
   DevBuf< SlabRow >   iface, interior, all;
   std::vector< long > ifaceOff; // per surface colour: first row
   long                allN = 0, allB1 = 0, allB2 = 0, allB3 = 0;
   bool                full = true; // false: only the surface colours' rows (large levels)
};

struct LevelHost
{
   LevelDev           dev{};
   std::unique_ptr< RowTables > rows; // built on first use (ensureRows)
   bool                         rowsTried = false;
   DevBuf< int32_t >  seg, xyz, blk, blkXYZ, pts, ptsC, quads, rowYZ;
   DevBuf< int4 >     pro; // prolongation table (LevelDev::pro)
   DevBuf< int32_t >  colourList;        // surface-DoF indices grouped by SOR colour
   std::vector< int > colourOff;         // per colour: offset, #vertex, #edge, #face DoFs
   int                cellBlocks   = 0;  // grid of the cell-interior row-segment loops
   int                ptsBlocks    = 0;  // grid of the loops over all interior points
   int                quadBlocks   = 0;  // grid of the loops over interior quads
   int                colourBlocks = 0;  // grid of the loops over one interior colour
   int                bdryBlocks   = 0;  // grid of the surface-DoF loops
   int                slabBlocks   = 0;  // blocks of 256 over one closure
};

struct Storage
{
   Topology                              topo;
   int                                   maxLevel = 0;
   int                                   numSMs   = 148;
   DevBuf< ClassDev >                    cls;
   DevBuf< int32_t >                     fEmb, eEmbOff, eEmb, vEmbOff, vEmb;
   DevBuf< uint8_t >                     fBc, eBc, vBc;
   DevBuf< int8_t >                      labels;
   DevBuf< double >                      cellCoords; // [nC][4][3] macro-cell vertex coordinates
   DevBuf< int32_t >                     cellOrder;  // [nC] local vertex indices sorted by global id, 2 bits each
   TopoDev                               td{};
   std::vector< std::unique_ptr< LevelHost > > lv;
   DevBuf< LevelDev >                    lvTable; // LevelDev of every level, for the program kernel
   DevBuf< double >                      partial; // dot-product partials
   DevBuf< double >                      scalars; // device scalars (dot results)
   double*                               hostScalar = nullptr;
   DevBuf< char >                        staging; // canonical-order transfer buffer (grow-only)

   char* stage( size_t bytes )
   {
      if ( staging.n < bytes )
      {
         HYB_CUDA( cudaDeviceSynchronize() ); // the old buffer may still be in use by queued copies
         staging.alloc( bytes );
      }
      return staging.p;
   }

   ~Storage()
   {
      if ( hostScalar )
         cudaFreeHost( hostScalar );
   }

   const LevelHost& L( int l ) const { return *lv.at( l ); }
};

inline int stridePad( int s ) { return ( s + 31 ) / 32 * 32; }

void buildStorage( Storage& s, const std::vector< std::array< double, 3 > >& V, const std::vector< std::array< int, 4 > >& T,
                   int maxLevel )
{
   require( maxLevel >= 0 && maxLevel <= 9, "max_level must be in [0, 9]" );
   require( !T.empty(), "mesh has no tetrahedra" );
   s.maxLevel = maxLevel;
   {
      int dev = 0;
      HYB_CUDA( cudaGetDevice( &dev ) );
      HYB_CUDA( cudaDeviceGetAttribute( &s.numSMs, cudaDevAttrMultiProcessorCount, dev ) );
   }
   s.topo.build( V, T );
   s.topo.computeColouring();
   auto& tp = s.topo;
   const int nC = int( tp.T.size() ), nF = int( tp.F.size() ), nE = int( tp.E.size() ), nV = int( tp.V.size() );
   require( nC < ( 1 << 24 ), "too many macro-cells for the packed embedding format" );
   // class table
   std::vector< ClassDev > cls( size_t( nC ) * 16 );
   for ( int c = 0; c < nC; ++c )
      for ( int m = 0; m < 16; ++m )
      {
         const auto& ci = tp.cls[c][m];
         ClassDev    d{};
         d.id    = ci.id;
         d.kind  = uint8_t( ci.kind < 0 ? 255 : ci.kind );
         d.bc    = ci.bc;
         d.owned = ci.owned ? 1 : 0;
         d.invN  = ci.ncells > 0 ? 1.0 / double( ci.ncells ) : 0.0;
         // local vertex indices of the primitive's sorted vertices in this cell
         std::vector< std::pair< int, int > > vs;
         for ( int k = 0; k < 4; ++k )
            if ( !( m & ( 1 << k ) ) )
               vs.push_back( { tp.T[c][k], k } );
         std::sort( vs.begin(), vs.end() );
         d.k0 = vs.size() > 0 ? uint8_t( vs[0].second ) : 0;
         d.k1 = vs.size() > 1 ? uint8_t( vs[1].second ) : 0;
         d.k2 = vs.size() > 2 ? uint8_t( vs[2].second ) : 0;
         cls[size_t( c ) * 16 + m] = d;
      }
   s.cls.upload( cls );
   std::vector< int32_t > fEmb( size_t( nF ) * 2, -1 );
   for ( int f = 0; f < nF; ++f )
      for ( size_t e = 0; e < tp.fEmb[f].size(); ++e )
         fEmb[2 * f + e] = packEmbedding( tp.fEmb[f][e] );
   auto csr = []( const std::vector< std::vector< Embedding > >& emb, std::vector< int32_t >& off, std::vector< int32_t >& val ) {
      off.assign( emb.size() + 1, 0 );
      val.clear();
      for ( size_t i = 0; i < emb.size(); ++i )
      {
         for ( auto& e : emb[i] )
            val.push_back( packEmbedding( e ) );
         off[i + 1] = int32_t( val.size() );
      }
   };
   std::vector< int32_t > eOff, eVal, vOff, vVal;
   csr( tp.eEmb, eOff, eVal );
   csr( tp.vEmb, vOff, vVal );
   s.fEmb.upload( fEmb );
   s.eEmbOff.upload( eOff );
   s.eEmb.upload( eVal );
   s.vEmbOff.upload( vOff );
   s.vEmb.upload( vVal );
   s.fBc.upload( tp.fBc );
   s.eBc.upload( tp.eBc );
   s.vBc.upload( tp.vBc );
   std::vector< int8_t > lab( size_t( nC ) * 4 );
   for ( int c = 0; c < nC; ++c )
      for ( int k = 0; k < 4; ++k )
         lab[4 * c + k] = int8_t( tp.labels[tp.T[c][k]] );
   s.labels.upload( lab );
   std::vector< double > cc( size_t( nC ) * 12 );
   for ( int c = 0; c < nC; ++c )
      for ( int k = 0; k < 4; ++k )
         for ( int d = 0; d < 3; ++d )
            cc[size_t( c ) * 12 + 3 * k + d] = tp.V[tp.T[c][k]][d];
   s.cellCoords.upload( cc );
   std::vector< int32_t > order( nC );
   for ( int c = 0; c < nC; ++c )
   {
      int k[4] = { 0, 1, 2, 3 };
      std::sort( k, k + 4, [&]( int a, int b ) { return tp.T[c][a] < tp.T[c][b]; } );
      order[c] = k[0] | k[1] << 2 | k[2] << 4 | k[3] << 6;
   }
   s.cellOrder.upload( order );
   s.td = TopoDev{ nC, nF, nE, nV, s.cls.p, s.fEmb.p, s.eEmbOff.p, s.eEmb.p, s.vEmbOff.p, s.vEmb.p,
                   s.fBc.p, s.eBc.p, s.vBc.p, s.labels.p, tp.colours };
   // per-level tables
   size_t maxPartial = 1;
   for ( int l = 0; l <= maxLevel; ++l )
   {
      auto      lh = std::make_unique< LevelHost >();
      LevelDev& d  = lh->dev;
      d.L          = l;
      d.N          = 1 << l;
      d.W          = d.N + 1;
      d.S          = tetSize( d.W );
      d.stride     = stridePad( d.S );
      d.nIntFace   = d.N >= 3 ? ( d.N - 1 ) * ( d.N - 2 ) / 2 : 0;
      d.nIntCell   = d.N >= 4 ? tetSize( d.N - 3 ) : 0;
      d.nBdry      = nV + nE * ( d.N - 1 ) + nF * d.nIntFace;
      std::vector< int32_t >                seg, xyz( d.S ), blk, blkXYZ, pts, quads, rowYZ;
      std::vector< std::vector< int32_t > > ptsC( kInteriorColours );
      for ( int z = 1; z <= d.N; ++z )
         for ( int y = 1; y <= d.N - z; ++y )
         {
            const int len = d.N - 1 - y - z; // interior x in [1, len]
            if ( len < 1 )
               continue;
            for ( int x0 = 1; x0 <= len; x0 += 32 )
               seg.push_back( z | ( y << 10 ) | ( x0 << 20 ) );
            const int row = int( rowYZ.size() );
            require( row < ( 1 << 23 ), "too many rows for the quad-table encoding" );
            rowYZ.push_back( y | ( z << 16 ) );
            for ( int g = 0; 4 * g <= len; ++g )
               quads.push_back( g | ( row << 8 ) );
         }
      // interior point tables: points in storage order, cut into blocks of consecutive
      // positions whose neighbour offsets agree (checked, not assumed from the layout)
      {
         std::vector< std::array< int, 2 > > order; // (position, packed x | y << 10 | z << 20)
         for ( int z = 1; z <= d.N; ++z )
            for ( int y = 1; y + z <= d.N - 2; ++y )
               for ( int x = 1; x + y + z <= d.N - 1; ++x )
                  order.push_back( { sidx( d.W, x, y, z ), x | ( y << 10 ) | ( z << 20 ) } );
         std::sort( order.begin(), order.end() );
         int prevPos = -2, start = 0, prevXYZ = -1;
         int prevD[15] = {};
         for ( const auto& o : order )
         {
            const int x = o[1] & 1023, y = ( o[1] >> 10 ) & 1023, z = o[1] >> 20;
            int       D[15];
            for ( int q = 0; q < 15; ++q )
               D[q] = sidx( d.W, x + offX( q ), y + offY( q ), z + offZ( q ) ) - o[0];
            const bool same = o[0] == prevPos + 1 && o[0] - start < 256 && std::equal( D, D + 15, prevD ) &&
                              o[1] == prevXYZ + 4;
            if ( !same )
            {
               start = o[0];
               require( blk.size() / 16 < ( 1u << 23 ), "too many blocks for the point-table encoding" );
               for ( int q = 0; q < 16; ++q )
                  blk.push_back( q < 15 ? start + D[q] : 0 );
               blkXYZ.push_back( o[1] );
            }
            const int32_t e = ( o[0] - start ) | ( int32_t( blk.size() / 16 - 1 ) << 8 );
            pts.push_back( e );
            ptsC[( x + 2 * y + 3 * z ) & 3].push_back( e );
            prevPos = o[0];
            prevXYZ = o[1];
            std::copy( D, D + 15, prevD );
         }
      }
      std::vector< int32_t > ptsFlat;
      for ( int c = 0; c < kInteriorColours; ++c )
      {
         d.ptsOff[c] = int( ptsFlat.size() );
         ptsFlat.insert( ptsFlat.end(), ptsC[c].begin(), ptsC[c].end() );
      }
      d.ptsOff[kInteriorColours] = int( ptsFlat.size() );
      d.nPts                     = int( pts.size() );
      d.nQuads = int( quads.size() );
      lh->quads.upload( quads );
      lh->rowYZ.upload( rowYZ );
      d.quads = lh->quads.p;
      d.rowYZ = lh->rowYZ.p;
      lh->blk.upload( blk );
      lh->blkXYZ.upload( blkXYZ );
      d.blkXYZ = lh->blkXYZ.p;
      lh->pts.upload( pts );
      lh->ptsC.upload( ptsFlat );
      d.blk  = lh->blk.p;
      d.pts  = lh->pts.p;
      d.ptsC = lh->ptsC.p;
      // prolongation table: the two coarse endpoints of every block's points (pattern of
      // interpolateFine), checked point by point against the closed-form indices
      if ( l >= 1 && !blkXYZ.empty() )
      {
         const int           Wc = d.W / 2 + 1; // N / 2 + 1
         std::vector< int4 > pro( 2 * blkXYZ.size() );
         auto                ends = [&]( int x, int y, int z, int* A, int* B, bool& single ) {
            const int px = x & 1, py = y & 1, pz = z & 1, pat = px | ( py << 1 ) | ( pz << 2 );
            int       ox = 0, oy = 0, oz = 0;
            switch ( pat )
            {
            case 0: break;
            case 1: ox = 1; break;
            case 2: oy = 1; break;
            case 4: oz = 1; break;
            case 3: ox = -1, oy = 1; break;
            case 5: ox = -1, oz = 1; break;
            case 6: oy = -1, oz = 1; break;
            default: ox = -1, oy = 1, oz = -1; break;
            }
            single = pat == 0;
            A[0] = ( x - ox ) >> 1, A[1] = ( y - oy ) >> 1, A[2] = ( z - oz ) >> 1;
            B[0] = ( x + ox ) >> 1, B[1] = ( y + oy ) >> 1, B[2] = ( z + oz ) >> 1;
         };
         // slab position of the first point of residue r in coarse row (Y, Z)
         auto base = [&]( int Y, int Z, int r ) { return rowStart( Wc, Y, Z ) + resOff( r, Wc - Y - Z ); };
         for ( size_t b = 0; b < blkXYZ.size(); ++b )
         {
            const int x0 = blkXYZ[b] & 1023, y = ( blkXYZ[b] >> 10 ) & 1023, z = blkXYZ[b] >> 20;
            int       A[3], B[3];
            bool      single;
            ends( x0, y, z, A, B, single );
            pro[2 * b]     = make_int4( base( A[1], A[2], A[0] & 3 ), base( A[1], A[2], ( A[0] + 2 ) & 3 ), A[0],
                                        base( B[1], B[2], B[0] & 3 ) );
            pro[2 * b + 1] = make_int4( base( B[1], B[2], ( B[0] + 2 ) & 3 ), B[0], single ? 1 : 0, 0 );
         }
         for ( const int32_t e : pts )
         {
            const int  g = e & 255, b = e >> 8;
            const int  x = ( blkXYZ[b] & 1023 ) + 4 * g, y = ( blkXYZ[b] >> 10 ) & 1023, z = blkXYZ[b] >> 20;
            int        A[3], B[3];
            bool       single;
            ends( x, y, z, A, B, single );
            const int4 P0 = pro[2 * b], P1 = pro[2 * b + 1];
            const int  cA = ( ( g & 1 ) ? P0.y : P0.x ) + ( ( P0.z + 2 * g ) >> 2 );
            const int  cB = ( ( g & 1 ) ? P1.x : P0.w ) + ( ( P1.y + 2 * g ) >> 2 );
            require( cA == sidx( Wc, A[0], A[1], A[2] ) && ( single || cB == sidx( Wc, B[0], B[1], B[2] ) ) &&
                         ( P1.z != 0 ) == single,
                     "prolongation table disagrees with the closed-form indices" );
         }
         lh->pro.upload( pro );
         d.pro = lh->pro.p;
      }
      for ( int z = 0; z <= d.N; ++z )
         for ( int y = 0; y <= d.N - z; ++y )
            for ( int x = 0; x <= d.N - y - z; ++x )
               xyz[sidx( d.W, x, y, z )] = x | ( y << 10 ) | ( z << 20 );
      lh->seg.upload( seg );
      lh->xyz.upload( xyz );
      d.nSeg = int( seg.size() );
      d.seg  = lh->seg.p;
      d.xyz  = lh->xyz.p;
      // grids: the loops are grid-stride, so a few resident blocks per SM suffice
      auto grid = [&]( long work, int perBlock, int perSM ) {
         return int( std::max< long >( 0, std::min< long >( ( work + perBlock - 1 ) / perBlock, long( s.numSMs ) * perSM ) ) );
      };
      lh->cellBlocks = grid( long( d.nSeg ) * nC, kCellWarps, 16 );
      lh->ptsBlocks  = grid( long( ( d.nPts + 63 ) / 64 ) * nC, kCellWarps, 16 );
      lh->quadBlocks = grid( long( ( d.nQuads + 31 ) / 32 ) * nC, kCellWarps, 16 );
      int maxColour  = 0;
      for ( int c = 0; c < kInteriorColours; ++c )
         maxColour = std::max( maxColour, d.ptsOff[c + 1] - d.ptsOff[c] );
      lh->colourBlocks = grid( long( ( maxColour + 31 ) / 32 ) * nC, kCellWarps, 16 );
      lh->bdryBlocks    = grid( bdryLaneCount( nV, nE * ( d.N - 1 ), nF * d.nIntFace ), kBdryThreads, 8 );
      lh->slabBlocks    = ( d.S + 255 ) / 256;
      maxPartial        = std::max( maxPartial, size_t( lh->slabBlocks ) * nC );
      // surface DoFs grouped by SOR colour: colour = sum of label(v) * micro-weight(v) over
      // the primitive's vertices (the same value in every adjacent cell)
      {
         const int                        m = tp.colours, N = d.N;
         std::vector< std::vector< int > > byColour( m );
         auto                             col = [&]( long s ) { return int( ( ( s % m ) + m ) % m ); };
         int                              t   = 0;
         for ( int v = 0; v < nV; ++v, ++t )
            byColour[col( long( tp.labels[v] ) * N )].push_back( t );
         for ( int e = 0; e < nE; ++e )
            for ( int i = 1; i < N; ++i, ++t )
               byColour[col( long( tp.labels[tp.E[e][0]] ) * ( N - i ) + long( tp.labels[tp.E[e][1]] ) * i )].push_back( t );
         for ( int f = 0; f < nF; ++f )
            for ( int j = 1; j <= N - 2; ++j )
               for ( int i = 1; i <= N - 1 - j; ++i, ++t )
                  byColour[col( long( tp.labels[tp.F[f][0]] ) * ( N - i - j ) + long( tp.labels[tp.F[f][1]] ) * i +
                                long( tp.labels[tp.F[f][2]] ) * j )]
                      .push_back( t );
         require( t == d.nBdry, "surface DoF enumeration mismatch" );
         // per colour: [vertex DoFs | edge DoFs | face DoFs] (ascending t keeps the kinds apart)
         std::vector< int32_t > flat;
         lh->colourOff.clear();
         const int tE = nV, tF = nV + nE * ( N - 1 );
         for ( auto& v : byColour )
         {
            int nv = 0, ne = 0, nf = 0;
            for ( int tt : v )
               ( tt < tE ? nv : tt < tF ? ne : nf )++;
            lh->colourOff.push_back( int( flat.size() ) );
            lh->colourOff.push_back( nv );
            lh->colourOff.push_back( ne );
            lh->colourOff.push_back( nf );
            flat.insert( flat.end(), v.begin(), v.end() );
         }
         lh->colourList.upload( flat );
      }
      s.lv.push_back( std::move( lh ) );
   }
   {
      std::vector< LevelDev > t;
      for ( auto& lh : s.lv )
         t.push_back( lh->dev );
      s.lvTable.upload( t );
   }
   s.partial.alloc( maxPartial );
   s.scalars.alloc( 64 );
   HYB_CUDA( cudaMallocHost( &s.hostScalar, 64 * sizeof( double ) ) );
}

// ---------------------------------------------------------------------------
// Functions
// ---------------------------------------------------------------------------
struct Function
{
   Storage*            st;
   int                 minL, maxL, dtype;
   std::vector< void* > data;  // per level, index l - minL
   std::vector< size_t > bytes; // allocation size per level

   ~Function()
   {
      for ( size_t i = 0; i < data.size(); ++i )
         if ( data[i] )
         {
            cudaFree( data[i] );
            g_deviceBytes.fetch_sub( (long long) bytes[i] );
         }
   }
   size_t elem() const { return dtype == HYB_F64 ? 8 : 4; }
   void*  at( int l ) const
   {
      require( l >= minL && l <= maxL, "level " + std::to_string( l ) + " outside the function's level range" );
      return data[l - minL];
   }
   template < typename T >
   T* ptr( int l ) const
   {
      return static_cast< T* >( at( l ) );
   }
   size_t levelBytes( int l ) const { return size_t( st->td.nC ) * st->L( l ).dev.stride * elem(); }
};

Function* makeFunction( Storage* s, int minL, int maxL, int dtype )
{
   require( minL >= 0 && minL <= maxL && maxL <= s->maxLevel, "invalid level range" );
   require( dtype == HYB_F64 || dtype == HYB_F32, "dtype must be HYB_F64 or HYB_F32" );
   auto f = std::make_unique< Function >();
   f->st = s;
   f->minL = minL;
   f->maxL = maxL;
   f->dtype = dtype;
   for ( int l = minL; l <= maxL; ++l )
   {
      void* p = nullptr;
      HYB_CUDA( cudaMalloc( &p, f->levelBytes( l ) ) );
      f->data.push_back( p );
      f->bytes.push_back( f->levelBytes( l ) );
      g_deviceBytes.fetch_add( (long long) f->levelBytes( l ) );
      HYB_CUDA( cudaMemset( p, 0, f->levelBytes( l ) ) );
   }
   return f.release();
}

// ---------------------------------------------------------------------------
// Operators
// ---------------------------------------------------------------------------
namespace {
const int kMicro[6][4][3] = {
    { { 0, 0, 0 }, { 1, 0, 0 }, { 0, 1, 0 }, { 0, 0, 1 } }, { { 1, 0, 0 }, { 1, 1, 0 }, { 0, 1, 0 }, { 1, 0, 1 } },
    { { 1, 0, 0 }, { 0, 1, 0 }, { 1, 0, 1 }, { 0, 0, 1 } }, { { 1, 1, 0 }, { 1, 1, 1 }, { 0, 1, 1 }, { 1, 0, 1 } },
    { { 1, 0, 1 }, { 0, 1, 1 }, { 0, 0, 1 }, { 0, 1, 0 } }, { { 0, 1, 0 }, { 1, 1, 0 }, { 1, 0, 1 }, { 0, 1, 1 } } };

// P1 stiffness  K_ij = |T| grad(phi_i).grad(phi_j)  of a tetrahedron
void stiffness( const double X[4][3], double K[4][4] )
{
   double J[3][3];
   for ( int r = 0; r < 3; ++r )
      for ( int c = 0; c < 3; ++c )
         J[r][c] = X[c + 1][r] - X[0][r];
   const double det = J[0][0] * ( J[1][1] * J[2][2] - J[1][2] * J[2][1] ) - J[0][1] * ( J[1][0] * J[2][2] - J[1][2] * J[2][0] ) +
                      J[0][2] * ( J[1][0] * J[2][1] - J[1][1] * J[2][0] );
   require( std::fabs( det ) > 0, "degenerate macro-cell" );
   // rows of J^-1 are the gradients of the barycentric coordinates 1..3
   double g[4][3];
   g[1][0] = ( J[1][1] * J[2][2] - J[1][2] * J[2][1] ) / det;
   g[1][1] = ( J[0][2] * J[2][1] - J[0][1] * J[2][2] ) / det;
   g[1][2] = ( J[0][1] * J[1][2] - J[0][2] * J[1][1] ) / det;
   g[2][0] = ( J[1][2] * J[2][0] - J[1][0] * J[2][2] ) / det;
   g[2][1] = ( J[0][0] * J[2][2] - J[0][2] * J[2][0] ) / det;
   g[2][2] = ( J[0][2] * J[1][0] - J[0][0] * J[1][2] ) / det;
   g[3][0] = ( J[1][0] * J[2][1] - J[1][1] * J[2][0] ) / det;
   g[3][1] = ( J[0][1] * J[2][0] - J[0][0] * J[2][1] ) / det;
   g[3][2] = ( J[0][0] * J[1][1] - J[0][1] * J[1][0] ) / det;
   for ( int d = 0; d < 3; ++d )
      g[0][d] = -g[1][d] - g[2][d] - g[3][d];
   const double vol = std::fabs( det ) / 6.0;
   for ( int i = 0; i < 4; ++i )
      for ( int j = 0; j < 4; ++j )
         K[i][j] = vol * ( g[i][0] * g[j][0] + g[i][1] * g[j][1] + g[i][2] * g[j][2] );
}

// element matrices of the six micro-tet shapes of a macro-cell at level L
void microMatrices( const Topology& tp, int c, int N, double K[6][4][4] )
{
   const auto& t = tp.T[c];
   for ( int ty = 0; ty < 6; ++ty )
   {
      double X[4][3];
      for ( int j = 0; j < 4; ++j )
         for ( int d = 0; d < 3; ++d )
         {
            const double v0 = tp.V[t[0]][d];
            X[j][d] = v0 + ( tp.V[t[1]][d] - v0 ) / N * kMicro[ty][j][0] + ( tp.V[t[2]][d] - v0 ) / N * kMicro[ty][j][1] +
                      ( tp.V[t[3]][d] - v0 ) / N * kMicro[ty][j][2];
         }
      stiffness( X, K[ty] );
   }
}

bool tetAllowed( int mask, const IncidentTet& it )
{
   for ( int j = 0; j < 4; ++j )
   {
      const int q = it.q[j];
      const int x = offX( q ), y = offY( q ), z = offZ( q );
      if ( ( mask & 1 ) && -( x + y + z ) < 0 )
         return false;
      if ( ( mask & 2 ) && x < 0 )
         return false;
      if ( ( mask & 4 ) && y < 0 )
         return false;
      if ( ( mask & 8 ) && z < 0 )
         return false;
   }
   return true;
}
} // namespace

struct Operator
{
   Storage* st;
   int      minL, maxL;
   bool     variable = false;
   // per level (index l - minL)
   std::vector< std::unique_ptr< DevBuf< double > > > st64, K64;
   std::vector< std::unique_ptr< DevBuf< float > > >  st32, K32;
   std::vector< std::vector< double > >               stHost; // [nC*16*15]
   std::unique_ptr< Function >                        kap64, kap32;

   template < typename T >
   OpDev< T > dev( int l ) const
   {
      require( l >= minL && l <= maxL, "level outside the operator's level range" );
      OpDev< T > o{};
      const int  i = l - minL;
      if constexpr ( std::is_same< T, double >::value )
      {
         o.st = variable ? nullptr : st64[i]->p;
         o.K  = variable ? K64[i]->p : nullptr;
         o.kap = variable ? kap64->ptr< double >( l ) : nullptr;
      }
      else
      {
         o.st = variable ? nullptr : st32[i]->p;
         o.K  = variable ? K32[i]->p : nullptr;
         o.kap = variable ? kap32->ptr< float >( l ) : nullptr;
      }
      o.stride = st->L( l ).dev.stride;
      return o;
   }
};

Operator* makeLaplace( Storage* s, int minL, int maxL )
{
   require( minL >= 0 && minL <= maxL && maxL <= s->maxLevel, "invalid level range" );
   auto op = std::make_unique< Operator >();
   op->st = s;
   op->minL = minL;
   op->maxL = maxL;
   const int nC = s->td.nC;
   for ( int l = minL; l <= maxL; ++l )
   {
      std::vector< double > st( size_t( nC ) * 16 * 15, 0.0 );
      for ( int c = 0; c < nC; ++c )
      {
         double K[6][4][4];
         microMatrices( s->topo, c, 1 << l, K );
         // partial stencil of each class = sum over the incident micro-tets inside the closure
         // (P1Elements.hpp:215-302, 464-526)
         for ( int mask = 0; mask < 16; ++mask )
            for ( int i = 0; i < 24; ++i )
            {
               const IncidentTet it = incidentTet( i );
               if ( !tetAllowed( mask, it ) )
                  continue;
               for ( int j = 0; j < 4; ++j )
                  st[( size_t( c ) * 16 + mask ) * 15 + it.q[j]] += K[it.t][it.k][j];
            }
      }
      auto b64 = std::make_unique< DevBuf< double > >();
      b64->upload( st );
      std::vector< float > f( st.begin(), st.end() );
      auto b32 = std::make_unique< DevBuf< float > >();
      b32->upload( f );
      op->st64.push_back( std::move( b64 ) );
      op->st32.push_back( std::move( b32 ) );
      op->stHost.push_back( std::move( st ) );
   }
   return op.release();
}

template < typename T >
void launchFromDofs( const Storage& s, int l, T* slab, const T* dofs, cudaStream_t stream );
template < typename TD, typename TS >
void launchConvert( const Storage& s, int l, TD* dst, const TS* src, cudaStream_t stream );

// The nodal coefficient of level l is written into the FP64 slab by fillK( l, slab ).
template < typename FillK >
Operator* makeDivKGradWith( Storage* s, int minL, int maxL, FillK&& fillK )
{
   require( minL >= 0 && minL <= maxL && maxL <= s->maxLevel, "invalid level range" );
   auto op = std::make_unique< Operator >();
   op->st = s;
   op->minL = minL;
   op->maxL = maxL;
   op->variable = true;
   op->kap64.reset( makeFunction( s, minL, maxL, HYB_F64 ) );
   op->kap32.reset( makeFunction( s, minL, maxL, HYB_F32 ) );
   const int nC = s->td.nC;
   for ( int l = minL; l <= maxL; ++l )
   {
      // micro-tet matrices with the 1/4 of the vertex average folded in: the reference form's
      // 5-point degree-3 rule integrates the P1 interpolant of k exactly, giving
      // A_e = mean_e(k) * K_e (p1_div_k_grad_affine_q3.cpp:179+)
      std::vector< double > Km( size_t( nC ) * 96 );
      for ( int c = 0; c < nC; ++c )
      {
         double K[6][4][4];
         microMatrices( s->topo, c, 1 << l, K );
         for ( int t = 0; t < 6; ++t )
            for ( int i = 0; i < 4; ++i )
               for ( int j = 0; j < 4; ++j )
                  Km[size_t( c ) * 96 + t * 16 + i * 4 + j] = 0.25 * K[t][i][j];
      }
      auto b64 = std::make_unique< DevBuf< double > >();
      b64->upload( Km );
      std::vector< float > f( Km.begin(), Km.end() );
      auto b32 = std::make_unique< DevBuf< float > >();
      b32->upload( f );
      op->K64.push_back( std::move( b64 ) );
      op->K32.push_back( std::move( b32 ) );
      fillK( l, op->kap64->ptr< double >( l ) );
      const int n = s->td.nC * s->L( l ).dev.stride;
      pdlLaunch( k_convert< float, double >, dim3( ( n + 255 ) / 256 ), dim3( 256 ), 0, 0, s->L( l ).dev, op->kap32->ptr< float >( l ),
                                                                 op->kap64->ptr< double >( l ), s->td.nC );
      HYB_CHECK_LAUNCH();
      HYB_CUDA( cudaDeviceSynchronize() );
   }
   return op.release();
}

Operator* makeDivKGrad( Storage* s, int minL, int maxL, const std::vector< std::vector< double > >& nodalK )
{
   require( int( nodalK.size() ) == maxL - minL + 1, "one nodal coefficient vector per level is required" );
   return makeDivKGradWith( s, minL, maxL, [&]( int l, double* slab ) {
      const auto& kv = nodalK[l - minL];
      require( int64_t( kv.size() ) == s->topo.numDofs( l ), "nodal coefficient vector has the wrong length" );
      DevBuf< double > tmp;
      tmp.upload( kv );
      launchFromDofs< double >( *s, l, slab, tmp.p, 0 );
   } );
}

// k = exp( sigma sqrt(2/M) sum_m cos( w_m . x + phase_m ) ) (random Fourier features of a
// Gaussian random field) written into the operator's nodal coefficient on every level, FP64
// and its FP32 copy; dW (modes x 3) and dPhase are device arrays. Asynchronous on `stream`;
// the slabs keep their addresses, so graphs captured with the operator stay valid.
void fillRff( Operator& op, const double* dW, const double* dPhase, int modes, double sigma, double radial,
              cudaStream_t stream )
{
   const Storage& s = *op.st;
   for ( int l = op.minL; l <= op.maxL; ++l )
   {
      const auto& L = s.L( l );
      pdlLaunch( k_fill_rff_coefficient< double >, dim3( dim3( L.slabBlocks, s.td.nC ) ), dim3( 256 ), 0, stream, s.td, L.dev, s.cellCoords.p, s.cellOrder.p, op.kap64->ptr< double >( l ), dW, dPhase, modes, sigma, radial );
      HYB_CHECK_LAUNCH();
      launchConvert< float, double >( s, l, op.kap32->ptr< float >( l ), op.kap64->ptr< double >( l ), stream );
   }
}

Operator* makeDivKGradRff( Storage* s, int minL, int maxL, const double* w, const double* phase, int modes, double sigma,
                           double radial )
{
   require( modes > 0 && w && phase, "random-feature parameters missing" );
   DevBuf< double > dw, dp;
   dw.upload( std::vector< double >( w, w + 3 * modes ) );
   dp.upload( std::vector< double >( phase, phase + modes ) );
   std::unique_ptr< Operator > op( makeDivKGradWith( s, minL, maxL, []( int, double* ) {} ) );
   fillRff( *op, dw.p, dp.p, modes, sigma, radial, 0 );
   HYB_CUDA( cudaDeviceSynchronize() );
   return op.release();
}

// Coordinates of every micro-vertex of a level in the canonical DoF order
// (vertexdof::macrocell::coordinateFromIndex, VertexDoFMacroCell.hpp:68-75, and its
// face/edge analogues), evaluated on the host.
void dofCoords( const Topology& tp, int l, std::vector< double >& out )
{
   const int     N        = 1 << l;
   const int64_t offE     = int64_t( tp.V.size() ), offF = offE + int64_t( tp.E.size() ) * ( N - 1 );
   const int64_t nIntFace = N >= 3 ? ( N - 1 ) * ( N - 2 ) / 2 : 0;
   const int64_t offC     = offF + int64_t( tp.F.size() ) * nIntFace;
   const int64_t nIntCell = N >= 4 ? ( N - 3 ) * ( N - 2 ) * ( N - 1 ) / 6 : 0;
   out.assign( size_t( tp.numDofs( l ) ) * 3, 0.0 );
   auto put = [&]( int64_t d, const double* x ) {
      for ( int k = 0; k < 3; ++k )
         out[3 * d + k] = x[k];
   };
   double x[3];
   for ( size_t v = 0; v < tp.V.size(); ++v )
      put( int64_t( v ), tp.V[v].data() );
   for ( size_t e = 0; e < tp.E.size(); ++e )
      for ( int i = 1; i < N; ++i )
      {
         for ( int d = 0; d < 3; ++d )
            x[d] = tp.V[tp.E[e][0]][d] + ( tp.V[tp.E[e][1]][d] - tp.V[tp.E[e][0]][d] ) / N * i;
         put( offE + int64_t( e ) * ( N - 1 ) + ( i - 1 ), x );
      }
   for ( size_t f = 0; f < tp.F.size(); ++f )
      for ( int j = 1; j <= N - 2; ++j )
         for ( int i = 1; i <= N - 1 - j; ++i )
         {
            const auto& F = tp.F[f];
            for ( int d = 0; d < 3; ++d )
               x[d] = tp.V[F[0]][d] + ( tp.V[F[1]][d] - tp.V[F[0]][d] ) / N * i + ( tp.V[F[2]][d] - tp.V[F[0]][d] ) / N * j;
            put( offF + int64_t( f ) * nIntFace + ( j - 1 ) * ( N - 1 ) - ( j - 1 ) * j / 2 + ( i - 1 ), x );
         }
   for ( size_t c = 0; c < tp.T.size(); ++c )
      for ( int zz = 1; zz <= N; ++zz )
         for ( int yy = 1; yy <= N - zz; ++yy )
            for ( int xx = 1; xx <= N - 1 - yy - zz; ++xx )
            {
               const auto& t = tp.T[c];
               for ( int d = 0; d < 3; ++d )
               {
                  const double v0 = tp.V[t[0]][d];
                  x[d] = v0 + ( tp.V[t[1]][d] - v0 ) / N * xx + ( tp.V[t[2]][d] - v0 ) / N * yy + ( tp.V[t[3]][d] - v0 ) / N * zz;
               }
               put( offC + int64_t( c ) * nIntCell + cidx( N - 3, xx - 1, yy - 1, zz - 1 ), x );
            }
}

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------
inline int bdryBlocks( const LevelDev& d ) { return ( d.nBdry + kBdryThreads - 1 ) / kBdryThreads; }

template < typename T >
void launchFromDofs( const Storage& s, int l, T* slab, const T* dofs, cudaStream_t stream )
{
   const auto& L = s.L( l );
   pdlLaunch( k_from_dofs< T >, dim3( dim3( L.slabBlocks, s.td.nC ) ), dim3( 256 ), 0, stream, s.td, L.dev, slab, dofs );
   HYB_CHECK_LAUNCH();
}

template < typename T >
void launchToDofs( const Storage& s, int l, const T* slab, T* dofs, cudaStream_t stream )
{
   const auto& L = s.L( l );
   pdlLaunch( k_to_dofs< T >, dim3( dim3( L.slabBlocks, s.td.nC ) ), dim3( 256 ), 0, stream, s.td, L.dev, slab, dofs );
   HYB_CHECK_LAUNCH();
}

// Levels whose closure slabs hold at most this many points (all cells) get full row tables
// (HYB_ROW_TABLE_MAX_POINTS overrides it, 0: none); larger levels up to the second bound
// get the surface colours' rows only (HYB_ROW_IFACE_MAX_POINTS): their interior passes
// are bandwidth bound and keep the interior point tables.
constexpr long kRowTableMaxPoints = 400000;
constexpr long kRowIfaceMaxPoints = 4000000;

long envLong( const char* name, long dflt )
{
   const char* e = std::getenv( name );
   return e ? std::atol( e ) : dflt;
}
long rowTableMaxPoints()
{
   static const long v = envLong( "HYB_ROW_TABLE_MAX_POINTS", kRowTableMaxPoints );
   return v;
}
long rowIfaceMaxPoints()
{
   static const long v = envLong( "HYB_ROW_IFACE_MAX_POINTS", kRowIfaceMaxPoints );
   return v;
}

// The row tables of level l, built on first use (not inside a stream capture); nullptr if
// the level is too large, or if a DoF has more embeddings than its lane group (then the
// passes keep the lane-group path).
const RowTables* ensureRows( Storage& s, int l )
{
   LevelHost& L = *s.lv[size_t( l )];
   if ( L.rowsTried )
      return L.rows.get();
   L.rowsTried = true;
   const LevelDev& d      = L.dev;
   const long      points = long( s.td.nC ) * d.stride;
   if ( points > std::max( rowTableMaxPoints(), rowIfaceMaxPoints() ) || d.stride >= 65536 )
      return nullptr;
   auto R  = std::make_unique< RowTables >();
   R->full = points <= rowTableMaxPoints();
   DevBuf< int >    err;
   err.alloc( 1 );
   HYB_CUDA( cudaMemset( err.p, 0, sizeof( int ) ) );
   auto grid = [&]( long n ) { return dim3( unsigned( std::max< long >( 1, std::min< long >( ( n + 255 ) / 256, 4096 ) ) ) ); };
   // surface colours
   long total = 0;
   for ( int c = 0; c < s.td.m; ++c )
   {
      R->ifaceOff.push_back( total );
      const int* co = &L.colourOff[4 * c];
      total += bdryLaneCount( co[1], co[2], co[3] );
   }
   R->iface.alloc( size_t( std::max< long >( total, 1 ) ) );
   for ( int c = 0; c < s.td.m; ++c )
   {
      const int* co    = &L.colourOff[4 * c];
      const long lanes = bdryLaneCount( co[1], co[2], co[3] );
      if ( lanes == 0 )
         continue;
      const int32_t*  list = L.colourList.p + co[0];
      const BdryLists bl{ list, list + co[1], list + co[1] + co[2], co[1], co[2], co[3] };
      k_rows_surface<<< grid( lanes ), 256 >>>( s.td, d, bl, lanes, R->iface.p + R->ifaceOff[size_t( c )], err.p );
      HYB_CHECK_LAUNCH();
   }
   if ( !R->full )
   {
      int bad = 0;
      HYB_CUDA( cudaMemcpy( &bad, err.p, sizeof( int ), cudaMemcpyDeviceToHost ) );
      if ( bad )
         return nullptr;
      L.rows = std::move( R );
      return L.rows.get();
   }
   // interior colours
   const long nInt = long( s.td.nC ) * d.nPts;
   R->interior.alloc( size_t( std::max< long >( nInt, 1 ) ) );
   for ( int c = 0; c < kInteriorColours; ++c )
   {
      const int count = d.ptsOff[c + 1] - d.ptsOff[c];
      if ( count == 0 )
         continue;
      k_rows_interior<<< grid( long( s.td.nC ) * count ), 256 >>>( s.td, d, d.ptsC + d.ptsOff[c], count,
                                                                  R->interior.p + long( s.td.nC ) * d.ptsOff[c] );
      HYB_CHECK_LAUNCH();
   }
   // all DoFs
   const int       nv = s.td.nV, ne = s.td.nE * ( d.N - 1 ), nf = s.td.nF * d.nIntFace;
   const BdryLists full{ nullptr, nullptr, nullptr, nv, ne, nf };
   const long      surf = bdryLaneCount( nv, ne, nf );
   R->allB1             = long( nv ) * 32;
   R->allB2             = R->allB1 + ( long( ne ) * 8 + 31 ) / 32 * 32;
   R->allB3             = surf;
   R->allN              = surf + nInt;
   R->all.alloc( size_t( std::max< long >( R->allN, 1 ) ) );
   if ( surf > 0 )
   {
      k_rows_surface<<< grid( surf ), 256 >>>( s.td, d, full, surf, R->all.p, err.p );
      HYB_CHECK_LAUNCH();
   }
   if ( nInt > 0 )
   {
      k_rows_interior<<< grid( nInt ), 256 >>>( s.td, d, d.pts, d.nPts, R->all.p + surf );
      HYB_CHECK_LAUNCH();
   }
   int bad = 0;
   HYB_CUDA( cudaMemcpy( &bad, err.p, sizeof( int ), cudaMemcpyDeviceToHost ) );
   if ( bad )
      return nullptr;
   L.rows = std::move( R );
   return L.rows.get();
}

// the row table of level l if it has been built (usable inside a capture)
const RowTables* rowsIf( const Storage& s, int l ) { return s.lv[size_t( l )]->rows.get(); }

RowPass rowPassAll( const RowTables* R )
{
   return R && R->full ? RowPass{ R->all.p, R->allN, R->allB1, R->allB2, R->allB3 } : RowPass{ nullptr, 0, 0, 0, 0 };
}

template < typename T >
void launchApply( const Operator& op, int l, const T* src, T* dst, const T* rhs, int flag, int mode, cudaStream_t stream )
{
   const Storage& s  = *op.st;
   const auto&    L  = s.L( l );
   const int      nc = L.dev.nPts > 0 ? ( op.variable ? L.ptsBlocks : L.quadBlocks ) : 0;
   const int      nb = nc + ( L.dev.nBdry > 0 ? L.bdryBlocks : 0 );
   if ( nb == 0 )
      return;
   const OpDev< T > od = op.dev< T >( l );
   if ( mode == kResidual || mode == kReplace )
      if ( const RowTables* R = rowsIf( s, l ); R && R->full )
      {
         // small and middle levels: the precomputed rows (residual r = b - A u, or r = A u)
         const RowPass rp = rowPassAll( R );
         const int     g  = int( std::max< long >( 1, std::min< long >( ( rp.n + 127 ) / 128, long( s.numSMs ) * 8 ) ) );
         T*            u  = const_cast< T* >( src );
#define HYB_ROWS( M, V ) pdlLaunch( k_row_pass< T, M, V >, dim3( g ), dim3( 128 ), 0, stream, rp, od, u, rhs, dst, T( 0 ), flag )
         if ( mode == kResidual )
         {
            if ( op.variable )
               HYB_ROWS( kRowResidual, true );
            else
               HYB_ROWS( kRowResidual, false );
         }
         else
         {
            if ( op.variable )
               HYB_ROWS( kRowApply, true );
            else
               HYB_ROWS( kRowApply, false );
         }
#undef HYB_ROWS
         HYB_CHECK_LAUNCH();
         return;
      }
#define HYB_APPLY( VAR, MODE ) pdlLaunch( k_apply< T, VAR, MODE >, dim3( nb ), dim3( 128 ), 0, stream, s.td, L.dev, od, src, dst, rhs, flag, nc )
   if ( op.variable )
   {
      if ( mode == kReplace )
         HYB_APPLY( true, kReplace );
      else if ( mode == kAdd )
         HYB_APPLY( true, kAdd );
      else
         HYB_APPLY( true, kResidual );
   }
   else
   {
      if ( mode == kReplace )
         HYB_APPLY( false, kReplace );
      else if ( mode == kAdd )
         HYB_APPLY( false, kAdd );
      else
         HYB_APPLY( false, kResidual );
   }
#undef HYB_APPLY
   HYB_CHECK_LAUNCH();
}

// levels whose cells hold at most this many interior points run the four interior SOR
// colours in one launch (a block per cell); HYB_FUSED_INTERIOR_MAX overrides it
static const int kFusedInteriorMaxPoints = [] {
   const char* e = std::getenv( "HYB_FUSED_INTERIOR_MAX" );
   return e ? std::atoi( e ) : 4096;
}();

template < typename T >
void launchSor( const Operator& op, int l, T* u, const T* rhs, T relax, int flag, cudaStream_t stream, bool backwards = false )
{
   const Storage&   s  = *op.st;
   const auto&      L  = s.L( l );
   const OpDev< T > od = op.dev< T >( l );
   // interface passes: one launch per colour over that colour's surface DoFs
   const RowTables* R = rowsIf( s, l );
   auto iface = [&]( int c ) {
      const int* co = &L.colourOff[4 * c];
      const long lanes = bdryLaneCount( co[1], co[2], co[3] );
      if ( lanes == 0 )
         return;
      const int       nb   = int( std::min< long >( ( lanes + 127 ) / 128, long( s.numSMs ) * 8 ) );
      if ( R )
      {
         const long b1 = long( co[1] ) * 32, b2 = b1 + ( long( co[2] ) * 8 + 31 ) / 32 * 32;
         const RowPass rp{ R->iface.p + R->ifaceOff[size_t( c )], lanes, b1, b2, lanes };
         if ( op.variable )
            pdlLaunch( k_row_pass< T, kRowSor, true >, dim3( nb ), dim3( 128 ), 0, stream, rp, od, u, rhs, (T*) nullptr,
                       relax, flag );
         else
            pdlLaunch( k_row_pass< T, kRowSor, false >, dim3( nb ), dim3( 128 ), 0, stream, rp, od, u, rhs, (T*) nullptr,
                       relax, flag );
         HYB_CHECK_LAUNCH();
         return;
      }
      const int32_t*  list = L.colourList.p + co[0];
      const BdryLists bl{ list, list + co[1], list + co[1] + co[2], co[1], co[2], co[3] };
      if ( op.variable )
         pdlLaunch( k_sor_iface< T, true >, dim3( nb ), dim3( 128 ), 0, stream, s.td, L.dev, od, u, rhs, relax, flag, bl );
      else
         pdlLaunch( k_sor_iface< T, false >, dim3( nb ), dim3( 128 ), 0, stream, s.td, L.dev, od, u, rhs, relax, flag, bl );
      HYB_CHECK_LAUNCH();
   };
   // interior passes
   auto interior = [&]() {
      if ( L.dev.nPts == 0 )
         return;
      // small levels: the four interior colours in one launch, a block per cell
      if ( L.dev.nPts <= kFusedInteriorMaxPoints )
      {
         const int* o  = L.dev.ptsOff;
         const int  bw = backwards ? 1 : 0;
         if ( op.variable )
            pdlLaunch( k_sor_interior_cells< T, true >, dim3( s.td.nC ), dim3( 256 ), 0, stream, s.td, L.dev, od, u, rhs,
                       relax, o[0], o[1], o[2], o[3], o[4], bw );
         else
            pdlLaunch( k_sor_interior_cells< T, false >, dim3( s.td.nC ), dim3( 256 ), 0, stream, s.td, L.dev, od, u, rhs,
                       relax, o[0], o[1], o[2], o[3], o[4], bw );
         HYB_CHECK_LAUNCH();
         return;
      }
      // one launch per colour
      for ( int k = 0; k < kInteriorColours; ++k )
      {
         const int c     = backwards ? kInteriorColours - 1 - k : k;
         const int begin = L.dev.ptsOff[c], count = L.dev.ptsOff[c + 1] - L.dev.ptsOff[c];
         if ( count == 0 )
            continue;
         if ( op.variable )
            pdlLaunch( k_sor_interior< T, true >, dim3( L.colourBlocks ), dim3( 128 ), 0, stream, s.td, L.dev, od, u, rhs,
                       relax, c, begin, count, L.colourBlocks );
         else
            pdlLaunch( k_sor_interior< T, false >, dim3( L.colourBlocks ), dim3( 128 ), 0, stream, s.td, L.dev, od, u, rhs,
                       relax, c, begin, count, L.colourBlocks );
         HYB_CHECK_LAUNCH();
      }
   };
   // forward: surface colours 0..m-1, then the interior colours 0..3; backwards (the
   // multicolour smooth_sor_backwards, P1Operator.hpp:385-400): the same passes reversed
   if ( !backwards )
   {
      for ( int c = 0; c < s.td.m; ++c )
         iface( c );
      interior();
   }
   else
   {
      interior();
      for ( int c = s.td.m - 1; c >= 0; --c )
         iface( c );
   }
}

template < typename T >
void launchJacobi( const Operator& op, int l, const T* src, T* dst, const T* rhs, T relax, int flag, cudaStream_t stream )
{
   const Storage& s  = *op.st;
   const auto&    L  = s.L( l );
   const int      nc = L.dev.nPts > 0 ? L.ptsBlocks : 0;
   const int      nb = nc + ( L.dev.nBdry > 0 ? L.bdryBlocks : 0 );
   if ( nb == 0 )
      return;
   const OpDev< T > od = op.dev< T >( l );
   if ( op.variable )
      pdlLaunch( k_jacobi< T, true >, dim3( nb ), dim3( 128 ), 0, stream, s.td, L.dev, od, src, dst, rhs, relax, flag, nc );
   else
      pdlLaunch( k_jacobi< T, false >, dim3( nb ), dim3( 128 ), 0, stream, s.td, L.dev, od, src, dst, rhs, relax, flag, nc );
   HYB_CHECK_LAUNCH();
}

template < typename T >
void launchProlongate( const Storage& s, int coarseL, const T* coarse, T* fine, int flag, bool add, cudaStream_t stream )
{
   const auto& F  = s.L( coarseL + 1 );
   const auto& C  = s.L( coarseL );
   const int   nc = F.dev.nPts > 0 ? F.ptsBlocks : 0;
   const int   nb = nc + ( F.dev.nBdry > 0 ? F.bdryBlocks : 0 );
   if ( nb == 0 )
      return;
   if ( add )
      pdlLaunch( k_prolongate< T, true >, dim3( nb ), dim3( 128 ), 0, stream, s.td, F.dev, C.dev.W, C.dev.stride, coarse, fine, flag, nc );
   else
      pdlLaunch( k_prolongate< T, false >, dim3( nb ), dim3( 128 ), 0, stream, s.td, F.dev, C.dev.W, C.dev.stride, coarse, fine, flag, nc );
   HYB_CHECK_LAUNCH();
}

template < typename T >
void launchRestrict( const Storage& s, int fineL, const T* fine, T* coarse, int flag, cudaStream_t stream )
{
   const auto& F  = s.L( fineL );
   const auto& C  = s.L( fineL - 1 );
   const int   nc = C.dev.nSeg > 0 ? C.cellBlocks : 0;
   const int   nb = nc + ( C.dev.nBdry > 0 ? C.bdryBlocks : 0 );
   if ( nb == 0 )
      return;
   pdlLaunch( k_restrict< T >, dim3( nb ), dim3( 128 ), 0, stream, s.td, C.dev, F.dev.W, F.dev.stride, fine, coarse, flag, nc );
   HYB_CHECK_LAUNCH();
}

template < typename T >
void launchLincomb( const Storage& s, int l, T* dst, int n, const double* sc, const T* const* src, bool add, int flag,
                    cudaStream_t stream )
{
   const auto& L = s.L( l );
   pdlLaunch( k_lincomb< T >, dim3( dim3( L.slabBlocks, s.td.nC ) ), dim3( 256 ), 0, stream, s.td, L.dev, dst, n, T( n > 0 ? sc[0] : 0 ), n > 0 ? src[0] : nullptr, T( n > 1 ? sc[1] : 0 ),
       n > 1 ? src[1] : nullptr, T( n > 2 ? sc[2] : 0 ), n > 2 ? src[2] : nullptr, add ? 1 : 0, flag );
   HYB_CHECK_LAUNCH();
}

// dot product into the device double `result`, with one partial sum per block in `partial`
// (at least maxPartialSlots( s ) doubles)
template < typename T >
void launchDot( const Storage& s, int l, const T* a, const T* b, int flag, double* partial, double* result,
                cudaStream_t stream )
{
   const auto& L = s.L( l );
   pdlLaunch( k_dot_partial< T >, dim3( dim3( L.slabBlocks, s.td.nC ) ), dim3( 256 ), 0, stream, s.td, L.dev, a, b, flag, partial );
   HYB_CHECK_LAUNCH();
   pdlLaunch( k_reduce_final, dim3( 1 ), dim3( 1024 ), 0, stream, partial, L.slabBlocks * s.td.nC, result );
   HYB_CHECK_LAUNCH();
}

// dot product into the storage's device scalar slot `slot`
template < typename T >
void launchDot( const Storage& s, int l, const T* a, const T* b, int flag, int slot, cudaStream_t stream )
{
   launchDot< T >( s, l, a, b, flag, s.partial.p, s.scalars.p + slot, stream );
}

template < typename TD, typename TS >
void launchConvert( const Storage& s, int l, TD* dst, const TS* src, cudaStream_t stream )
{
   const auto&  L = s.L( l );
   const size_t n = size_t( s.td.nC ) * L.dev.stride;
   pdlLaunch( k_convert< TD, TS >, dim3( unsigned( ( n + 255 ) / 256 ) ), dim3( 256 ), 0, stream, L.dev, dst, src, s.td.nC );
   HYB_CHECK_LAUNCH();
}

template < typename T >
void launchAddCorrection( const Storage& s, int l, double* x, const T* e, int flag, cudaStream_t stream )
{
   const auto& L = s.L( l );
   pdlLaunch( k_add_correction< double, T >, dim3( dim3( L.slabBlocks, s.td.nC ) ), dim3( 256 ), 0, stream, s.td, L.dev, x, e, flag );
   HYB_CHECK_LAUNCH();
}

// Coarse CG in FP64 on device scratch (x, b given; r, p, ap scratch)
struct CgScratch
{
   std::unique_ptr< Function > r, p, ap;
   DevBuf< int >               status;
};


void launchCg( const Operator& op, int l, double* x, const double* b, CgScratch& cs, double tol, int maxIter,
               cudaStream_t stream )
{
   const Storage& s = *op.st;
   if ( !cs.r || cs.r->minL > l || cs.r->maxL < l )
   {
      cs.r.reset( makeFunction( op.st, l, l, HYB_F64 ) );
      cs.p.reset( makeFunction( op.st, l, l, HYB_F64 ) );
      cs.ap.reset( makeFunction( op.st, l, l, HYB_F64 ) );
      cs.status.alloc( 4 );
   }
   const OpDev< double > od = op.dev< double >( l );
   const RowPass         rp = rowPassAll( rowsIf( s, l ) );
   if ( op.variable )
      pdlLaunch( k_cg< true >, dim3( 1 ), dim3( 256 ), 0, stream, s.td, s.L( l ).dev, od, x, b, cs.r->ptr< double >( l ), cs.p->ptr< double >( l ),
                                             cs.ap->ptr< double >( l ), tol, maxIter, cs.status.p, rp );
   else
      pdlLaunch( k_cg< false >, dim3( 1 ), dim3( 256 ), 0, stream, s.td, s.L( l ).dev, od, x, b, cs.r->ptr< double >( l ), cs.p->ptr< double >( l ),
                                              cs.ap->ptr< double >( l ), tol, maxIter, cs.status.p, rp );
   HYB_CHECK_LAUNCH();
}

// ChebyshevSmoother::setupCoefficients (src/hyteg/solvers/ChebyshevSmoother.hpp:98-188):
// the power-basis coefficients w_0 .. w_{k-1} of p with 1 - l p(l) = T_k((th - l) / de) /
// T_k(th / de) on the eigenvalue interval [lower, upper] of D^-1 A (th, de its midpoint and
// half width, T_k the Chebyshev polynomial of the first kind, expanded by its three-term
// recurrence); the smoother adds p(D^-1 A) D^-1 (b - A x) to x. Orders 1 to 5.
std::vector< double > chebyshevCoefficients( int order, double lower, double upper )
{
   require( order >= 1 && order <= 5, "Chebyshev order must be in [1, 5]" );
   require( std::isfinite( lower ) && std::isfinite( upper ) && 0 < lower && lower < upper,
            "Chebyshev bounds must satisfy 0 < lower < upper" );
   const double th = 0.5 * ( upper + lower ), de = 0.5 * ( upper - lower );
   const double a = th / de, c = -1.0 / de; // T_k's argument a + c l
   std::vector< double > prev( order + 1, 0.0 ), cur( order + 1, 0.0 ), next( order + 1, 0.0 );
   prev[0] = 1.0;
   cur[0]  = a;
   cur[1]  = c;
   for ( int n = 1; n < order; ++n )
   {
      std::fill( next.begin(), next.end(), 0.0 );
      for ( int i = 0; i <= n; ++i )
      {
         next[i] += 2 * a * cur[i] - prev[i];
         next[i + 1] += 2 * c * cur[i];
      }
      prev.swap( cur );
      cur.swap( next );
   }
   std::vector< double > w( order );
   for ( int i = 1; i <= order; ++i )
      w[i - 1] = -cur[i] / cur[0];
   return w;
}

// diag(A)^-1 of level l into out (every replica)
template < typename T >
void launchInvDiag( const Operator& op, int l, const T* zeros, T* out, cudaStream_t stream )
{
   const Storage& s  = *op.st;
   const auto&    L  = s.L( l );
   const int      nc = L.dev.nPts > 0 ? L.ptsBlocks : 0;
   const int      nb = nc + ( L.dev.nBdry > 0 ? L.bdryBlocks : 0 );
   if ( nb == 0 )
      return;
   const OpDev< T > od = op.dev< T >( l );
   if ( op.variable )
      k_inv_diag< T, true ><<< nb, 128, 0, stream >>>( s.td, L.dev, od, zeros, out, nc );
   else
      k_inv_diag< T, false ><<< nb, 128, 0, stream >>>( s.td, L.dev, od, zeros, out, nc );
   HYB_CHECK_LAUNCH();
}

template < typename T >
void launchChebUpdate( const Storage& s, int l, const T* inv, T* t, T* x, T w, cudaStream_t stream )
{
   const long long n = (long long) s.td.nC * s.L( l ).dev.stride;
   const int       g = int( std::max< long long >( 1, std::min< long long >( ( n + 255 ) / 256, (long long) s.numSMs * 8 ) ) );
   pdlLaunch( k_cheb_update< T >, dim3( g ), dim3( 256 ), 0, stream, n, inv, t, x, w );
   HYB_CHECK_LAUNCH();
}

// ---------------------------------------------------------------------------
// Geometric multigrid (GeometricMultigridSolver.hpp:136-235)
// ---------------------------------------------------------------------------
struct Gmg
{
   Storage*  st;
   Operator* op;
   int       minL, maxL, pre, post, smoother, coarseMaxIter;
   int       cycleType = HYB_CYCLE_V;
   double    relax, coarseTol;
   std::unique_ptr< Function > tmp64;         // gmg_tmp
   std::unique_ptr< Function > x32, b32, t32; // FP32 inner hierarchy (mixed precision)
   std::unique_ptr< Function > r64;           // FP64 residual (mixed precision)
   std::unique_ptr< Function > cx64, cb64;    // FP64 coarse-solve copies of the FP32 hierarchy
   std::vector< double >       cheb;          // Chebyshev smoother: omega_0 .. omega_{order-1}
   std::unique_ptr< Function > inv64, inv32;  // Chebyshev smoother: diag(A)^-1 per level
   std::unique_ptr< Function > ch64, ch32;    // Chebyshev smoother: second temporary
   CgScratch                   cg;
   // reduction scratch of this solver, so that solvers sharing a storage can run on
   // different streams at the same time: scalars[0] = ||r||^2, scalars[1] = ||b||^2
   DevBuf< double >            partial, scalars;
   double*                     hostScalar = nullptr; // pinned, 2 doubles
   // Levels <= progTop of a V-cycle run as one program-kernel launch (-1: none), with one
   // recorded phase list per (x, b, compute type, top level).
   int progTop = -1;
   struct Program
   {
      const void*     x;
      const void*     b;
      int             dtype, top, n;
      DevBuf< Phase > phases;
   };
   std::vector< std::unique_ptr< Program > > programs;
   cudaStream_t                cap = nullptr; // capture stream
   // captured graphs keyed by (x, b, level, kind)
   struct G
   {
      const void* x;
      const void* b;
      int         level, kind;
      cudaGraphExec_t exec;
      long long       kernels; // kernel launches captured in the graph
   };
   std::vector< G > graphs;

   ~Gmg()
   {
      for ( auto& g : graphs )
         cudaGraphExecDestroy( g.exec );
      if ( cap )
         cudaStreamDestroy( cap );
      if ( hostScalar )
         cudaFreeHost( hostScalar );
   }
};

constexpr int kGmgFlag = HYB_INNER | HYB_NEUMANN;

template < typename T >
void smooth( Gmg& g, int l, T* x, const T* b, T* scratch, cudaStream_t stream )
{
   if ( g.smoother == HYB_SMOOTHER_SOR )
      launchSor< T >( *g.op, l, x, b, T( g.relax ), kGmgFlag, stream );
   else if ( g.smoother == HYB_SMOOTHER_SYMMETRIC_SOR )
   {
      // SymmetricSORSmoother::solve (SymmetricSORSmoother.hpp:38-57): forward, then backwards
      launchSor< T >( *g.op, l, x, b, T( g.relax ), kGmgFlag, stream );
      launchSor< T >( *g.op, l, x, b, T( g.relax ), kGmgFlag, stream, true );
   }
   else if ( g.smoother == HYB_SMOOTHER_CHEBYSHEV )
   {
      // ChebyshevSmoother::solve (ChebyshevSmoother.hpp:49-96): t = D^-1 (b - A x), x += w_0 t,
      // then t = D^-1 A t, x += w_k t. scratch (the solver's residual vector) and the second
      // temporary are only written on Inner|Neumann DoFs, so they hold 0 elsewhere.
      const bool      f64 = std::is_same< T, double >::value;
      const T*        inv = ( f64 ? g.inv64 : g.inv32 )->template ptr< T >( l );
      T*              t   = scratch;
      T*              t2  = ( f64 ? g.ch64 : g.ch32 )->template ptr< T >( l );
      launchApply< T >( *g.op, l, x, t, b, kGmgFlag, kResidual, stream );
      launchChebUpdate< T >( *g.st, l, inv, t, x, T( g.cheb[0] ), stream );
      for ( size_t k = 1; k < g.cheb.size(); ++k )
      {
         launchApply< T >( *g.op, l, t, t2, nullptr, kGmgFlag, kReplace, stream );
         launchChebUpdate< T >( *g.st, l, inv, t2, x, T( g.cheb[k] ), stream );
         std::swap( t, t2 );
      }
   }
   else
   {
      // Jacobi needs the old iterate: scratch = x, then x = scratch + relax D^-1 (b - A scratch)
      HYB_CUDA( cudaMemcpyAsync( scratch, x, size_t( g.st->td.nC ) * g.st->L( l ).dev.stride * sizeof( T ),
                                 cudaMemcpyDeviceToDevice, stream ) );
      launchJacobi< T >( *g.op, l, scratch, x, b, T( g.relax ), kGmgFlag, stream );
   }
}

// coarse solve: FP64 CG; an FP32 hierarchy is solved through FP64 copies
void coarseSolve( Gmg& g, double* x, const double* b, cudaStream_t stream )
{
   launchCg( *g.op, g.minL, x, b, g.cg, g.coarseTol, g.coarseMaxIter, stream );
}
void coarseSolve( Gmg& g, float* x, const float* b, cudaStream_t stream )
{
   const int l = g.minL;
   launchConvert< double, float >( *g.st, l, g.cx64->ptr< double >( l ), x, stream );
   launchConvert< double, float >( *g.st, l, g.cb64->ptr< double >( l ), b, stream );
   launchCg( *g.op, l, g.cx64->ptr< double >( l ), g.cb64->ptr< double >( l ), g.cg, g.coarseTol, g.coarseMaxIter, stream );
   launchConvert< float, double >( *g.st, l, x, g.cx64->ptr< double >( l ), stream );
}

// ---------------------------------------------------------------------------
// Program-kernel V-cycle for the small levels: the phases mirror vcycle() below, launch
// for launch, with each launch's grid as the phase's virtual grid.
// ---------------------------------------------------------------------------
// levels whose slabs hold at most this many points (all cells) run in the program kernel;
// HYB_PROGRAM_MAX_POINTS overrides it (0: never)
constexpr long kProgramMaxPoints = 4096;

struct PhaseList
{
   const Gmg&           g;
   std::vector< Phase > ph;

   // one thread block runs the program: a phase has one virtual block for its cell-interior
   // loop (if the launch it replaces has one) and one for its surface or flat loop
   Phase& add( int kind, int level, int blocks, int cellBlocks )
   {
      Phase P{};
      P.kind       = kind;
      P.level      = level;
      P.cellBlocks = cellBlocks > 0 ? 1 : 0;
      P.blocks     = std::max( P.cellBlocks + ( blocks > cellBlocks ? 1 : 0 ), 1 );
      P.op32       = g.op->dev< float >( level );
      P.op64       = g.op->dev< double >( level );
      ph.push_back( P );
      return ph.back();
   }
   long slabElems( int l ) const { return long( g.st->td.nC ) * g.st->L( l ).dev.stride; }
   // the row table of level l for the passes of this (constant) operator, built on first use
   const RowTables* rows( int l ) const
   {
      const RowTables* R = ensureRows( *g.st, l );
      return R && R->full ? R : nullptr;
   }
   int  flatBlocks( long n ) const
   {
      return int( std::min< long >( ( n + 127 ) / 128, long( g.st->numSMs ) * 8 ) );
   }

   template < typename T >
   void smooth( int l, T* x, const T* b, T* scratch )
   {
      const Storage& s = *g.st;
      const auto&    L = s.L( l );
      if ( g.smoother == HYB_SMOOTHER_SOR || g.smoother == HYB_SMOOTHER_SYMMETRIC_SOR )
      {
         auto iface = [&]( int c ) {
            const int* co    = &L.colourOff[4 * c];
            const long lanes = bdryLaneCount( co[1], co[2], co[3] );
            if ( lanes == 0 )
               return;
            const int32_t* list = L.colourList.p + co[0];
            Phase&         P    = add( kPhSorIface, l, int( std::min< long >( ( lanes + 127 ) / 128, long( s.numSMs ) * 8 ) ), 0 );
            P.p0                = x;
            P.p1                = const_cast< T* >( b );
            P.relax             = g.relax;
            P.flag              = kGmgFlag;
            P.bl                = BdryLists{ list, list + co[1], list + co[1] + co[2], co[1], co[2], co[3] };
            if ( const RowTables* R = rows( l ) )
            {
               const long b1 = long( co[1] ) * 32, b2 = b1 + ( long( co[2] ) * 8 + 31 ) / 32 * 32;
               P.rp          = RowPass{ R->iface.p + R->ifaceOff[size_t( c )], lanes, b1, b2, lanes };
               P.blocks      = 1;
               P.cellBlocks  = 0;
            }
         };
         auto interior = [&]( int c ) {
            const int count = L.dev.ptsOff[c + 1] - L.dev.ptsOff[c];
            if ( count == 0 )
               return;
            Phase& P = add( kPhSorInterior, l, L.colourBlocks, L.colourBlocks );
            P.p0     = x;
            P.p1     = const_cast< T* >( b );
            P.relax  = g.relax;
            P.a0     = c;
            P.a1     = L.dev.ptsOff[c];
            P.a2     = count;
            if ( const RowTables* R = rows( l ) )
            {
               const long n = long( s.td.nC ) * count;
               P.rp         = RowPass{ R->interior.p + long( s.td.nC ) * L.dev.ptsOff[c], n, 0, 0, 0 };
               P.blocks     = 1;
               P.cellBlocks = 0;
            }
         };
         for ( int c = 0; c < s.td.m; ++c )
            iface( c );
         for ( int c = 0; c < kInteriorColours; ++c )
            interior( c );
         if ( g.smoother == HYB_SMOOTHER_SYMMETRIC_SOR )
         {
            for ( int c = kInteriorColours - 1; c >= 0; --c )
               interior( c );
            for ( int c = s.td.m - 1; c >= 0; --c )
               iface( c );
         }
      }
      else
      {
         Phase& C = add( kPhCopy, l, flatBlocks( slabElems( l ) ), 0 );
         C.p0     = scratch;
         C.p1     = x;
         C.n      = slabElems( l );
         const int nc = L.dev.nPts > 0 ? L.ptsBlocks : 0;
         Phase&    P  = add( kPhJacobi, l, nc + ( L.dev.nBdry > 0 ? L.bdryBlocks : 0 ), nc );
         P.p0         = scratch;
         P.p1         = x;
         P.p2         = const_cast< T* >( b );
         P.relax      = g.relax;
         P.flag       = kGmgFlag;
      }
   }

   void cg( int l, double* x, const double* b )
   {
      Phase& P = add( kPhCg, l, 1, 0 );
      P.p0     = x;
      P.p1     = const_cast< double* >( b );
      P.p2     = g.cg.r->ptr< double >( l );
      P.p3     = g.cg.p->ptr< double >( l );
      P.p4     = g.cg.ap->ptr< double >( l );
      P.status = g.cg.status.p;
      P.relax  = g.coarseTol;
      P.a0     = g.coarseMaxIter;
      P.rp     = rowPassAll( rows( l ) );
   }

   void coarse( double* x, const double* b ) { cg( g.minL, x, b ); }
   void coarse( float* x, const float* b )
   {
      const int  l = g.minL;
      const long n = slabElems( l );
      Phase&     A = add( kPhToF64, l, flatBlocks( n ), 0 );
      A.p0         = g.cx64->ptr< double >( l );
      A.p1         = x;
      A.n          = n;
      Phase& B     = add( kPhToF64, l, flatBlocks( n ), 0 );
      B.p0         = g.cb64->ptr< double >( l );
      B.p1         = const_cast< float* >( b );
      B.n          = n;
      cg( l, g.cx64->ptr< double >( l ), g.cb64->ptr< double >( l ) );
      Phase& C = add( kPhToF32, l, flatBlocks( n ), 0 );
      C.p0     = x;
      C.p1     = g.cx64->ptr< double >( l );
      C.n      = n;
   }

   template < typename T >
   void vcycle( Function& x, Function& b, Function& tmp, int l )
   {
      if ( l == g.minL )
      {
         coarse( x.ptr< T >( l ), b.ptr< T >( l ) );
         return;
      }
      const Storage& s = *g.st;
      for ( int i = 0; i < g.pre; ++i )
         smooth< T >( l, x.ptr< T >( l ), b.ptr< T >( l ), tmp.ptr< T >( l ) );
      {
         const auto& L  = s.L( l );
         const int   nc = L.dev.nPts > 0 ? L.ptsBlocks : 0;
         Phase&      P  = add( kPhResidual, l, nc + ( L.dev.nBdry > 0 ? L.bdryBlocks : 0 ), nc );
         P.p0           = x.ptr< T >( l );
         P.p1           = tmp.ptr< T >( l );
         P.p2           = b.ptr< T >( l );
         P.flag         = kGmgFlag;
         if ( const RowTables* R = rows( l ) )
         {
            P.rp         = rowPassAll( R );
            P.blocks     = 1;
            P.cellBlocks = 0;
         }
      }
      {
         const auto& C  = s.L( l - 1 );
         const int   nc = C.dev.nSeg > 0 ? C.cellBlocks : 0;
         Phase&      P  = add( kPhRestrict, l - 1, nc + ( C.dev.nBdry > 0 ? C.bdryBlocks : 0 ), nc );
         P.p0           = tmp.ptr< T >( l );
         P.p1           = b.ptr< T >( l - 1 );
         P.flag         = kGmgFlag;
      }
      {
         Phase& P = add( kPhZero, l - 1, flatBlocks( slabElems( l - 1 ) ), 0 );
         P.p0     = x.ptr< T >( l - 1 );
         P.n      = slabElems( l - 1 );
      }
      vcycle< T >( x, b, tmp, l - 1 );
      if ( g.cycleType == HYB_CYCLE_W )
         vcycle< T >( x, b, tmp, l - 1 );
      {
         const auto& F  = s.L( l );
         const int   nc = F.dev.nPts > 0 ? F.ptsBlocks : 0;
         Phase&      P  = add( kPhProlongAdd, l, nc + ( F.dev.nBdry > 0 ? F.bdryBlocks : 0 ), nc );
         P.p0           = x.ptr< T >( l - 1 );
         P.p1           = x.ptr< T >( l );
         P.flag         = kGmgFlag;
      }
      for ( int i = 0; i < g.post; ++i )
         smooth< T >( l, x.ptr< T >( l ), b.ptr< T >( l ), tmp.ptr< T >( l ) );
   }
};

// Record (once, outside any stream capture) the program of the sub-cycle at level `top`
// for the V-cycle on (x, b, tmp) in type T.
template < typename T >
void ensureProgram( Gmg& g, Function& x, Function& b, Function& tmp, int top )
{
   const int dtype = std::is_same< T, double >::value ? HYB_F64 : HYB_F32;
   for ( auto& p : g.programs )
      if ( p->x == &x && p->b == &b && p->dtype == dtype && p->top == top )
         return;
   PhaseList pl{ g, {} };
   pl.vcycle< T >( x, b, tmp, top );
   auto prog   = std::make_unique< Gmg::Program >();
   prog->x     = &x;
   prog->b     = &b;
   prog->dtype = dtype;
   prog->top   = top;
   prog->n     = int( pl.ph.size() );
   prog->phases.upload( pl.ph );
   g.programs.push_back( std::move( prog ) );
}

template < typename T >
void launchProgram( Gmg& g, Function& x, Function& b, int top, cudaStream_t stream )
{
   const int           dtype = std::is_same< T, double >::value ? HYB_F64 : HYB_F32;
   const Gmg::Program* prog  = nullptr;
   for ( auto& p : g.programs )
      if ( p->x == &x && p->b == &b && p->dtype == dtype && p->top == top )
         prog = p.get();
   require( prog != nullptr, "program of the coarse V-cycle was not recorded" );
   const Phase* ph  = prog->phases.p;
   const auto*  lt  = (const LevelDev*) g.st->lvTable.p;
   const int    nLv = int( g.st->lvTable.n );
   if ( g.op->variable )
      pdlLaunch( k_program< T, true >, dim3( 1 ), dim3( kProgramThreads ), 0, stream, g.st->td, lt, ph, prog->n, nLv );
   else
      pdlLaunch( k_program< T, false >, dim3( 1 ), dim3( kProgramThreads ), 0, stream, g.st->td, lt, ph, prog->n, nLv );
   HYB_CHECK_LAUNCH();
}

template < typename T >
void vcycle( Gmg& g, Function& x, Function& b, Function& tmp, int l, cudaStream_t stream )
{
   if ( l <= g.progTop )
   {
      launchProgram< T >( g, x, b, l, stream );
      return;
   }
   if ( l == g.minL )
   {
      coarseSolve( g, x.ptr< T >( l ), b.ptr< T >( l ), stream );
      return;
   }
   for ( int i = 0; i < g.pre; ++i )
      smooth< T >( g, l, x.ptr< T >( l ), b.ptr< T >( l ), tmp.ptr< T >( l ), stream );
   // tmp = b - A x ; restricted straight into b on the coarser level (b.assign(tmp) on flag)
   launchApply< T >( *g.op, l, x.ptr< T >( l ), tmp.ptr< T >( l ), b.ptr< T >( l ), kGmgFlag, kResidual, stream );
   launchRestrict< T >( *g.st, l, tmp.ptr< T >( l ), b.ptr< T >( l - 1 ), kGmgFlag, stream );
   HYB_CUDA( cudaMemsetAsync( x.ptr< T >( l - 1 ), 0, x.levelBytes( l - 1 ), stream ) ); // x.interpolate(0, l-1)
   vcycle< T >( g, x, b, tmp, l - 1, stream );
   if ( g.cycleType == HYB_CYCLE_W ) // GeometricMultigridSolver.hpp:201-204
      vcycle< T >( g, x, b, tmp, l - 1, stream );
   launchProlongate< T >( *g.st, l - 1, x.ptr< T >( l - 1 ), x.ptr< T >( l ), kGmgFlag, true, stream );
   for ( int i = 0; i < g.post; ++i )
      smooth< T >( g, l, x.ptr< T >( l ), b.ptr< T >( l ), tmp.ptr< T >( l ), stream );
}

// Graph-captured work units.
enum GraphKind : int
{
   kCycle64      = 0, // one FP64 V-cycle
   kCycle64Norm  = 1, // FP64 V-cycle, then r = b - A x and ||r||^2 into scalar slot 0
   kMixedStep    = 2, // FP32 V-cycle on A e = r (r from the previous step), x += e, new r and ||r||^2
   kNorm64       = 3, // r = b - A x into gmg_tmp and ||r||^2
   kNormMixed    = 4, // r = b - A x into the FP64 residual of the mixed solver and ||r||^2
   kFmg64        = 8, // full multigrid, kFmg64 + c: c FP64 V-cycles per level (1 <= c <= 8)
};

void enqueue( Gmg& g, Function& x, Function& b, int l, int kind, cudaStream_t s )
{
   if ( kind == kCycle64 || kind == kCycle64Norm )
      vcycle< double >( g, x, b, *g.tmp64, l, s );
   if ( kind == kMixedStep )
   {
      // FP32 V-cycle on the residual equation (mixedPrecisionIterativeRefinement.cpp:162-171)
      launchConvert< float, double >( *g.st, l, g.b32->ptr< float >( l ), g.r64->ptr< double >( l ), s );
      HYB_CUDA( cudaMemsetAsync( g.x32->ptr< float >( l ), 0, g.x32->levelBytes( l ), s ) );
      vcycle< float >( g, *g.x32, *g.b32, *g.t32, l, s );
      launchAddCorrection< float >( *g.st, l, x.ptr< double >( l ), g.x32->ptr< float >( l ), kGmgFlag, s );
   }
   if ( kind > kFmg64 && kind <= kFmg64 + 8 )
   {
      // FullMultigridSolver::solve (FullMultigridSolver.hpp:51-75) with linear FMG
      // prolongation on inner and Neumann DoFs
      for ( int lc = g.minL; lc <= l; ++lc )
      {
         for ( int c = 0; c < kind - kFmg64; ++c )
            vcycle< double >( g, x, b, *g.tmp64, lc, s );
         if ( lc < l )
            launchProlongate< double >( *g.st, lc, x.ptr< double >( lc ), x.ptr< double >( lc + 1 ), kGmgFlag, false, s );
      }
      return;
   }
   if ( kind != kCycle64 )
   {
      Function& r = ( kind == kCycle64Norm || kind == kNorm64 ) ? *g.tmp64 : *g.r64;
      launchApply< double >( *g.op, l, x.ptr< double >( l ), r.ptr< double >( l ), b.ptr< double >( l ), kGmgFlag, kResidual, s );
      launchDot< double >( *g.st, l, r.ptr< double >( l ), r.ptr< double >( l ), kGmgFlag, g.partial.p, g.scalars.p, s );
   }
}

// everything a captured graph needs is allocated before capture begins
// the Chebyshev smoother's inverse diagonals and temporaries for the hierarchies in use
void ensureChebyshev( Gmg& g )
{
   if ( g.smoother != HYB_SMOOTHER_CHEBYSHEV )
      return;
   require( !g.cheb.empty(), "the Chebyshev smoother needs its coefficients (hyb_gmg_setup_chebyshev)" );
   auto fill = [&]( std::unique_ptr< Function >& inv, std::unique_ptr< Function >& t2, int dtype ) {
      if ( inv )
         return;
      inv.reset( makeFunction( g.st, g.minL, g.maxL, dtype ) );
      t2.reset( makeFunction( g.st, g.minL, g.maxL, dtype ) );
      for ( int l = g.minL; l <= g.maxL; ++l )
         if ( dtype == HYB_F64 )
            launchInvDiag< double >( *g.op, l, t2->ptr< double >( l ), inv->ptr< double >( l ), nullptr );
         else
            launchInvDiag< float >( *g.op, l, t2->ptr< float >( l ), inv->ptr< float >( l ), nullptr );
      HYB_CUDA( cudaDeviceSynchronize() );
   };
   fill( g.inv64, g.ch64, HYB_F64 );
   if ( g.x32 )
      fill( g.inv32, g.ch32, HYB_F32 );
}

void prepare( Gmg& g )
{
   ensureChebyshev( g );
   for ( int l = g.minL; l <= g.maxL; ++l )
      ensureRows( *g.st, l );
   if ( !g.cg.r )
   {
      g.cg.r.reset( makeFunction( g.st, g.minL, g.minL, HYB_F64 ) );
      g.cg.p.reset( makeFunction( g.st, g.minL, g.minL, HYB_F64 ) );
      g.cg.ap.reset( makeFunction( g.st, g.minL, g.minL, HYB_F64 ) );
      g.cg.status.alloc( 4 );
   }
}

void initGmg( Gmg& g, Storage* s, Operator* op, int minL, int maxL, int pre, int post, double relax, int smoother,
              double coarseTol, int coarseMaxIter )
{
   g.st            = s;
   g.op            = op;
   g.minL          = minL;
   g.maxL          = maxL;
   g.pre           = pre;
   g.post          = post;
   g.relax         = relax;
   g.smoother      = smoother;
   g.coarseTol     = coarseTol;
   g.coarseMaxIter = coarseMaxIter;
   g.tmp64.reset( makeFunction( s, minL, maxL, HYB_F64 ) );
   g.partial.alloc( s->partial.n );
   g.scalars.alloc( 2 );
   HYB_CUDA( cudaMallocHost( &g.hostScalar, 2 * sizeof( double ) ) );
   long maxPoints = kProgramMaxPoints;
   if ( const char* e = std::getenv( "HYB_PROGRAM_MAX_POINTS" ) )
      maxPoints = std::atol( e );
   g.progTop = -1;
   for ( int l = minL; l <= maxL; ++l )
      if ( long( s->td.nC ) * s->L( l ).dev.stride <= maxPoints )
         g.progTop = l;
   if ( smoother == HYB_SMOOTHER_CHEBYSHEV )
      g.progTop = -1; // the program kernel has no Chebyshev phases
}


// the FP32 hierarchy and FP64 residual of the mixed-precision solver
void ensureMixed( Gmg& g )
{
   if ( g.x32 )
      return;
   Storage* s = g.st;
   g.x32.reset( makeFunction( s, g.minL, g.maxL, HYB_F32 ) );
   g.b32.reset( makeFunction( s, g.minL, g.maxL, HYB_F32 ) );
   g.t32.reset( makeFunction( s, g.minL, g.maxL, HYB_F32 ) );
   g.r64.reset( makeFunction( s, g.minL, g.maxL, HYB_F64 ) );
   g.cx64.reset( makeFunction( s, g.minL, g.minL, HYB_F64 ) );
   g.cb64.reset( makeFunction( s, g.minL, g.minL, HYB_F64 ) );
}

void runGraph( Gmg& g, Function& x, Function& b, int l, int kind, cudaStream_t stream )
{
   for ( auto& G : g.graphs )
      if ( G.x == &x && G.b == &b && G.level == l && G.kind == kind )
      {
         HYB_CUDA( cudaGraphLaunch( G.exec, stream ) );
         g_launches.fetch_add( G.kernels, std::memory_order_relaxed );
         return;
      }
   prepare( g );
   if ( g.progTop >= g.minL )
   {
      const int top = std::min( l, g.progTop );
      if ( kind == kCycle64 || kind == kCycle64Norm )
         ensureProgram< double >( g, x, b, *g.tmp64, top );
      if ( kind > kFmg64 && kind <= kFmg64 + 8 )
         for ( int t = g.minL; t <= top; ++t )
            ensureProgram< double >( g, x, b, *g.tmp64, t );
      if ( kind == kMixedStep )
         ensureProgram< float >( g, *g.x32, *g.b32, *g.t32, top );
   }
   if ( !g.cap )
      HYB_CUDA( cudaStreamCreateWithFlags( &g.cap, cudaStreamNonBlocking ) );
   // make the capture stream wait for prior work on the caller's stream
   cudaEvent_t ev;
   HYB_CUDA( cudaEventCreateWithFlags( &ev, cudaEventDisableTiming ) );
   HYB_CUDA( cudaEventRecord( ev, stream ) );
   HYB_CUDA( cudaStreamWaitEvent( g.cap, ev, 0 ) );
   HYB_CUDA( cudaStreamSynchronize( g.cap ) );
   HYB_CUDA( cudaEventDestroy( ev ) );
   cudaGraph_t     graph = nullptr;
   const long long before = g_launches.load();
   HYB_CUDA( cudaStreamBeginCapture( g.cap, cudaStreamCaptureModeThreadLocal ) );
   try
   {
      enqueue( g, x, b, l, kind, g.cap );
   }
   catch ( ... )
   {
      cudaStreamEndCapture( g.cap, &graph );
      if ( graph )
         cudaGraphDestroy( graph );
      throw;
   }
   HYB_CUDA( cudaStreamEndCapture( g.cap, &graph ) );
   const long long captured = g_launches.load() - before;
   g_launches.fetch_sub( captured ); // counted when the graph runs
   cudaGraphExec_t exec;
   HYB_CUDA( cudaGraphInstantiate( &exec, graph, 0 ) );
   HYB_CUDA( cudaGraphDestroy( graph ) );
   g.graphs.push_back( { &x, &b, l, kind, exec, captured } );
   HYB_CUDA( cudaGraphLaunch( exec, stream ) );
   g_launches.fetch_add( captured );
}

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

int hyb_operator_create_divkgrad_rff( hyb_storage* s, int minL, int maxL, const double* w, const double* phase,
                                      int modes, double sigma, double radial, hyb_operator** out )
{
   HYB_API_BEGIN
   require( s && w && phase && out, "null argument" );
   require( modes > 0 && modes <= 4096, "modes must be in [1, 4096]" );
   *out = reinterpret_cast< hyb_operator* >( makeDivKGradRff( ST( s ), minL, maxL, w, phase, modes, sigma, radial ) );
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
   require( !op->variable, "stencils are stored for constant-coefficient operators only" );
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
                smoother == HYB_SMOOTHER_CHEBYSHEV,
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
   g->graphs.clear();
   g->programs.clear();
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
// address is looked up once per device, with that device current.
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
          st.td, L.dev, a->ptr< double >( level ), b->ptr< double >( level ), flag, scratch );
   else
      k_dot_partial< float ><<< dim3( L.slabBlocks, st.td.nC ), 256, 0, S( stream ) >>>(
          st.td, L.dev, a->ptr< float >( level ), b->ptr< float >( level ), flag, scratch );
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
