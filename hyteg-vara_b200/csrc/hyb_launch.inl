// Kernel launchers of the level operations, row tables, coarse CG and the Chebyshev
// coefficients.
// (part of the single translation unit hyb_capi.cu, included inside namespace hyb)

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
// The VAR template argument of an operator's kernels: 0 constant stencils, 1 variable
// coefficient from nodal values, 2 variable coefficient at quadrature points. withVar calls
// f with it as a compile-time constant (std::integral_constant).
inline int varKind( const Operator& op ) { return !op.variable ? 0 : ( op.kq64.empty() ? 1 : 2 ); }
template < typename F >
void withVar( const Operator& op, F&& f )
{
   switch ( varKind( op ) )
   {
   case 2: f( std::integral_constant< int, 2 >{} ); break;
   case 1: f( std::integral_constant< int, 1 >{} ); break;
   default: f( std::integral_constant< int, 0 >{} ); break;
   }
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
std::unique_ptr< RowTables > buildRows( Storage& s, int l, bool full, bool relative = false );

// Bytes of shared memory the reference-order SOR's face and cell wavefronts need on level l
// in T, and the most a block may take; above it the stages run the plain hyperplane kernels.
constexpr size_t kSorRefMaxSmem = 220 * 1024;
template < typename T >
size_t sorRefFaceSmem( const LevelDev& d ) { return size_t( d.nIntFace ) * sizeof( T ); }
template < typename T >
size_t sorRefCellSmem( const LevelDev& d ) { return size_t( 4 ) * d.lexCellMax * sizeof( T ); }

// Hyperplane tables of the reference-order SOR (LevelDev::lex*), built on first use: the
// cell-interior points x | y << 10 | z << 20 grouped by t = x + 2y + 3z, the face-interior
// points i | j << 16 grouped by t = i + 2j, and, where the cell wavefront's ring fits
// (FP32 sizes the check, so both precisions can use it where FP64 does), each interior
// point's earlier neighbours as positions within their hyperplanes.
void ensureLex( Storage& s, int l )
{
   LevelHost& lh = *s.lv.at( size_t( l ) );
   if ( lh.lexBuilt )
      return;
   LevelDev& d = lh.dev;
   const int N = d.N;
   require( N <= 1023, "the reference-order SOR's tables take levels up to 9" );
   for ( int m = 0; m < 7; ++m )
      require( offT( sorRefEarlier( 0, m ) ) < 0 && offT( sorRefEarlier( 1, m ) ) > 0, "offset order" );
   std::vector< std::vector< int32_t > > cellT( size_t( 3 * N + 1 ) ), faceT( size_t( 2 * N + 1 ) );
   for ( int z = 1; z <= N; ++z )
      for ( int y = 1; y + z <= N - 2; ++y )
         for ( int x = 1; x + y + z <= N - 1; ++x )
            cellT[size_t( x + 2 * y + 3 * z )].push_back( x | ( y << 10 ) | ( z << 20 ) );
   for ( int j = 1; j <= N - 2; ++j )
      for ( int i = 1; i + j <= N - 1; ++i )
         faceT[size_t( i + 2 * j )].push_back( i | ( j << 16 ) );
   auto flatten = [&]( const std::vector< std::vector< int32_t > >& byT, std::vector< int32_t >& p,
                       std::vector< int32_t >& o ) {
      o.assign( 1, 0 );
      for ( const auto& v : byT )
      {
         p.insert( p.end(), v.begin(), v.end() );
         o.push_back( int32_t( p.size() ) );
      }
   };
   std::vector< int32_t > cp, co, fp, fo;
   flatten( cellT, cp, co );
   flatten( faceT, fp, fo );
   int maxPts = 0;
   for ( const auto& v : cellT )
      maxPts = std::max( maxPts, int( v.size() ) );
   lh.lexCell.upload( cp );
   {
      std::vector< int32_t > si( cp.size() );
      for ( size_t k = 0; k < cp.size(); ++k )
         si[k] = sidx( N + 1, cp[k] & 1023, ( cp[k] >> 10 ) & 1023, cp[k] >> 20 );
      lh.lexSidx.upload( si );
      d.lexSidx = lh.lexSidx.p;
   }
   lh.lexCellOff.upload( co );
   lh.lexFace.upload( fp );
   lh.lexFaceOff.upload( fo );
   d.nLexCellT  = int( cellT.size() );
   d.nLexFaceT  = int( faceT.size() );
   d.nLexCell   = int( cp.size() );
   d.lexCellMax = maxPts;
   d.lexCell    = lh.lexCell.p;
   d.lexCellOff = lh.lexCellOff.p;
   d.lexFace    = lh.lexFace.p;
   d.lexFaceOff = lh.lexFaceOff.p;
   d.lexCellNbr = nullptr;
   d.lexOfPts   = nullptr;
   if ( !cp.empty() && sorRefCellSmem< float >( d ) <= kSorRefMaxSmem )
   {
      // position of every interior point within its hyperplane
      const size_t W = size_t( N ) + 1;
      std::vector< int32_t > posIn( W * W * W, -1 );
      for ( const auto& v : cellT )
         for ( size_t k = 0; k < v.size(); ++k )
         {
            const int32_t q = v[k];
            posIn[( size_t( q >> 20 ) * W + size_t( ( q >> 10 ) & 1023 ) ) * W + size_t( q & 1023 )] = int32_t( k );
         }
      std::vector< int16_t > nb( cp.size() * 16, int16_t( -1 ) );
      for ( size_t k = 0; k < cp.size(); ++k )
      {
         const int x = cp[k] & 1023, y = ( cp[k] >> 10 ) & 1023, z = cp[k] >> 20;
         for ( int bw = 0; bw < 2; ++bw )
            for ( int m = 0; m < 7; ++m )
            {
               const int q  = sorRefEarlier( bw, m );
               const int xq = x + offX( q ), yq = y + offY( q ), zq = z + offZ( q );
               if ( xq >= 1 && yq >= 1 && zq >= 1 && xq + yq + zq <= N - 1 )
                  nb[k * 16 + size_t( bw * 8 + m )] =
                      int16_t( posIn[( size_t( zq ) * W + size_t( yq ) ) * W + size_t( xq )] );
            }
      }
      // two blocks of int4: all points' forward entries, then all points' backward entries
      std::vector< int4 > nb4( cp.size() * 2 );
      for ( size_t k = 0; k < cp.size(); ++k )
      {
         std::memcpy( &nb4[k], &nb[k * 16], sizeof( int4 ) );
         std::memcpy( &nb4[cp.size() + k], &nb[k * 16 + 8], sizeof( int4 ) );
      }
      lh.lexCellNbr.upload( nb4 );
      d.lexCellNbr = lh.lexCellNbr.p;
      // hyperplane-list position of each entry of the point table (storage order)
      require( d.nPts == int( cp.size() ), "point tables disagree" );
      std::vector< int32_t > pts( size_t( d.nPts ) ), bx( lh.blkXYZ.n );
      HYB_CUDA( cudaMemcpy( pts.data(), d.pts, pts.size() * sizeof( int32_t ), cudaMemcpyDeviceToHost ) );
      HYB_CUDA( cudaMemcpy( bx.data(), lh.blkXYZ.p, bx.size() * sizeof( int32_t ), cudaMemcpyDeviceToHost ) );
      std::vector< int32_t > lop( pts.size() );
      for ( size_t k = 0; k < pts.size(); ++k )
      {
         const int32_t p0 = bx[size_t( pts[k] >> 8 )];
         const int x = ( p0 & 1023 ) + 4 * ( pts[k] & 255 ), y = ( p0 >> 10 ) & 1023, z = p0 >> 20;
         lop[k] = co[size_t( x + 2 * y + 3 * z )] + posIn[( size_t( z ) * W + size_t( y ) ) * W + size_t( x )];
      }
      lh.lexOfPts.upload( lop );
      d.lexOfPts = lh.lexOfPts.p;
   }
   lh.lexBuilt = true;
}

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
   L.rows = buildRows( s, l, points <= rowTableMaxPoints() );
   return L.rows.get();
}

// full row tables of level l for blending operators (their only execution path)
const RowTables* ensureBlendRows( Storage& s, int l )
{
   LevelHost& L = *s.lv[size_t( l )];
   if ( L.blendRows )
      return L.blendRows.get();
   // relative rows: a neighbour's offset from its point (at most a z-slice and a row) must fit
   // 16 signed bits, and cell * stride + position 32 signed bits
   const long W = L.dev.W;
   require( W * ( W + 1 ) / 2 + 2 * W < 32768, "the blending operator supports levels up to 7" );
   require( long( s.td.nC ) * L.dev.stride < ( 1l << 31 ), "too many cells for the blending operator at this level" );
   L.blendRows = buildRows( s, l, true, true );
   require( L.blendRows != nullptr, "row table construction failed (a DoF has more cells than its lane group)" );
   return L.blendRows.get();
}

// the row tables of level l: the surface colours' rows, and with full also every colour's
// interior rows and the rows of all DoFs; nullptr if a DoF has more embeddings than its lane
// group has lanes
std::unique_ptr< RowTables > buildRows( Storage& s, int l, bool withInterior, bool relative )
{
   LevelHost&      L = *s.lv[size_t( l )];
   const LevelDev& d = L.dev;
   auto R  = std::make_unique< RowTables >();
   R->full = withInterior;
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
      k_rows_surface<<< grid( lanes ), 256 >>>( s.td, d, bl, lanes, R->iface.p + R->ifaceOff[size_t( c )], err.p,
                                               int( relative ) );
      HYB_CHECK_LAUNCH();
   }
   if ( !R->full )
   {
      int bad = 0;
      HYB_CUDA( cudaMemcpy( &bad, err.p, sizeof( int ), cudaMemcpyDeviceToHost ) );
      if ( bad )
         return nullptr;
      return R;
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
                                                                  R->interior.p + long( s.td.nC ) * d.ptsOff[c],
                                                                  int( relative ) );
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
      k_rows_surface<<< grid( surf ), 256 >>>( s.td, d, full, surf, R->all.p, err.p, int( relative ) );
      HYB_CHECK_LAUNCH();
   }
   if ( nInt > 0 )
   {
      k_rows_interior<<< grid( nInt ), 256 >>>( s.td, d, d.pts, d.nPts, R->all.p + surf, int( relative ) );
      HYB_CHECK_LAUNCH();
   }
   int bad = 0;
   HYB_CUDA( cudaMemcpy( &bad, err.p, sizeof( int ), cudaMemcpyDeviceToHost ) );
   if ( bad )
      return nullptr;
   return R;
}

// the row table of level l if it has been built (usable inside a capture)
const RowTables* rowsIf( const Storage& s, int l ) { return s.lv[size_t( l )]->rows.get(); }

RowPass rowPassAll( const RowTables* R )
{
   return R && R->full ? RowPass{ R->all.p, R->allN, R->allB1, R->allB2, R->allB3 } : RowPass{ nullptr, 0, 0, 0, 0 };
}

// grid of a row pass over n rows (128 threads a block, at most 8 blocks per SM)
inline int rowGrid( const Storage& s, long long n )
{
   return int( std::max< long long >( 1, std::min< long long >( ( n + 127 ) / 128, (long long) s.numSMs * 8 ) ) );
}

const RowTables& blendRowsOf( const Storage& s, int l )
{
   const RowTables* R = s.lv[size_t( l )]->blendRows.get();
   require( R != nullptr && R->full, "the blending operator's row tables are missing" );
   return *R;
}

template < typename T >
void launchApply( const Operator& op, int l, const T* src, T* dst, const T* rhs, int flag, int mode, cudaStream_t stream )
{
   const Storage& s  = *op.st;
   if ( op.blend )
   {
      const RowPass    rp = rowPassAll( &blendRowsOf( s, l ) );
      const OpDev< T > od = op.dev< T >( l );
      const int        g  = rowGrid( s, rp.n );
      T*               u  = const_cast< T* >( src );
      if ( mode == kResidual )
         pdlLaunch( k_row_pass_blend< T, kRowResidual >, dim3( g ), dim3( 128 ), 0, stream, rp, od, u, rhs, dst, T( 0 ), flag );
      else if ( mode == kAdd )
         pdlLaunch( k_row_pass_blend< T, kRowApplyAdd >, dim3( g ), dim3( 128 ), 0, stream, rp, od, u, rhs, dst, T( 0 ), flag );
      else
         pdlLaunch( k_row_pass_blend< T, kRowApply >, dim3( g ), dim3( 128 ), 0, stream, rp, od, u, rhs, dst, T( 0 ), flag );
      HYB_CHECK_LAUNCH();
      return;
   }
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
         withVar( op, [&]( auto V ) {
            if ( mode == kResidual )
               HYB_ROWS( kRowResidual, decltype( V )::value );
            else
               HYB_ROWS( kRowApply, decltype( V )::value );
         } );
#undef HYB_ROWS
         HYB_CHECK_LAUNCH();
         return;
      }
#define HYB_APPLY( VAR, MODE ) pdlLaunch( k_apply< T, VAR, MODE >, dim3( nb ), dim3( 128 ), 0, stream, s.td, L.dev, od, src, dst, rhs, flag, nc )
   withVar( op, [&]( auto V ) {
      constexpr int var = decltype( V )::value;
      if ( mode == kReplace )
         HYB_APPLY( var, kReplace );
      else if ( mode == kAdd )
         HYB_APPLY( var, kAdd );
      else
         HYB_APPLY( var, kResidual );
   } );
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
   if ( op.blend )
   {
      // the same passes in the same order as below, every one through the blending rows
      const RowTables& R    = blendRowsOf( s, l );
      auto             pass = [&]( const RowPass& rp ) {
         if ( rp.n == 0 )
            return;
         pdlLaunch( k_row_pass_blend< T, kRowSor >, dim3( rowGrid( s, rp.n ) ), dim3( 128 ), 0, stream, rp, od, u,
                    rhs, (T*) nullptr, relax, flag );
         HYB_CHECK_LAUNCH();
      };
      auto surface = [&]( int c ) {
         const int* co    = &L.colourOff[4 * c];
         const long lanes = bdryLaneCount( co[1], co[2], co[3] );
         const long b1 = long( co[1] ) * 32, b2 = b1 + ( long( co[2] ) * 8 + 31 ) / 32 * 32;
         pass( RowPass{ R.iface.p + R.ifaceOff[size_t( c )], lanes, b1, b2, lanes } );
      };
      auto interiorColour = [&]( int c ) {
         const long count = long( s.td.nC ) * ( L.dev.ptsOff[c + 1] - L.dev.ptsOff[c] );
         pass( RowPass{ R.interior.p + long( s.td.nC ) * L.dev.ptsOff[c], count, 0, 0, 0 } );
      };
      if ( !backwards )
      {
         for ( int c = 0; c < s.td.m; ++c )
            surface( c );
         for ( int c = 0; c < kInteriorColours; ++c )
            interiorColour( c );
      }
      else
      {
         for ( int c = kInteriorColours - 1; c >= 0; --c )
            interiorColour( c );
         for ( int c = s.td.m - 1; c >= 0; --c )
            surface( c );
      }
      return;
   }
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
         withVar( op, [&]( auto V ) {
            pdlLaunch( k_row_pass< T, kRowSor, decltype( V )::value >, dim3( nb ), dim3( 128 ), 0, stream, rp, od, u, rhs,
                       (T*) nullptr, relax, flag );
         } );
         HYB_CHECK_LAUNCH();
         return;
      }
      const int32_t*  list = L.colourList.p + co[0];
      const BdryLists bl{ list, list + co[1], list + co[1] + co[2], co[1], co[2], co[3] };
      withVar( op, [&]( auto V ) {
         pdlLaunch( k_sor_iface< T, decltype( V )::value >, dim3( nb ), dim3( 128 ), 0, stream, s.td, L.dev, od, u, rhs,
                    relax, flag, bl );
      } );
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
         withVar( op, [&]( auto V ) {
            pdlLaunch( k_sor_interior_cells< T, decltype( V )::value >, dim3( s.td.nC ), dim3( 256 ), 0, stream, s.td,
                       L.dev, od, u, rhs, relax, o[0], o[1], o[2], o[3], o[4], bw );
         } );
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
         withVar( op, [&]( auto V ) {
            pdlLaunch( k_sor_interior< T, decltype( V )::value >, dim3( L.colourBlocks ), dim3( 128 ), 0, stream, s.td,
                       L.dev, od, u, rhs, relax, c, begin, count, L.colourBlocks );
         } );
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

// Elements of the face-coupling scratch the reference-order SOR needs on level l
inline size_t sorRefCoefElems( const Storage& s, int l ) { return size_t( s.td.nF ) * s.L( l ).dev.nIntFace * 4; }

// Everything the reference-order SOR on level l needs before a launch (and before a graph
// that holds one is captured): the hyperplane tables and the opt-in to more than 48 KB of
// dynamic shared memory for the wavefront kernels.
template < typename T >
void sorRefPrepare( Storage& s, int l )
{
   ensureLex( s, l );
   static const bool attrs = [] {
      const int mx = int( kSorRefMaxSmem );
      const cudaFuncAttribute a = cudaFuncAttributeMaxDynamicSharedMemorySize;
      HYB_CUDA( cudaFuncSetAttribute( k_sorref_cells_wave< T, 0 >, a, mx ) );
      HYB_CUDA( cudaFuncSetAttribute( k_sorref_cells_wave< T, 1 >, a, mx ) );
      HYB_CUDA( cudaFuncSetAttribute( k_sorref_faces_stage< T, 0 >, a, mx ) );
      HYB_CUDA( cudaFuncSetAttribute( k_sorref_faces_stage< T, 1 >, a, mx ) );
      HYB_CUDA( cudaFuncSetAttribute( k_sorref_cells_stage< T, 0 >, a, mx ) );
      HYB_CUDA( cudaFuncSetAttribute( k_sorref_cells_stage< T, 1 >, a, mx ) );
      return true;
   }();
   (void) attrs;
}

// Reference-order SOR: the staged lexicographic sweep of the reference's smooth_sor /
// smooth_sor_backwards (P1Operator.hpp:352-431). snap is a level-sized scratch in T that
// takes the start-of-sweep copy (and, backwards, the copy before each later stage); coef
// holds sorRefCoefElems(s, l) elements of T for the face couplings. Macro-cell interiors are Inner DoFs: they move when flag has HYB_INNER. Each stage runs
// as affine precompute + on-chip recurrence (k_sorref_*_fast, k_sorref_cells_pre/_wave)
// where its shared memory fits, else as the plain hyperplane walk (k_sorref_edges/_faces/
// _cells; also with HYB_SORREF_SIMPLE=1, and for the cells of coefficient operators).
template < typename T >
void launchSorReference( const Operator& op, int l, T* u, const T* rhs, T relax, int flag, T* snap, T* coef,
                         cudaStream_t stream, bool backwards )
{
   require( !op.blend, "the reference-order SOR takes the stencil and coefficient operators" );
   Storage& s = *op.st;
   sorRefPrepare< T >( s, l );
   const auto&      L      = s.L( l );
   const OpDev< T > od     = op.dev< T >( l );
   const size_t     bytes  = size_t( s.td.nC ) * L.dev.stride * sizeof( T );
   const int        bw     = backwards ? 1 : 0;
   static const bool simple = envLong( "HYB_SORREF_SIMPLE", 0 ) != 0;
   // the fast kernels take the direction as a template argument
   auto withBw = [&]( auto&& f ) {
      if ( backwards )
         f( std::integral_constant< int, 1 >() );
      else
         f( std::integral_constant< int, 0 >() );
   };
   auto snapshot = [&]() { HYB_CUDA( cudaMemcpyAsync( snap, u, bytes, cudaMemcpyDeviceToDevice, stream ) ); };
   auto vertices = [&]() {
      if ( s.td.nV == 0 )
         return;
      withVar( op, [&]( auto V ) {
         k_sorref_vertices< T, decltype( V )::value ><<< ( s.td.nV * 32 + 127 ) / 128, 128, 0, stream >>>(
             s.td, L.dev, od, u, snap, rhs, relax, flag );
      } );
      HYB_CHECK_LAUNCH();
   };
   auto edges = [&]() {
      if ( s.td.nE == 0 || L.dev.N < 2 )
         return;
      if ( simple )
      {
         withVar( op, [&]( auto V ) {
            k_sorref_edges< T, decltype( V )::value ><<< ( s.td.nE * 32 + 127 ) / 128, 128, 0, stream >>>(
                s.td, L.dev, od, u, snap, rhs, relax, flag, bw );
         } );
         HYB_CHECK_LAUNCH();
         return;
      }
      // a block per edge; c0 and a of its points: 2 (N - 1) values, 16 KB at level 10 in FP64
      const size_t sm = size_t( 2 ) * ( L.dev.N - 1 ) * sizeof( T );
      withVar( op, [&]( auto V ) {
         withBw( [&]( auto B ) {
            k_sorref_edges_fast< T, decltype( V )::value, decltype( B )::value >
                <<< s.td.nE, 128, sm, stream >>>( s.td, L.dev, od, u, snap, rhs, relax, flag );
         } );
      } );
      HYB_CHECK_LAUNCH();
   };
   auto faces = [&]() {
      if ( s.td.nF == 0 || L.dev.nIntFace == 0 )
         return;
      // the face's interior plus the couplings of kSorRefAhead + 1 hyperplanes of at most
      // N / 2 + 1 points
      const size_t sm =
          sorRefFaceSmem< T >( L.dev ) + size_t( kSorRefAhead + 1 ) * ( L.dev.N / 2 + 1 ) * 4 * sizeof( T );
      if ( simple || sm > kSorRefMaxSmem )
      {
         withVar( op, [&]( auto V ) {
            k_sorref_faces< T, decltype( V )::value ><<< s.td.nF, 256, 0, stream >>>( s.td, L.dev, od, u, snap, rhs,
                                                                                      relax, flag, bw );
         } );
         HYB_CHECK_LAUNCH();
         return;
      }
      const long lanes = long( s.td.nF ) * L.dev.nIntFace * 2;
      const int  nb    = int( std::min< long >( ( lanes + 255 ) / 256, long( s.numSMs ) * 8 ) );
      withVar( op, [&]( auto V ) {
         withBw( [&]( auto B ) {
            k_sorref_faces_pre< T, decltype( V )::value, decltype( B )::value >
                <<< nb, 256, 0, stream >>>( s.td, L.dev, od, u, snap, rhs, relax, flag, coef );
         } );
      } );
      HYB_CHECK_LAUNCH();
      withBw( [&]( auto B ) {
         k_sorref_faces_stage< T, decltype( B )::value ><<< s.td.nF, 128, sm, stream >>>( s.td, L.dev, u, coef, flag );
      } );
      HYB_CHECK_LAUNCH();
   };
   auto cells = [&]() {
      if ( !( flag & HYB_INNER ) || L.dev.nLexCell == 0 )
         return;
      const size_t sm = sorRefCellSmem< T >( L.dev );
      if ( !simple && varKind( op ) == 0 && L.dev.lexCellNbr && sm <= kSorRefMaxSmem )
      {
         const long total = long( s.td.nC ) * L.dev.nPts;
         const int  nb    = int( std::min< long >( ( total + 255 ) / 256, long( s.numSMs ) * 8 ) );
         withBw( [&]( auto B ) {
            k_sorref_cells_pre< T, decltype( B )::value ><<< nb, 256, 0, stream >>>( s.td, L.dev, od, u, snap, rhs,
                                                                                    relax );
         } );
         HYB_CHECK_LAUNCH();
         const size_t smStage = sorRefCellStageSmem< T >( L.dev.lexCellMax, L.dev.nLexCellT );
         withBw( [&]( auto B ) {
            if ( smStage <= kSorRefMaxSmem )
            {
               k_sorref_cells_stage< T, decltype( B )::value ><<< s.td.nC, 1024, smStage, stream >>>( L.dev, od, snap,
                                                                                                       relax );
               HYB_CHECK_LAUNCH();
               k_sorref_cells_scatter< T ><<< nb, 256, 0, stream >>>( s.td, L.dev, u, snap );
            }
            else
               k_sorref_cells_wave< T, decltype( B )::value ><<< s.td.nC, 1024, sm, stream >>>( L.dev, od, u, snap,
                                                                                                relax );
         } );
         HYB_CHECK_LAUNCH();
         return;
      }
      withVar( op, [&]( auto V ) {
         k_sorref_cells< T, decltype( V )::value >
             <<< s.td.nC, sorRefCellThreads( decltype( V )::value ), 0, stream >>>( s.td, L.dev, od, u, rhs, relax, bw );
      } );
      HYB_CHECK_LAUNCH();
   };
   snapshot();
   if ( !backwards )
   {
      vertices();
      edges();
      faces();
      cells();
   }
   else
   {
      // C -> F -> E -> V with the ghost layers (here: the snapshot) refreshed before each of
      // the last three stages
      cells();
      snapshot();
      faces();
      snapshot();
      edges();
      snapshot();
      vertices();
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
   if ( op.blend )
   {
      const RowPass rp = rowPassAll( &blendRowsOf( s, l ) );
      pdlLaunch( k_row_pass_blend< T, kRowJacobi >, dim3( rowGrid( s, rp.n ) ), dim3( 128 ), 0, stream, rp, od,
                 const_cast< T* >( src ), rhs, dst, relax, flag );
      HYB_CHECK_LAUNCH();
      return;
   }
   withVar( op, [&]( auto V ) {
      pdlLaunch( k_jacobi< T, decltype( V )::value >, dim3( nb ), dim3( 128 ), 0, stream, s.td, L.dev, od, src, dst, rhs,
                 relax, flag, nc );
   } );
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
                cudaStream_t stream, float* cvt = nullptr )
{
   const auto& L = s.L( l );
   pdlLaunch( k_dot_partial< T >, dim3( dim3( L.slabBlocks, s.td.nC ) ), dim3( 256 ), 0, stream, s.td, L.dev, a, b, flag, partial,
              cvt );
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

// ||b - A x||^2 (owned DoFs on flag) into *result without storing the residual (levels
// without full row tables), float(r) into cvt when given. Returns false, launching nothing,
// when partial has fewer slots than the launch has blocks.
template < typename T >
bool launchResidualNorm( const Operator& op, int l, const T* x, const T* b, int flag, double* partial, size_t partialSlots,
                         double* result, float* cvt, cudaStream_t stream )
{
   const Storage& s  = *op.st;
   const auto&    L  = s.L( l );
   const int      nc = L.dev.nPts > 0 ? ( op.variable ? L.ptsBlocks : L.quadBlocks ) : 0;
   const int      nb = nc + ( L.dev.nBdry > 0 ? L.bdryBlocks : 0 );
   if ( op.blend || nb < 1 || size_t( nb ) > partialSlots )
      return false;
   const OpDev< T > od = op.dev< T >( l );
   withVar( op, [&]( auto V ) {
      pdlLaunch( k_residual_norm< T, decltype( V )::value >, dim3( nb ), dim3( 128 ), 0, stream, s.td, L.dev, od, x, b,
                 flag, nc, partial, cvt );
   } );
   HYB_CHECK_LAUNCH();
   pdlLaunch( k_reduce_final, dim3( 1 ), dim3( 1024 ), 0, stream, partial, nb, result );
   HYB_CHECK_LAUNCH();
   return true;
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
   if ( op.blend )
   {
      pdlLaunch( k_cg< false, true >, dim3( 1 ), dim3( 256 ), 0, stream, s.td, s.L( l ).dev, od, x, b, cs.r->ptr< double >( l ),
                 cs.p->ptr< double >( l ), cs.ap->ptr< double >( l ), tol, maxIter, cs.status.p, rowPassAll( &blendRowsOf( s, l ) ) );
      HYB_CHECK_LAUNCH();
      return;
   }
   const RowPass         rp = rowPassAll( rowsIf( s, l ) );
   withVar( op, [&]( auto V ) {
      pdlLaunch( k_cg< decltype( V )::value >, dim3( 1 ), dim3( 256 ), 0, stream, s.td, s.L( l ).dev, od, x, b,
                 cs.r->ptr< double >( l ), cs.p->ptr< double >( l ), cs.ap->ptr< double >( l ), tol, maxIter, cs.status.p,
                 rp );
   } );
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
   if ( op.blend )
   {
      const RowPass rp = rowPassAll( &blendRowsOf( s, l ) );
      k_row_pass_blend< T, kRowInvDiag ><<< rowGrid( s, rp.n ), 128, 0, stream >>>( rp, od, const_cast< T* >( zeros ),
                                                                                   nullptr, out, T( 0 ), kAll );
      HYB_CHECK_LAUNCH();
      return;
   }
   withVar( op, [&]( auto V ) {
      k_inv_diag< T, decltype( V )::value ><<< nb, 128, 0, stream >>>( s.td, L.dev, od, zeros, out, nc );
   } );
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
