// Storage, functions and operators of the B200 P1 multigrid path: per-level tables, slab
// layout, canonical-order transfers, operator assembly.
// (part of the single translation unit hyb_capi.cu, included inside namespace hyb)

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
   std::unique_ptr< RowTables > blendRows; // full rows for blending operators (ensureBlendRows)
   DevBuf< int32_t >  seg, xyz, blk, blkXYZ, pts, ptsC, quads, rowYZ;
   DevBuf< int32_t >  lexCell, lexCellOff, lexFace, lexFaceOff; // LevelDev::lex* (ensureLex)
   DevBuf< int4 >     lexCellNbr;                                  // LevelDev::lexCellNbr
   DevBuf< int32_t >  lexOfPts, lexSidx;                           // LevelDev::lexOfPts, lexSidx
   bool               lexBuilt = false;
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
   int                                   device   = 0; // the CUDA device the storage lives on
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

   DevBuf< char > sorSnap; // start-of-sweep copy of the reference-order SOR (grow-only)
   template < typename T >
   T* snapScratch( int l )
   {
      const size_t bytes = size_t( td.nC ) * L( l ).dev.stride * sizeof( T );
      if ( sorSnap.n < bytes )
      {
         HYB_CUDA( cudaDeviceSynchronize() ); // the old buffer may still be in use by queued sweeps
         sorSnap.alloc( bytes );
      }
      return reinterpret_cast< T* >( sorSnap.p );
   }

   DevBuf< char > sorCoef; // face couplings of the reference-order SOR's C ABI calls (grow-only)
   template < typename T >
   T* sorCoefScratch( size_t n )
   {
      const size_t bytes = std::max< size_t >( n, 1 ) * sizeof( T );
      if ( sorCoef.n < bytes )
      {
         HYB_CUDA( cudaDeviceSynchronize() ); // the old buffer may still be in use by queued sweeps
         sorCoef.alloc( bytes );
      }
      return reinterpret_cast< T* >( sorCoef.p );
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
      s.device = dev;
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
   // blending operator: per-cell shell maps, the coefficient's exponent, full row tables
   bool             blend = false;
   double           alpha = 0;
   DevBuf< double > bmap;
   // per level (index l - minL)
   std::vector< std::unique_ptr< DevBuf< double > > > st64, K64;
   std::vector< std::unique_ptr< DevBuf< float > > >  st32, K32;
   std::vector< std::vector< double > >               stHost; // [nC*16*15]
   std::unique_ptr< Function >                        kap64, kap32;
   // coefficient integrated at quadrature points: per level [nC][6][stride] factors (OpDev::kq)
   std::vector< std::unique_ptr< DevBuf< double > > > kq64;
   std::vector< std::unique_ptr< DevBuf< float > > >  kq32;

   template < typename T >
   OpDev< T > dev( int l ) const
   {
      require( l >= minL && l <= maxL, "level outside the operator's level range" );
      OpDev< T > o{};
      const int  i = l - minL;
      o.stride     = st->L( l ).dev.stride;
      if ( blend )
      {
         // no stencils or element matrices: the rows integrate the blended matrices
         o.bcell  = st->cellCoords.p;
         o.bmap   = bmap.p;
         o.balpha = alpha;
         o.bN     = st->L( l ).dev.N;
         return o;
      }
      if constexpr ( std::is_same< T, double >::value )
      {
         o.st = variable ? nullptr : st64[i]->p;
         o.K  = variable ? K64[i]->p : nullptr;
         o.kap = variable ? kap64->ptr< double >( l ) : nullptr;
         o.kq  = kq64.empty() ? nullptr : kq64[i]->p;
      }
      else
      {
         o.st = variable ? nullptr : st32[i]->p;
         o.K  = variable ? K32[i]->p : nullptr;
         o.kap = variable ? kap32->ptr< float >( l ) : nullptr;
         o.kq  = kq32.empty() ? nullptr : kq32[i]->p;
      }
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

// IcosahedralShellMap of macro-cell c (src/hyteg/geometry/IcosahedralShellMap.hpp:299-492):
// vertices are inner or outer by radius (within 0.1 % of the radial extent of the outer
// one): one outer vertex = an outwards cell, three = inwards, two = skew. The first local
// vertex pair whose cross product vanishes relative to their radii (1e-14) lies on one ray;
// outwards: ref = the pair's outer vertex, inwards: its inner one; thr = the last other local
// vertex, for = the remaining one. A skew cell takes the map of the second cell of its first
// face (local order 012, 013, 023, 123) that does not hold both pair vertices. Stored as the
// ray vertex, n = (thr - ray) x (for - ray), radRay and (radRef - radRay) / ((ref - ray) . n).
bool shellMapOfCell( const Topology& tp, int c, double out[8], int depth = 0 )
{
   if ( depth > 16 )
      return false;
   const auto& t = tp.T[size_t( c )];
   auto        norm = []( const std::array< double, 3 >& a ) { return std::sqrt( a[0] * a[0] + a[1] * a[1] + a[2] * a[2] ); };
   double      rad[4], inner = 1e300, outer = 0;
   for ( int k = 0; k < 4; ++k )
   {
      rad[k] = norm( tp.V[t[k]] );
      inner  = std::min( inner, rad[k] );
      outer  = std::max( outer, rad[k] );
   }
   const double eps    = ( outer - inner ) * 0.001;
   int          nOuter = 0;
   for ( int k = 0; k < 4; ++k )
      nOuter += ( outer - rad[k] ) < eps ? 1 : 0;
   if ( nOuter < 1 || nOuter > 3 )
      return false;
   int iRef = -1, iRay = -1;
   for ( int k = 0; k < 4 && iRef < 0; ++k )
      for ( int j = k + 1; j < 4 && iRef < 0; ++j )
      {
         const auto& a  = tp.V[t[k]];
         const auto& b  = tp.V[t[j]];
         const double cr[3] = { a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0] };
         if ( std::abs( cr[0] ) / ( rad[k] * rad[j] ) <= 1e-14 && std::abs( cr[1] ) / ( rad[k] * rad[j] ) <= 1e-14 &&
              std::abs( cr[2] ) / ( rad[k] * rad[j] ) <= 1e-14 )
         {
            iRef = k;
            iRay = j;
         }
      }
   if ( iRef < 0 )
      return false;
   if ( nOuter == 2 )
   {
      static const int kFace[4][3] = { { 0, 1, 2 }, { 0, 1, 3 }, { 0, 2, 3 }, { 1, 2, 3 } };
      for ( const auto& f : kFace )
      {
         const bool hasRef = f[0] == iRef || f[1] == iRef || f[2] == iRef;
         const bool hasRay = f[0] == iRay || f[1] == iRay || f[2] == iRay;
         if ( hasRef && hasRay )
            continue;
         std::array< int, 3 > key = { t[f[0]], t[f[1]], t[f[2]] };
         std::sort( key.begin(), key.end() );
         for ( const Embedding& e : tp.fEmb[size_t( tp.faceId.at( key ) )] )
            if ( e.cell != c )
               return shellMapOfCell( tp, e.cell, out, depth + 1 );
      }
      return false;
   }
   int iThr = -1, iFor = -1;
   for ( int k = 0; k < 4; ++k )
      if ( k != iRef && k != iRay )
         iThr = k;
   for ( int k = 0; k < 4; ++k )
      if ( k != iRef && k != iRay && k != iThr )
         iFor = k;
   if ( ( nOuter == 1 && rad[iRef] < rad[iRay] ) || ( nOuter == 3 && rad[iRef] > rad[iRay] ) )
      std::swap( iRef, iRay );
   const auto &ref = tp.V[t[iRef]], &ray = tp.V[t[iRay]], &thr = tp.V[t[iThr]], &fou = tp.V[t[iFor]];
   const double b[3] = { thr[0] - ray[0], thr[1] - ray[1], thr[2] - ray[2] };
   const double d[3] = { fou[0] - ray[0], fou[1] - ray[1], fou[2] - ray[2] };
   const double n[3] = { b[1] * d[2] - b[2] * d[1], b[2] * d[0] - b[0] * d[2], b[0] * d[1] - b[1] * d[0] };
   const double volT = ( ref[0] - ray[0] ) * n[0] + ( ref[1] - ray[1] ) * n[1] + ( ref[2] - ray[2] ) * n[2];
   out[0] = ray[0];
   out[1] = ray[1];
   out[2] = ray[2];
   out[3] = n[0];
   out[4] = n[1];
   out[5] = n[2];
   out[6] = norm( ray );
   out[7] = ( norm( ref ) - out[6] ) / volT;
   return true;
}

const RowTables* ensureBlendRows( Storage& s, int l );

// P1ElementwiseBlendingDivKGradOperator (src/hyteg/elementwiseoperators/P1ElementwiseOperator.hpp:349,
// form p1_div_k_grad_blending_q3) on the cells' IcosahedralShellMaps with
// k(y) = exp( alpha (1 - |y|) ) at the mapped quadrature points (alpha = 0: the Laplacian of
// the curved shell). Every operation runs through full row tables, so the levels are
// limited to cell closures below 65536 points (level 6).
Operator* makeBlendDivKGrad( Storage* s, int minL, int maxL, double alpha )
{
   require( minL >= 0 && minL <= maxL && maxL <= s->maxLevel, "invalid level range" );
   require( std::isfinite( alpha ), "alpha must be finite" );
   auto op   = std::make_unique< Operator >();
   op->st    = s;
   op->minL  = minL;
   op->maxL  = maxL;
   op->blend = true;
   op->alpha = alpha;
   const int             nC = s->td.nC;
   std::vector< double > maps( size_t( nC ) * 8 );
   for ( int c = 0; c < nC; ++c )
      require( shellMapOfCell( s->topo, c, &maps[size_t( c ) * 8] ),
               "the mesh is not a spherical shell: a macro-cell has no shell map" );
   op->bmap.upload( maps );
   for ( int l = minL; l <= maxL; ++l )
      ensureBlendRows( *s, l );
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

// The variable-coefficient operator with the coefficient evaluated as the reference's form
// does it: the callback k at the 5 quadrature points of every micro-tet on every level
// (p1_div_k_grad_affine_q3::integrateAll, src/hyteg/forms/form_hyteg_generated/p1/
// p1_div_k_grad_affine_q3.cpp:179+, applied per level by P1ElementwiseOperator.cpp:64-221).
// k is one of the functions of CoefFn (kind 1 tanh, kind 2 random features); its nodal
// values are kept as well (for callers that read the operator's coefficient).
Operator* makeDivKGradQuadrature( Storage* s, int minL, int maxL, int kind, const double* w, const double* phase,
                                  int modes, double sigma, double radial )
{
   require( kind == 1 || kind == 2, "coefficient kind must be 1 (tanh) or 2 (random features)" );
   require( kind == 1 || ( modes > 0 && w && phase ), "random-feature parameters missing" );
   DevBuf< double > dw, dp;
   if ( kind == 2 )
   {
      dw.upload( std::vector< double >( w, w + 3 * modes ) );
      dp.upload( std::vector< double >( phase, phase + modes ) );
   }
   const CoefFn f{ kind, kind == 2 ? modes : 0, sigma, radial, dw.p, dp.p };
   std::unique_ptr< Operator > op( makeDivKGradWith( s, minL, maxL, []( int, double* ) {} ) );
   for ( int l = minL; l <= maxL; ++l )
   {
      const auto&  L = s->L( l );
      const size_t n = size_t( s->td.nC ) * 6 * L.dev.stride;
      k_fill_coefficient<<< dim3( L.slabBlocks, s->td.nC ), 256 >>>( L.dev, s->cellCoords.p, s->cellOrder.p,
                                                                      op->kap64->ptr< double >( l ), f );
      HYB_CHECK_LAUNCH();
      launchConvert< float, double >( *s, l, op->kap32->ptr< float >( l ), op->kap64->ptr< double >( l ), 0 );
      auto q64 = std::make_unique< DevBuf< double > >();
      auto q32 = std::make_unique< DevBuf< float > >();
      q64->alloc( n );
      q32->alloc( n );
      k_fill_tet_factors<<< dim3( L.slabBlocks, s->td.nC ), 256 >>>( L.dev, s->cellCoords.p, s->cellOrder.p, q64->p, f );
      HYB_CHECK_LAUNCH();
      pdlLaunch( k_convert< float, double >, dim3( unsigned( ( n + 255 ) / 256 ) ), dim3( 256 ), 0, 0, L.dev, q32->p,
                 q64->p, 6 * s->td.nC );
      HYB_CHECK_LAUNCH();
      op->kq64.push_back( std::move( q64 ) );
      op->kq32.push_back( std::move( q32 ) );
   }
   HYB_CUDA( cudaDeviceSynchronize() );
   return op.release();
}

// The quadrature-point operator with a host callback: for every micro-tet (type t, vertex 0
// at closure point (x, y, z)) of every cell and level, k at the 5 quadrature points of
// p1_div_k_grad_affine_q3's rule (centroid, weight -2/15; barycentric (1/2, 1/6, 1/6, 1/6),
// weight 3/40), the factor 24 sum_q w_q k(x_q) at slab position (cell * 6 + t) * stride +
// sidx(x, y, z); micro-vertex coordinates v0 + (v_j - v0) i_j / N
// (vertexdof::macrocell::coordinateFromIndex, VertexDoFMacroCell.hpp:68-75). The nodal values
// of the same callback are kept as well.
void dofCoords( const Topology& tp, int l, std::vector< double >& out );

Operator* makeDivKGradCallbackQuadrature( Storage* s, int minL, int maxL, double ( *kfun )( const double*, void* ),
                                          void* ctx )
{
   const Topology& tp = s->topo;
   std::vector< std::vector< double > > nodal;
   for ( int l = minL; l <= maxL; ++l )
   {
      std::vector< double > xyz;
      dofCoords( tp, l, xyz );
      std::vector< double > kv( xyz.size() / 3 );
      for ( size_t i = 0; i < kv.size(); ++i )
         kv[i] = kfun( &xyz[3 * i], ctx );
      nodal.push_back( std::move( kv ) );
   }
   std::unique_ptr< Operator > op( makeDivKGrad( s, minL, maxL, nodal ) );
   const int nC = s->td.nC;
   // the micro-tet of type t with vertex 0 at a point: role 0 of the incident-tet table
   int q[6][4];
   for ( int i = 0; i < 24; ++i )
   {
      const IncidentTet it = incidentTet( i );
      if ( it.k == 0 )
         for ( int j = 0; j < 4; ++j )
            q[it.t][j] = it.q[j];
   }
   for ( int l = minL; l <= maxL; ++l )
   {
      const LevelDev& d = s->L( l ).dev;
      const int       N = d.N;
      std::vector< double > f( size_t( nC ) * 6 * d.stride, 0.0 );
      for ( int c = 0; c < nC; ++c )
      {
         const auto& T = tp.T[size_t( c )];
         double      v0[3], h[3][3];
         for ( int k = 0; k < 3; ++k )
         {
            v0[k] = tp.V[size_t( T[0] )][k];
            for ( int j = 0; j < 3; ++j )
               h[j][k] = ( tp.V[size_t( T[j + 1] )][k] - v0[k] ) / N;
         }
         for ( int z = 0; z <= N; ++z )
            for ( int y = 0; y + z <= N; ++y )
               for ( int x = 0; x + y + z <= N; ++x )
                  for ( int t = 0; t < 6; ++t )
                  {
                     double X[4][3];
                     bool   inside = true;
                     for ( int j = 0; j < 4 && inside; ++j )
                     {
                        const int xx = x + offX( q[t][j] ), yy = y + offY( q[t][j] ), zz = z + offZ( q[t][j] );
                        inside       = xx >= 0 && yy >= 0 && zz >= 0 && xx + yy + zz <= N;
                        for ( int k = 0; k < 3 && inside; ++k )
                           X[j][k] = v0[k] + h[0][k] * xx + h[1][k] * yy + h[2][k] * zz;
                     }
                     if ( !inside )
                        continue;
                     double sum = 0;
                     for ( int qp = 0; qp < 5; ++qp )
                     {
                        double p[3];
                        for ( int k = 0; k < 3; ++k )
                        {
                           double acc = 0;
                           for ( int j = 0; j < 4; ++j )
                              acc += ( qp == 0 ? 0.25 : ( j == qp - 1 ? 0.5 : 1.0 / 6.0 ) ) * X[j][k];
                           p[k] = acc;
                        }
                        sum += ( qp == 0 ? -2.0 / 15.0 : 3.0 / 40.0 ) * kfun( p, ctx );
                     }
                     f[( size_t( c ) * 6 + t ) * d.stride + size_t( sidx( d.W, x, y, z ) )] = 24.0 * sum;
                  }
      }
      auto q64 = std::make_unique< DevBuf< double > >();
      q64->upload( f );
      std::vector< float > f32( f.begin(), f.end() );
      auto q32 = std::make_unique< DevBuf< float > >();
      q32->upload( f32 );
      op->kq64.push_back( std::move( q64 ) );
      op->kq32.push_back( std::move( q32 ) );
   }
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
