// sm_100a kernels of the P1 multigrid path and their launchers.
//
// Every level operation is ONE launch whose first blocks sweep macro-cell
// interiors (one warp per 32-point row segment of the tetrahedral layout, all
// 15 neighbours at closed-form index offsets) and whose remaining blocks handle
// the micro-vertices on macro-faces, -edges and -vertices (one thread per DoF,
// summing the partial rows of all adjacent cells and writing every replica).
// The work is HBM-bound integer-indexed stencil arithmetic on CUDA cores; no
// tensor-core path applies.
#pragma once


#include "hyb_device.cuh"

namespace hyb {

enum ApplyMode : int
{
   kReplace  = 0,
   kAdd      = 1,
   kResidual = 2, // dst = rhs - A src
   kResidualNorm = 3, // r = rhs - A src is not stored: its squares over the owned active DoFs
                      // accumulate into *acc, and float(r) goes to cvt when given
};

// Programmatic dependent launch: a kernel lets the next kernel of its stream be scheduled
// as soon as all its blocks run (launch_dependents), and every kernel waits for the
// previous one to complete and its memory to be visible before touching any data (wait).
// Launches with cudaLaunchAttributeProgrammaticStreamSerialization thus overlap the launch
// latency of a kernel with the tail of its predecessor; without the attribute both
// instructions do nothing.
#define HYB_PDL_PROLOGUE() asm volatile( "griddepcontrol.launch_dependents;\n\tgriddepcontrol.wait;" ::: "memory" )

constexpr int kCellWarps  = 4; // warps (row segments) per cell block
constexpr int kBdryThreads = 128;

// ---------------------------------------------------------------------------
// Boundary-DoF enumeration: [vertices | edge interiors | face interiors]
// ---------------------------------------------------------------------------
struct BdryPoint
{
   int kind, prim, i, j;
};

__device__ __forceinline__ BdryPoint decodeBdry( const TopoDev& tp, const LevelDev& lv, int t )
{
   BdryPoint p{ 0, 0, 0, 0 };
   if ( t < tp.nV )
   {
      p.kind = 0;
      p.prim = t;
      return p;
   }
   t -= tp.nV;
   const int ne = tp.nE * ( lv.N - 1 );
   if ( t < ne )
   {
      p.kind = 1;
      p.prim = t / ( lv.N - 1 );
      p.i    = t % ( lv.N - 1 ) + 1;
      return p;
   }
   t -= ne;
   p.kind = 2;
   p.prim = t / lv.nIntFace;
   const int q  = t % lv.nIntFace;
   const int rr = lv.nIntFace - 1 - q; // index counted from the short rows
   int       k  = int( ( sqrtf( 8.0f * float( rr ) + 1.0f ) - 1.0f ) * 0.5f );
   while ( ( k + 1 ) * ( k + 2 ) / 2 <= rr )
      ++k;
   while ( k * ( k + 1 ) / 2 > rr )
      --k;
   p.i = ( k + 1 ) * ( k + 2 ) / 2 - 1 - rr + 1;
   p.j = lv.N - 2 - k;
   return p;
}

__device__ __forceinline__ int numEmb( const TopoDev& tp, int kind, int prim )
{
   if ( kind == 2 )
      return tp.fEmb[2 * prim + 1] >= 0 ? 2 : 1;
   if ( kind == 1 )
      return tp.eEmbOff[prim + 1] - tp.eEmbOff[prim];
   return tp.vEmbOff[prim + 1] - tp.vEmbOff[prim];
}
__device__ __forceinline__ int32_t embAt( const TopoDev& tp, int kind, int prim, int e )
{
   if ( kind == 2 )
      return tp.fEmb[2 * prim + e];
   if ( kind == 1 )
      return tp.eEmb[tp.eEmbOff[prim] + e];
   return tp.vEmb[tp.vEmbOff[prim] + e];
}
__device__ __forceinline__ uint8_t primBc( const TopoDev& tp, int kind, int prim )
{
   return kind == 2 ? tp.fBc[prim] : kind == 1 ? tp.eBc[prim] : tp.vBc[prim];
}

// Full row (sum of partial rows over adjacent cells) of a boundary DoF.
template < typename T, int VAR >
__device__ __forceinline__ void bdryRow( const TopoDev& tp, const LevelDev& lv, const OpDev< T >& op, const T* u,
                                         const BdryPoint& p, T& diag, T& off )
{
   const int ne = numEmb( tp, p.kind, p.prim );
   for ( int e = 0; e < ne; ++e )
   {
      int c, x, y, z;
      embeddingCoords( embAt( tp, p.kind, p.prim, e ), p.kind, lv.N, p.i, p.j, c, x, y, z );
      partialRow< T, VAR >( op, u + size_t( c ) * lv.stride, c, lv.W, x, y, z, diag, off );
   }
}

template < typename T >
__device__ __forceinline__ size_t bdryReplica( const TopoDev& tp, const LevelDev& lv, const BdryPoint& p, int e )
{
   int c, x, y, z;
   embeddingCoords( embAt( tp, p.kind, p.prim, e ), p.kind, lv.N, p.i, p.j, c, x, y, z );
   return size_t( c ) * lv.stride + sidx( lv.W, x, y, z );
}

template < typename T >
__device__ __forceinline__ void bdryWriteAll( const TopoDev& tp, const LevelDev& lv, const BdryPoint& p, T* dst, T v )
{
   const int ne = numEmb( tp, p.kind, p.prim );
   for ( int e = 0; e < ne; ++e )
      dst[bdryReplica< T >( tp, lv, p, e )] = v;
}

// ---------------------------------------------------------------------------
// Lane groups for surface DoFs. A DoF on a macro-vertex gets 32 lanes, on a
// macro-edge 8, on a macro-face 2; lane `sub` of the group handles the adjacent
// cells e = sub, sub + G, ... and the group reduces with warp shuffles. Each kind's
// lane range is padded to whole warps, so all lanes of a warp share G and every
// shuffle is executed by the full warp.
// ---------------------------------------------------------------------------
struct BdryLists
{
   const int32_t* v; // surface-DoF indices of each kind, or nullptr for the full range
   const int32_t* e;
   const int32_t* f;
   int            nv, ne, nf;
};

__device__ __forceinline__ BdryLists fullBdryLists( const TopoDev& tp, const LevelDev& lv )
{
   return BdryLists{ nullptr, nullptr, nullptr, tp.nV, tp.nE * ( lv.N - 1 ), tp.nF * lv.nIntFace };
}

__host__ __device__ __forceinline__ long bdryLaneCount( int nv, int ne, int nf )
{
   return long( nv ) * 32 + ( long( ne ) * 8 + 31 ) / 32 * 32 + ( long( nf ) * 2 + 31 ) / 32 * 32;
}

struct LaneTask
{
   int  t;      // surface-DoF index in [vertices | edge interiors | face interiors]
   int  G, sub; // group size and lane within the group
   bool valid;  // false for padding lanes
};

__device__ __forceinline__ LaneTask laneTask( const TopoDev& tp, const LevelDev& lv, const BdryLists& bl, long gt )
{
   LaneTask  tk{ 0, 32, 0, false };
   const long nvl = long( bl.nv ) * 32, nel = ( long( bl.ne ) * 8 + 31 ) / 32 * 32;
   if ( gt < nvl )
   {
      const int idx = int( gt >> 5 );
      tk            = { bl.v ? bl.v[idx] : idx, 32, int( gt & 31 ), true };
   }
   else if ( ( gt -= nvl ) < nel )
   {
      const int idx = int( gt >> 3 );
      tk.G          = 8;
      tk.sub        = int( gt & 7 );
      tk.valid      = idx < bl.ne;
      tk.t          = tk.valid ? ( bl.e ? bl.e[idx] : tp.nV + idx ) : 0;
   }
   else
   {
      gt -= nel;
      const int idx = int( gt >> 1 );
      tk.G          = 2;
      tk.sub        = int( gt & 1 );
      tk.valid      = idx < bl.nf;
      tk.t          = tk.valid ? ( bl.f ? bl.f[idx] : tp.nV + tp.nE * ( lv.N - 1 ) + idx ) : 0;
   }
   return tk;
}

template < typename T >
__device__ __forceinline__ T groupSum( T v, int G )
{
   for ( int o = G >> 1; o > 0; o >>= 1 )
      v += __shfl_xor_sync( 0xffffffffu, v, o );
   return v;
}

// Partial rows of the group's adjacent cells, summed over the group (all lanes get it).
template < typename T, int VAR >
__device__ __forceinline__ void bdryRowGroup( const TopoDev& tp, const LevelDev& lv, const OpDev< T >& op, const T* u,
                                              const BdryPoint& p, const LaneTask& tk, bool active, T& diag, T& off )
{
   diag = 0;
   off  = 0;
   if ( active )
   {
      const int ne = numEmb( tp, p.kind, p.prim );
      for ( int e = tk.sub; e < ne; e += tk.G )
      {
         int c, x, y, z;
         embeddingCoords( embAt( tp, p.kind, p.prim, e ), p.kind, lv.N, p.i, p.j, c, x, y, z );
         partialRow< T, VAR >( op, u + size_t( c ) * lv.stride, c, lv.W, x, y, z, diag, off );
      }
   }
   diag = groupSum( diag, tk.G );
   off  = groupSum( off, tk.G );
}

template < typename T >
__device__ __forceinline__ void bdryWriteGroup( const TopoDev& tp, const LevelDev& lv, const BdryPoint& p,
                                                const LaneTask& tk, T* dst, T v )
{
   const int ne = numEmb( tp, p.kind, p.prim );
   for ( int e = tk.sub; e < ne; e += tk.G )
      dst[bdryReplica< T >( tp, lv, p, e )] = v;
}

// Block index of a grid-stride loop: the block of a kernel launch, or a virtual block of a
// phase of the program kernel (which runs many level operations in one launch).
struct Blk
{
   int x, n;
};
__device__ __forceinline__ Blk launchBlk() { return Blk{ int( blockIdx.x ), int( gridDim.x ) }; }

// Warp-uniform grid-stride loop over the lanes of the surface-DoF blocks.
#define HYB_BDRY_LANES( BL )                                                                                         \
   const long total_ = bdryLaneCount( ( BL ).nv, ( BL ).ne, ( BL ).nf );                                             \
   const int  nbb_   = vb.n - nCellBlocks;                                                                           \
   for ( long gt = long( vb.x - nCellBlocks ) * blockDim.x + threadIdx.x;                                            \
         gt - ( threadIdx.x & 31 ) < total_; gt += long( nbb_ ) * blockDim.x )

// ---------------------------------------------------------------------------
// Interior stencil evaluation with all 15 neighbours inside the cell
// ---------------------------------------------------------------------------
template < typename T, int VAR >
struct InteriorOp
{
   T w[15];       // constant operator: the class-0 stencil of the cell
   T ku[36];      // variable operator: the 6 off-diagonal entries (pairs 01 02 03 12 13 23)
                  // of each of the cell's 6 micro-tet matrices, held in registers
   const T* kv;   // variable operator: nodal k slab of the cell
   const T* kqc;  // variable operator at quadrature points: the cell's 6 micro-tet factor slabs
   int      kqs;  // their stride

   // index of the unordered vertex pair (a, b), a != b, in the order 01 02 03 12 13 23
   __host__ __device__ static constexpr int pairIdx( int a, int b )
   {
      const int lo = a < b ? a : b, hi = a < b ? b : a;
      return lo == 0 ? hi - 1 : ( lo == 1 ? hi + 1 : 5 );
   }

   __device__ __forceinline__ void load( const OpDev< T >& op, int cell )
   {
      if constexpr ( !VAR )
      {
         const T* st = op.st + size_t( cell ) * 16 * 15;
#pragma unroll
         for ( int q = 0; q < 15; ++q )
            w[q] = st[q];
      }
      else
      {
         const T* K = op.K + size_t( cell ) * 96;
#pragma unroll
         for ( int t = 0; t < 6; ++t )
#pragma unroll
            for ( int a = 0; a < 4; ++a )
#pragma unroll
               for ( int b = a + 1; b < 4; ++b )
                  ku[6 * t + pairIdx( a, b )] = K[t * 16 + a * 4 + b];
         kv  = op.kap + size_t( cell ) * op.stride;
         kqc = VAR == 2 ? op.kq + size_t( cell ) * 6 * op.stride : nullptr;
         kqs = op.stride;
      }
   }

   // diag and off-diagonal sum at the interior point of table entry g whose neighbours
   // sit at no.d[q] + g
   __device__ __forceinline__ void row( const T* u, int g, const NbrOff& no, T& diag, T& off ) const
   {
      if constexpr ( !VAR )
      {
         diag = w[0];
         T s  = 0;
#pragma unroll
         for ( int q = 1; q < 15; ++q )
            s += w[q] * u[no.d[q] + g];
         off = s;
      }
      else if constexpr ( VAR == 2 )
      {
         // one quadrature factor per incident micro-tet, at its vertex 0
         T uq[15];
#pragma unroll
         for ( int q = 0; q < 15; ++q )
            uq[q] = u[no.d[q] + g];
         T d = 0, s = 0;
#pragma unroll
         for ( int i = 0; i < 24; ++i )
         {
            const IncidentTet it = incidentTet( i );
            const T ks = kqc[it.t * kqs + no.d[it.q[0]] + g];
            T       rowsum = 0, acc = 0;
#pragma unroll
            for ( int j = 0; j < 4; ++j )
               if ( j != it.k )
               {
                  const T c = ku[6 * it.t + pairIdx( it.k, j )];
                  rowsum += c;
                  acc += c * uq[it.q[j]];
               }
            d -= ks * rowsum;
            s += ks * acc;
         }
         diag = d;
         off  = s;
      }
      else
      {
         T kq[15], uq[15];
#pragma unroll
         for ( int q = 0; q < 15; ++q )
         {
            kq[q] = kv[no.d[q] + g];
            uq[q] = u[no.d[q] + g];
         }
         // element matrices of P1 stiffness have zero row sums, so the diagonal entry is
         // minus the sum of the row's off-diagonal entries (symmetric: one value per pair)
         T d = 0, s = 0;
#pragma unroll
         for ( int i = 0; i < 24; ++i )
         {
            const IncidentTet it = incidentTet( i );
            const T ks = kq[it.q[0]] + kq[it.q[1]] + kq[it.q[2]] + kq[it.q[3]];
            T       rowsum = 0, acc = 0;
#pragma unroll
            for ( int j = 0; j < 4; ++j )
               if ( j != it.k )
               {
                  const T c = ku[6 * it.t + pairIdx( it.k, j )];
                  rowsum += c;
                  acc += c * uq[it.q[j]];
               }
            d -= ks * rowsum;
            s += ks * acc;
         }
         diag = d;
         off  = s;
      }
   }
};

// ---------------------------------------------------------------------------
// Work decomposition shared by the level kernels. A launch has nCellBlocks blocks
// that loop over cell-interior row segments (item = cell * nSeg + seg, one warp per
// item, consecutive items in the same cell) and gridDim.x - nCellBlocks blocks that
// loop over surface DoFs (one thread per DoF). Both loops are grid-stride, and the
// host sizes the grid to a few blocks per SM.
// ---------------------------------------------------------------------------
#define HYB_CELL_LOOP( NSEG )                                                                                        \
   const int wpb_    = int( blockDim.x >> 5 );                                                                       \
   const int nItems_ = tp.nC * ( NSEG );                                                                             \
   for ( int it_ = vb.x * wpb_ + int( threadIdx.x >> 5 ); it_ < nItems_; it_ += nCellBlocks * wpb_ )

// The same items in block steps of S consecutive items per warp: block b's warps take the
// items [b S w, (b + 1) S w) of each step (w warps per block), so they work on neighbouring
// rows and share the rows around them in L1.
#define HYB_CELL_LOOP_STRIP( NSEG, S )                                                                               \
   const int wpb_ = int( blockDim.x >> 5 ), warp_ = int( threadIdx.x >> 5 );                                        \
   const int nItems_ = tp.nC * ( NSEG ), step_ = ( S ) * wpb_;                                                      \
   for ( int b0_ = vb.x * step_; b0_ < nItems_; b0_ += nCellBlocks * step_ )                                       \
      for ( int it_ = b0_ + warp_; it_ < b0_ + step_ && it_ < nItems_; it_ += wpb_ )

// ---------------------------------------------------------------------------
// Cell-interior loops run over the level's interior point table: a warp takes 32
// consecutive entries (consecutive storage positions, so every neighbour read is a
// contiguous run across the warp) and reads the neighbour positions of each entry's
// residue block from the block table (one broadcast per block).
// ---------------------------------------------------------------------------
__device__ __forceinline__ NbrOff blockNbr( const int32_t* __restrict__ blk, int b )
{
   const int4* p = reinterpret_cast< const int4* >( blk + 16 * size_t( b ) );
   const int4  a = __ldg( p ), c = __ldg( p + 1 ), e = __ldg( p + 2 ), f = __ldg( p + 3 );
   NbrOff      o;
   o.d[0]  = a.x;
   o.d[1]  = a.y;
   o.d[2]  = a.z;
   o.d[3]  = a.w;
   o.d[4]  = c.x;
   o.d[5]  = c.y;
   o.d[6]  = c.z;
   o.d[7]  = c.w;
   o.d[8]  = e.x;
   o.d[9]  = e.y;
   o.d[10] = e.z;
   o.d[11] = e.w;
   o.d[12] = f.x;
   o.d[13] = f.y;
   o.d[14] = f.z;
   return o;
}

// Interior points per lane and item: independent load chains that the warp keeps in
// flight together (the loops are latency bound, not bandwidth bound, at one point per lane).
// Measured on B200 at level 7, two beat one by 1.2-1.3x and beat four for FP32 (four cost
// registers and with them resident warps); three beat two by ~2 % for FP64 and lose ~5 %
// for FP32.
template < typename T, int VAR >
__host__ __device__ constexpr int interiorBatch()
{
   return VAR ? 1 : ( sizeof( T ) == 8 ? 3 : 2 );
}

// The K table entries i0 + 32 k of a point table. Entries past the end are clamped to the
// last one, so every read stays in bounds; valid[k] tells the caller not to store them.
template < int K >
struct PointBatch
{
   int    g[K];
   NbrOff no[K];
   bool   valid[K];
   __device__ __forceinline__ void load( const int32_t* __restrict__ pts, const int32_t* __restrict__ blk, int nPts,
                                         int i0 )
   {
#pragma unroll
      for ( int k = 0; k < K; ++k )
      {
         const int i     = i0 + 32 * k;
         valid[k]        = i < nPts;
         const int32_t e = __ldg( pts + ( valid[k] ? i : nPts - 1 ) );
         g[k]            = e & 255;
         no[k]           = blockNbr( blk, e >> 8 );
      }
   }
};

// ---------------------------------------------------------------------------
// Row tables of small levels. On coarse levels a pass has little
// work, and its time is the length of one lane's dependent chain: the DoF from the list,
// its embedding, class and stencil positions, then the loads. A row table stores the end
// of that chain per lane -- the cell, the partial-stencil class, the DoF's boundary flag
// and the slab positions of the 15 neighbours -- so a pass reads one row (three 16-byte
// loads), gathers, and sums the group as before.
// ---------------------------------------------------------------------------
// Rows of the constant and variable operators: base = cell * stride and pos[q] the slab
// position of neighbour q within the cell (16 bits: closures below 65536 points, level <= 6).
// Rows of the blending operator ("relative" rows): base = cell * stride + the point's own slab
// position, pos[q] the signed offset of neighbour q from the point (pos[0] = 0), which fits
// 16 bits through level 7 (a neighbour is at most a z-slice and a row away), and xyz the
// point's logical coordinates, which the on-the-fly integration needs.
struct SlabRow
{
   int32_t  base;    // see above; -1: no row (padding lane)
   int32_t  wsel;    // (cell * 16 + class) * 15: the partial stencil of the row
   uint16_t valid;   // neighbour mask of the class
   uint8_t  bc;      // boundary flag of the DoF
   uint8_t  pad0;
   uint16_t pos[15]; // neighbour positions (absolute in the cell, or relative to the point)
   uint16_t xyz[3];  // the point's x, y, z
};
static_assert( sizeof( SlabRow ) == 48, "three 16-byte loads per row" );

__device__ __forceinline__ SlabRow noRow()
{
   SlabRow R{};
   R.base = -1;
   return R;
}

__device__ __forceinline__ SlabRow makeRow( const LevelDev& lv, int c, int x, int y, int z, uint8_t bc, bool rel )
{
   SlabRow           R{};
   const int         mask  = classMask( lv.N, x, y, z );
   const uint32_t    valid = kValidOffsets[mask];
   const StencilRows S     = stencilRows( lv.W, y, z );
   const int         self  = S.start[offRow( 0 )] + resOff( x & 3, S.len[offRow( 0 )] ) + ( x >> 2 );
   for ( int q = 0; q < 15; ++q )
   {
      const int xq = x + offX( q ), k = offRow( q );
      const int p  = ( valid & ( 1u << q ) ) ? S.start[k] + resOff( xq & 3, S.len[k] ) + ( xq >> 2 ) : self;
      R.pos[q]     = uint16_t( rel ? p - self : p );
   }
   R.base   = c * lv.stride + ( rel ? self : 0 );
   R.wsel   = ( c * 16 + mask ) * 15;
   R.valid  = uint16_t( valid );
   R.bc     = bc;
   R.xyz[0] = uint16_t( x );
   R.xyz[1] = uint16_t( y );
   R.xyz[2] = uint16_t( z );
   return R;
}

// one row per lane of the surface lists bl, in the lane order of HYB_BDRY_LANES; *err is
// set when a lane's DoF has more embeddings than its group has lanes
__global__ void k_rows_surface( TopoDev tp, LevelDev lv, BdryLists bl, long n, SlabRow* out, int* err, int rel )
{
   for ( long gt = long( blockIdx.x ) * blockDim.x + threadIdx.x; gt < n; gt += long( gridDim.x ) * blockDim.x )
   {
      SlabRow        R  = noRow();
      const LaneTask tk = laneTask( tp, lv, bl, gt );
      if ( tk.valid )
      {
         const BdryPoint p  = decodeBdry( tp, lv, tk.t );
         const int       ne = numEmb( tp, p.kind, p.prim );
         if ( tk.sub + tk.G < ne )
            atomicExch( err, 1 );
         if ( tk.sub < ne )
         {
            int c, x, y, z;
            embeddingCoords( embAt( tp, p.kind, p.prim, tk.sub ), p.kind, lv.N, p.i, p.j, c, x, y, z );
            R = makeRow( lv, c, x, y, z, primBc( tp, p.kind, p.prim ), rel != 0 );
         }
      }
      out[gt] = R;
   }
}

// one row per (cell, entry) of an interior point list, cell-major; interior points are Inner
__global__ void k_rows_interior( TopoDev tp, LevelDev lv, const int32_t* list, int nList, SlabRow* out, int rel )
{
   const long n = long( tp.nC ) * nList;
   for ( long t = long( blockIdx.x ) * blockDim.x + threadIdx.x; t < n; t += long( gridDim.x ) * blockDim.x )
   {
      const int     cell = int( t / nList );
      const int32_t e    = list[t - long( cell ) * nList];
      const int     g    = e & 255;
      const NbrOff  no   = blockNbr( lv.blk, e >> 8 );
      const int32_t p0   = lv.blkXYZ[e >> 8]; // x | y << 10 | z << 20 of the block's g = 0 point
      const int     self = no.d[0] + g;
      SlabRow       R{};
      R.base  = cell * lv.stride + ( rel ? self : 0 );
      R.wsel  = cell * 16 * 15;
      R.valid = 0x7fff;
      R.bc    = 1; // Inner
      for ( int q = 0; q < 15; ++q )
         R.pos[q] = uint16_t( rel ? no.d[q] - no.d[0] : no.d[q] + g );
      R.xyz[0] = uint16_t( ( p0 & 1023 ) + 4 * g );
      R.xyz[1] = uint16_t( ( p0 >> 10 ) & 1023 );
      R.xyz[2] = uint16_t( p0 >> 20 );
      out[t] = R;
   }
}

// ---------------------------------------------------------------------------
// Blending operator (P1ElementwiseBlendingDivKGradOperator: p1_div_k_grad_blending_q3 on the
// IcosahedralShellMap, src/hyteg/forms/form_hyteg_generated/p1/p1_div_k_grad_blending_q3.cpp:412+,
// src/hyteg/geometry/IcosahedralShellMap.hpp:99-223). The element matrix of a micro-tet
// depends on its position, so a row integrates the matrices of its incident micro-tets on
// the fly:
//   A_kj = sum_q w_q k(F(xi_q)) |det J| |det DF(xi_q)| (G_q g_k) . (G_q g_j),  G_q = (DF J)^-T,
// with the 5-point degree-3 rule (centroid: -2/15; barycentric (1/2,1/6,1/6,1/6): 3/40).
// The shell map F(x) = x R(x)/|x|, R = radRay + s (x - ray) . n, has the rank-one Jacobian
// DF = a I + u v^T (a = R/|x|, u = x/|x|, v = s n - R x/|x|^2), so det DF = a^2 (a + v.u) and
// DF^-T c = (c - v (u.c)/(a + v.u)) / a, with a + v.u = s (n.x)/|x|; the 1/a^2 of the
// gradient product cancels against det DF, leaving the weight w_q k_q |det J| |s n.x| / |x|.
// k(y) = exp(alpha (1 - |y|)) with |F(xi)| = R(xi).
// ---------------------------------------------------------------------------
constexpr int kBlendMaxThreads = 256; // block size bound of the blended row passes

// kv[j] = exp(alpha (1 - R(X_j)) / 12) at the tet's vertices (alpha != 0): R is affine, so
// at the quadrature points k = exp(alpha (1 - R)) is a product of integer powers of them
// (centroid: (k0 k1 k2 k3)^3; the point weighted 1/2 on vertex j: kj^6 times the others^2)
template < typename C >
__device__ __forceinline__ void blendTetRow( const double* __restrict__ m, const C P[3], const C e[3][3], C alpha,
                                             const C kv[4], C row[4] )
{
   // the row's point is vertex 0
   C kq5[5] = { C( 1 ), C( 1 ), C( 1 ), C( 1 ), C( 1 ) };
   if ( alpha != C( 0 ) )
   {
      const C P = kv[0] * kv[1] * kv[2] * kv[3], P2 = P * P;
      kq5[0] = P2 * P;
#pragma unroll
      for ( int j = 0; j < 4; ++j )
      {
         const C k2 = kv[j] * kv[j];
         kq5[j + 1] = P2 * ( k2 * k2 );
      }
   }
   // columns of J^-T (the computational gradients of vertices 1..3; vertex 0's is minus their
   // sum, so its mapped gradient is minus the sum of the others' and the row sums to zero)
   C c[4][3];
#pragma unroll
   for ( int d = 0; d < 3; ++d )
   {
      const int d1 = ( d + 1 ) % 3, d2 = ( d + 2 ) % 3;
      c[1][d] = e[1][d1] * e[2][d2] - e[1][d2] * e[2][d1];
      c[2][d] = e[2][d1] * e[0][d2] - e[2][d2] * e[0][d1];
      c[3][d] = e[0][d1] * e[1][d2] - e[0][d2] * e[1][d1];
   }
   const C detJ = e[0][0] * c[1][0] + e[0][1] * c[1][1] + e[0][2] * c[1][2];
   const C inv  = C( 1 ) / detJ;
#pragma unroll
   for ( int d = 0; d < 3; ++d )
   {
      c[1][d] *= inv;
      c[2][d] *= inv;
      c[3][d] *= inv;
   }
   const C n[3] = { C( m[3] ), C( m[4] ), C( m[5] ) }, sc = C( m[7] );
   // R(x) = R0 + s n.x
   const C R0 = C( m[6] ) - sc * ( n[0] * C( m[0] ) + n[1] * C( m[1] ) + n[2] * C( m[2] ) );
#pragma unroll
   for ( int j = 0; j < 4; ++j )
      row[j] = C( 0 );
#pragma unroll
   for ( int q = 0; q < 5; ++q )
   {
      // xi = X0 + sum_j lambda_j (X_j - X0)
      C xi[3];
#pragma unroll
      for ( int d = 0; d < 3; ++d )
      {
         C acc = P[d];
#pragma unroll
         for ( int j = 1; j < 4; ++j )
            acc += C( q == 0 ? 0.25 : ( j == q - 1 ? 0.5 : 1.0 / 6.0 ) ) * e[j - 1][d];
         xi[d] = acc;
      }
      const C r2  = xi[0] * xi[0] + xi[1] * xi[1] + xi[2] * xi[2];
      const C ir  = rsqrt( r2 );
      const C snx = sc * ( n[0] * xi[0] + n[1] * xi[1] + n[2] * xi[2] );
      const C R   = R0 + snx; // |F(xi)|
      // a + v.u = s (n.x) / |x|
      C v[3];
#pragma unroll
      for ( int d = 0; d < 3; ++d )
         v[d] = sc * n[d] - R * ir * ir * xi[d];
      const C w  = C( q == 0 ? -2.0 / 15.0 : 3.0 / 40.0 ) * kq5[q] * fabs( detJ ) * fabs( snx ) * ir;
      const C t  = C( 1 ) / snx;
      // c' = c - v (u.c) / (a + v.u) = c - v (x.c) / (s n.x) for vertices 1..3; vertex 0: minus their sum
      C g[4][3];
#pragma unroll
      for ( int j = 1; j < 4; ++j )
      {
         const C xc = ( xi[0] * c[j][0] + xi[1] * c[j][1] + xi[2] * c[j][2] ) * t;
#pragma unroll
         for ( int d = 0; d < 3; ++d )
            g[j][d] = c[j][d] - v[d] * xc;
      }
#pragma unroll
      for ( int d = 0; d < 3; ++d )
         g[0][d] = -( g[1][d] + g[2][d] + g[3][d] );
#pragma unroll
      for ( int j = 1; j < 4; ++j )
         row[j] += w * ( g[0][0] * g[j][0] + g[0][1] * g[j][1] + g[0][2] * g[j][2] );
   }
   row[0] = -( row[1] + row[2] + row[3] );
}

// diag and off-diagonal sum of the partial row of the closure point (x, y, z) of `cell`,
// whose neighbours are read at uc[pos(q)]: the blended matrices of the incident micro-tets allowed by the class (validT);
// vertex coordinates as vertexdof::macrocell::coordinateFromIndex
// (src/hyteg/p1functionspace/VertexDoFMacroCell.hpp:68-75): v0 + (v_k - v0)/N i_k. The
// integration runs in the row type: FP64 rows reproduce the reference's matrices, FP32 rows
// (the single-precision V-cycles of the mixed solver) evaluate them in FP32.
template < typename T, typename Pos >
__device__ __forceinline__ void blendRow( const OpDev< T >& op, const T* uc, int cell, int x, int y, int z, uint32_t validT,
                                          Pos&& pos, T& diag, T& off )
{
   using C          = T;
   const double* v  = op.bcell + size_t( cell ) * 12;
   const double* m  = op.bmap + size_t( cell ) * 8;
   C             h[3][3], v0[3];
#pragma unroll
   for ( int j = 0; j < 3; ++j )
#pragma unroll
      for ( int d = 0; d < 3; ++d )
         h[j][d] = C( ( v[3 * ( j + 1 ) + d] - v[d] ) / double( op.bN ) );
#pragma unroll
   for ( int d = 0; d < 3; ++d )
      v0[d] = C( v[d] );
   // the coefficient's factors at the 15 stencil points (shared memory: indexed at run time)
   __shared__ C sK[15][kBlendMaxThreads];
   const C      alpha = C( op.balpha );
   if ( alpha != C( 0 ) )
   {
      const C sc = C( m[7] ), n[3] = { C( m[3] ), C( m[4] ), C( m[5] ) };
      const C R0 = C( m[6] ) - sc * ( n[0] * C( m[0] ) + n[1] * C( m[1] ) + n[2] * C( m[2] ) );
#pragma unroll
      for ( int q = 0; q < 15; ++q )
      {
         C p[3];
#pragma unroll
         for ( int d = 0; d < 3; ++d )
            p[d] = v0[d] + h[0][d] * C( x + offX( q ) ) + h[1][d] * C( y + offY( q ) ) + h[2][d] * C( z + offZ( q ) );
         const C R             = R0 + sc * ( n[0] * p[0] + n[1] * p[1] + n[2] * p[2] );
         sK[q][threadIdx.x] = exp( alpha * ( C( 1 ) - R ) * C( 1.0 / 12.0 ) );
      }
   }
   // the row's point is vertex 0 of every incident tet (the element matrix is equivariant
   // under relabelling its vertices), so the row is row 0
   C P[3];
#pragma unroll
   for ( int d = 0; d < 3; ++d )
      P[d] = v0[d] + h[0][d] * C( x ) + h[1][d] * C( y ) + h[2][d] * C( z );
   const C k0   = alpha != C( 0 ) ? sK[0][threadIdx.x] : C( 1 );
   C       dsum = C( 0 ), osum = C( 0 );
#pragma unroll 1
   for ( int i = 0; i < 24; ++i )
   {
      if ( !( validT & ( 1u << i ) ) )
         continue;
      const IncidentOthers& it = kIncidentOthers[i];
      C                     e[3][3], kv[4] = { k0, C( 1 ), C( 1 ), C( 1 ) };
#pragma unroll
      for ( int j = 0; j < 3; ++j )
      {
         const C dx = C( it.d[j][0] ), dy = C( it.d[j][1] ), dz = C( it.d[j][2] );
#pragma unroll
         for ( int d = 0; d < 3; ++d )
            e[j][d] = h[0][d] * dx + h[1][d] * dy + h[2][d] * dz;
         if ( alpha != C( 0 ) )
            kv[j + 1] = sK[it.q[j]][threadIdx.x];
      }
      C row[4];
      blendTetRow< C >( m, P, e, alpha, kv, row );
      dsum += row[0];
#pragma unroll
      for ( int j = 1; j < 4; ++j )
         osum += row[j] * uc[pos( it.q[j - 1] )];
   }
   diag += dsum;
   off += osum;
}

// the rows of a pass: lanes [0, b1) in groups of 32, [b1, b2) of 8, [b2, b3) of 2, the rest
// single (b1, b2, b3 are multiples of 32, so a warp has one group size)
struct RowPass
{
   const SlabRow* rows;
   long long      n, b1, b2, b3;
};

enum RowMode : int
{
   kRowSor      = 0, // u = (1 - relax) u + relax (b - off) / diag
   kRowResidual = 1, // r = b - A u
   kRowApply    = 2, // r = A u
   kRowApplyAdd = 3, // r += A u
   kRowJacobi   = 4, // r = u + relax (b - A u) / diag (u the old iterate, read only)
   kRowInvDiag  = 5  // r = 1 / diag
};

// one pass over the rows, lanes start, start + step, ... (start - lane and step multiples
// of 32; the rows of one DoF are adjacent lanes of one warp). Constant operator: the
// partial stencil st[wsel + q]; variable operator: the row's positions drive the
// incident micro-tets' matrices and nodal coefficients (the variable branch of partialRow).
template < typename T, int MODE, int VAR, bool BLEND = false >
__device__ __forceinline__ void rowPassBody( const RowPass& rp, const OpDev< T >& op, T* u, const T* b, T* r, T relax,
                                             int flag, long long start, long long step )
{
   for ( long long gt = start; gt - ( threadIdx.x & 31 ) < rp.n; gt += step )
   {
      int4 A = make_int4( -1, 0, 0, 0 ), B = make_int4( 0, 0, 0, 0 ), C = make_int4( 0, 0, 0, 0 );
      if ( gt < rp.n )
      {
         const int4* p = reinterpret_cast< const int4* >( rp.rows + gt );
         A             = __ldg( p );
         B             = __ldg( p + 1 );
         C             = __ldg( p + 2 );
      }
      const bool active = A.x >= 0 && ( ( A.z >> 16 ) & flag );
      T          diag = 0, off = 0;
      if ( active )
      {
         const T*       uc    = u + A.x;
         const uint32_t valid = uint32_t( A.z ) & 0xffffu;
         // pos[q] of the row: 16-bit halves of A.w, B.xyzw, C.xyz
         const uint32_t h[8] = { uint32_t( A.w ), uint32_t( B.x ), uint32_t( B.y ), uint32_t( B.z ),
                                 uint32_t( B.w ), uint32_t( C.x ), uint32_t( C.y ), uint32_t( C.z ) };
         auto           pos  = [&]( int q ) { return int( ( q & 1 ) ? ( h[q >> 1] >> 16 ) : ( h[q >> 1] & 0xffffu ) ); };
         if constexpr ( BLEND )
         {
            // the blended row loops over its micro-tets at run time: the row's positions go
            // through shared memory (a local array indexed at run time would live in local
            // memory); blocks of at most kBlendMaxThreads threads
            __shared__ uint32_t sPos[8][kBlendMaxThreads];
#pragma unroll
            for ( int w = 0; w < 8; ++w )
               sPos[w][threadIdx.x] = h[w];
            // relative rows: signed offsets from the point (uc), its x, y, z in C.z's upper
            // and C.w's halves
            auto spos = [&]( int q ) {
               const uint32_t v = sPos[q >> 1][threadIdx.x];
               return int( int16_t( ( q & 1 ) ? ( v >> 16 ) : ( v & 0xffffu ) ) );
            };
            blendRow( op, uc, A.y / 240, int( uint32_t( C.z ) >> 16 ), int( uint32_t( C.w ) & 0xffffu ),
                      int( uint32_t( C.w ) >> 16 ), kValidTets[( A.y / 15 ) & 15], spos, diag, off );
         }
         else if constexpr ( !VAR )
         {
            const T* w = op.st + A.y;
            diag += w[0];
#pragma unroll
            for ( int q = 1; q < 15; ++q )
               if ( valid & ( 1u << q ) )
                  off += w[q] * uc[pos( q )];
         }
         else
         {
            const int      cls    = ( A.y / 15 ) & 15, cell = A.y / 240;
            const T*       kv     = op.kap + A.x;
            const T*       kqc    = VAR == 2 ? op.kq + size_t( cell ) * 6 * op.stride : nullptr;
            const T*       K      = op.K + size_t( cell ) * 96;
            const uint32_t validT = kValidTets[cls];
#pragma unroll
            for ( int i = 0; i < 24; ++i )
            {
               const IncidentTet it = incidentTet( i );
               if ( !( validT & ( 1u << i ) ) )
                  continue;
               T ks;
               if constexpr ( VAR == 2 )
                  ks = kqc[size_t( it.t ) * op.stride + pos( it.q[0] )];
               else
                  ks = kv[pos( it.q[0] )] + kv[pos( it.q[1] )] + kv[pos( it.q[2] )] + kv[pos( it.q[3] )];
               const T* Kr = K + it.t * 16 + it.k * 4;
#pragma unroll
               for ( int j = 0; j < 4; ++j )
               {
                  if ( j == it.k )
                     diag += ks * Kr[j];
                  else
                     off += ks * Kr[j] * uc[pos( it.q[j] )];
               }
            }
         }
      }
      const int G = gt < rp.b1 ? 32 : gt < rp.b2 ? 8 : gt < rp.b3 ? 2 : 1;
      diag        = groupSum( diag, G );
      off         = groupSum( off, G );
      if ( !active )
         continue;
      const size_t i = size_t( A.x ) + ( uint32_t( A.w ) & 0xffffu );
      if constexpr ( MODE == kRowSor )
         u[i] = ( T( 1 ) - relax ) * u[i] + relax * ( b[i] - off ) / diag;
      else if constexpr ( MODE == kRowResidual )
         r[i] = b[i] - ( diag * u[i] + off );
      else if constexpr ( MODE == kRowApplyAdd )
         r[i] += diag * u[i] + off;
      else if constexpr ( MODE == kRowJacobi )
         r[i] = u[i] + relax * ( b[i] - off - diag * u[i] ) / diag;
      else if constexpr ( MODE == kRowInvDiag )
         r[i] = T( 1 ) / diag;
      else
         r[i] = diag * u[i] + off;
   }
}

// a row pass as its own launch (levels between the program kernel's and the large ones)
template < typename T, int MODE, int VAR, bool BLEND = false >
__global__ void __launch_bounds__( 128 ) k_row_pass( RowPass rp, OpDev< T > op, T* u, const T* b, T* r, T relax, int flag )
{
   HYB_PDL_PROLOGUE();
   rowPassBody< T, MODE, VAR, BLEND >( rp, op, u, b, r, relax, flag, (long long) blockIdx.x * blockDim.x + threadIdx.x,
                                       (long long) gridDim.x * blockDim.x );
}

// the blended row pass (arithmetic bound; FP64: three blocks of 128 threads per SM without
// spills measured faster than four with them, FP32 fits four)
template < typename T, int MODE >
__global__ void __launch_bounds__( 128, sizeof( T ) == 8 ? 3 : 4 ) k_row_pass_blend( RowPass rp, OpDev< T > op, T* u, const T* b, T* r, T relax,
                                                              int flag )
{
   HYB_PDL_PROLOGUE();
   rowPassBody< T, MODE, false, true >( rp, op, u, b, r, relax, flag, (long long) blockIdx.x * blockDim.x + threadIdx.x,
                                        (long long) gridDim.x * blockDim.x );
}

// Constant-stencil quad: the points x = 4g + r, r = 0..3, of row (y, z). Each of the seven
// rows the stencil touches is read once for the four points: rows whose offsets have dx in
// {-1, 0} need x' = 4g-1 .. 4g+3, rows with dx in {0, +1} need 4g .. 4g+4, the centre row
// 4g-1 .. 4g+4 (36 reads for 4 points instead of 60). Reads outside the row give 0 and
// are only used for points that are not interior.
template < typename T >
__device__ __forceinline__ T rowValue( const T* u, const StencilRows& R, int k, int g, int v )
{
   const int len = R.len[k];
   const int xq  = 4 * g + v;
   return ( xq >= 0 && xq < len ) ? u[R.start[k] + resOff( v & 3, len ) + g + resCarry( v )] : T( 0 );
}

// ax[r] = (A u) at the quad's points (constant stencil w)
template < typename T >
__device__ __forceinline__ void quadApply( const T* u, const T w[15], const StencilRows& R, int g, T ax[4] )
{
   {
      T c[6];
#pragma unroll
      for ( int v = -1; v <= 4; ++v )
         c[v + 1] = rowValue( u, R, 0, g, v );
#pragma unroll
      for ( int r = 0; r < 4; ++r )
         ax[r] = w[0] * c[r + 1] + w[1] * c[r + 2] + w[2] * c[r];
   }
   // dx = 0 offset and the other offset of row k: rows 1, 3, 6 pair dx 0 with dx -1, rows
   // 2, 4, 5 pair dx 0 with dx +1
   constexpr int qa[7] = { 0, 3, 4, 5, 6, 11, 12 };
   constexpr int qb[7] = { 0, 7, 8, 9, 10, 14, 13 };
#pragma unroll
   for ( int k = 1; k < 7; ++k )
   {
      const bool minus = ( k == 1 || k == 3 || k == 6 );
      T          a[5];
#pragma unroll
      for ( int i = 0; i < 5; ++i )
         a[i] = rowValue( u, R, k, g, minus ? i - 1 : i );
#pragma unroll
      for ( int r = 0; r < 4; ++r )
      {
         if ( minus ) // a[i] holds v = i - 1: dx 0 -> a[r + 1], dx -1 -> a[r]
            ax[r] += w[qa[k]] * a[r + 1] + w[qb[k]] * a[r];
         else // a[i] holds v = i: dx 0 -> a[r], dx +1 -> a[r + 1]
            ax[r] += w[qa[k]] * a[r] + w[qb[k]] * a[r + 1];
      }
   }
}

// ---------------------------------------------------------------------------
// apply / residual (P1Operator::apply, P1Operator.hpp:196-324;
// P1ElementwiseOperator::apply, P1ElementwiseOperator.cpp:64-221)
// ---------------------------------------------------------------------------
template < typename T, int VAR, int MODE >
__device__ __forceinline__ void applyBody( Blk vb, TopoDev tp, LevelDev lv, OpDev< T > op, const T* src,
                                                  T* dst, const T* rhs, int flag,
                                                  int nCellBlocks, double* acc = nullptr, float* cvt = nullptr )
{
   if constexpr ( !VAR )
   {
      if ( vb.x < nCellBlocks )
      {
         const int nChunks = ( lv.nQuads + 31 ) >> 5;
         HYB_CELL_LOOP( nChunks )
         {
            const int cell = it_ / nChunks;
            const int i    = ( ( it_ - cell * nChunks ) << 5 ) + int( threadIdx.x & 31 );
            if ( i >= lv.nQuads )
               continue;
            const int32_t     e  = __ldg( lv.quads + i );
            const int         g  = e & 255;
            const int32_t     yz = __ldg( lv.rowYZ + ( e >> 8 ) );
            const int         y = yz & 0xffff, z = yz >> 16;
            const StencilRows R  = stencilRows( lv.W, y, z );
            InteriorOp< T, VAR > io;
            io.load( op, cell );
            const size_t co = size_t( cell ) * lv.stride;
            T            ax[4];
            quadApply( src + co, io.w, R, g, ax );
            const int len = lv.N - 1 - y - z; // interior x in [1, len]
#pragma unroll
            for ( int r = 0; r < 4; ++r )
            {
               const int x = 4 * g + r;
               if ( x < 1 || x > len )
                  continue;
               const size_t idx = co + R.start[0] + resOff( r, R.len[0] ) + g;
               if constexpr ( MODE == kReplace )
                  dst[idx] = ax[r];
               else if constexpr ( MODE == kAdd )
                  dst[idx] += ax[r];
               else if constexpr ( MODE == kResidual )
                  dst[idx] = rhs[idx] - ax[r];
               else
               {
                  const T res = rhs[idx] - ax[r];
                  *acc += double( res ) * double( res );
                  if ( cvt )
                     cvt[idx] = float( res );
               }
            }
         }
         return;
      }
   }
   else if ( vb.x < nCellBlocks )
   {
      constexpr int K       = interiorBatch< T, VAR >();
      const int     nChunks = ( lv.nPts + 32 * K - 1 ) / ( 32 * K );
      HYB_CELL_LOOP( nChunks )
      {
         const int     cell = it_ / nChunks;
         PointBatch< K > pb;
         pb.load( lv.pts, lv.blk, lv.nPts, ( it_ - cell * nChunks ) * 32 * K + int( threadIdx.x & 31 ) );
         InteriorOp< T, VAR > io;
         io.load( op, cell );
         const size_t co = size_t( cell ) * lv.stride;
         const T* su = src + co;
         T ax[K];
#pragma unroll
         for ( int k = 0; k < K; ++k )
         {
            T diag, off;
            io.row( su, pb.g[k], pb.no[k], diag, off );
            ax[k] = diag * su[pb.no[k].d[0] + pb.g[k]] + off;
         }
#pragma unroll
         for ( int k = 0; k < K; ++k )
         {
            if ( !pb.valid[k] )
               continue;
            const size_t idx = co + pb.no[k].d[0] + pb.g[k];
            if constexpr ( MODE == kReplace )
               dst[idx] = ax[k];
            else if constexpr ( MODE == kAdd )
               dst[idx] += ax[k];
            else if constexpr ( MODE == kResidual )
               dst[idx] = rhs[idx] - ax[k];
            else
            {
               const T res = rhs[idx] - ax[k];
               *acc += double( res ) * double( res );
               if ( cvt )
                  cvt[idx] = float( res );
            }
         }
      }
      return;
   }
   const BdryLists bl = fullBdryLists( tp, lv );
   HYB_BDRY_LANES( bl )
   {
      const LaneTask  tk     = laneTask( tp, lv, bl, gt );
      const BdryPoint p      = decodeBdry( tp, lv, tk.t );
      const bool      active = tk.valid && ( primBc( tp, p.kind, p.prim ) & flag );
      T               diag, off;
      bdryRowGroup< T, VAR >( tp, lv, op, src, p, tk, active, diag, off );
      if ( !active )
         continue;
      const size_t r0 = bdryReplica< T >( tp, lv, p, 0 );
      const T      ax = diag * src[r0] + off;
      T            v;
      if constexpr ( MODE == kReplace )
         v = ax;
      else if constexpr ( MODE == kAdd )
         v = dst[r0] + ax;
      else
         v = rhs[r0] - ax;
      if constexpr ( MODE == kResidualNorm )
      {
         // the first embedding's lane counts the DoF once; every replica gets float(r)
         if ( tk.sub == 0 )
            *acc += double( v ) * double( v );
         if ( cvt )
            bdryWriteGroup( tp, lv, p, tk, cvt, float( v ) );
         continue;
      }
      // every lane of the group has read dst[r0] before any replica is written
      __syncwarp( __activemask() );
      bdryWriteGroup( tp, lv, p, tk, dst, v );
   }
}

template < typename T, int VAR, int MODE >
__global__ void __launch_bounds__( 128, VAR ? 3 : 8 ) k_apply( TopoDev tp, LevelDev lv, OpDev< T > op, const T* __restrict__ src,
                                                  T* __restrict__ dst, const T* __restrict__ rhs, int flag,
                                                  int nCellBlocks )
{
   HYB_PDL_PROLOGUE();
   applyBody< T, VAR, MODE >( launchBlk(), tp, lv, op, src, dst, rhs, flag, nCellBlocks );
}

__device__ double blockSum( double v, double* red );

// ||rhs - A src||^2 over the owned active DoFs without storing the residual: one partial
// per block (summed by k_reduce_final in a fixed order); float(r) into cvt when given.
template < typename T, int VAR >
__global__ void __launch_bounds__( 128, VAR ? 3 : 8 ) k_residual_norm( TopoDev tp, LevelDev lv, OpDev< T > op,
                                                                      const T* __restrict__ src, const T* __restrict__ rhs,
                                                                      int flag, int nCellBlocks, double* __restrict__ partial,
                                                                      float* __restrict__ cvt )
{
   HYB_PDL_PROLOGUE();
   __shared__ double red[32];
   double            acc = 0;
   applyBody< T, VAR, kResidualNorm >( launchBlk(), tp, lv, op, src, nullptr, rhs, flag, nCellBlocks, &acc, cvt );
   const double s = blockSum( acc, red );
   if ( threadIdx.x == 0 )
      partial[blockIdx.x] = s;
}

// ---------------------------------------------------------------------------
// Multicolour SOR: u <- (1-w) u + w (b - sum_{o!=0} a_o u_o) / a_0 (reference update
// formula: P1Operator.hpp:1638, sor_3D_macrocell_P1.cpp:31-77). One sweep is
//   interface passes: DoFs on macro-faces/-edges/-vertices of global colour
//     sum_k label(V_k) b_k mod m, c = 0..m-1 (each pass walks a precomputed list of
//     the surface DoFs of its colour), then
//   interior passes: macro-cell interior points of local colour (x + 2y + 3z) mod 4,
//     c = 0..3 (interiors of different cells are not coupled).
// Like the reference's V -> E -> F -> C staging, interfaces are relaxed before the
// cell interiors. No two DoFs of one pass are coupled.
// ---------------------------------------------------------------------------
constexpr int kInteriorColours = 4;
// consecutive interior batches a warp takes per block step at most (measured at level 7
// on B200: 1 -> 435 us, 2 -> 428, 4 -> 413, 8 -> 422, 16 -> 476 us per FP64 sweep; on
// smaller levels long strips leave blocks idle, so the strip shrinks with the work)
constexpr int kInteriorStrip = 4;

template < typename T, int VAR >
__device__ __forceinline__ void sorIfaceBody( Blk vb, TopoDev tp, LevelDev lv, OpDev< T > op, T* u,
                                                      const T* rhs, T relax, int flag, BdryLists bl )
{
   const int nCellBlocks = 0;
   HYB_BDRY_LANES( bl )
   {
      const LaneTask  tk     = laneTask( tp, lv, bl, gt );
      const BdryPoint p      = decodeBdry( tp, lv, tk.t );
      const bool      active = tk.valid && ( primBc( tp, p.kind, p.prim ) & flag );
      T               diag, off;
      bdryRowGroup< T, VAR >( tp, lv, op, u, p, tk, active, diag, off );
      if ( !active )
         continue;
      const size_t r0 = bdryReplica< T >( tp, lv, p, 0 );
      const T      v  = ( T( 1 ) - relax ) * u[r0] + relax * ( rhs[r0] - off ) / diag;
      // all lanes of the group read u[r0] before any replica is written
      __syncwarp( __activemask() );
      bdryWriteGroup( tp, lv, p, tk, u, v );
   }
}

template < typename T, int VAR >
__global__ void __launch_bounds__( 128, VAR ? 4 : 8 ) k_sor_iface( TopoDev tp, LevelDev lv, OpDev< T > op, T* __restrict__ u,
                                                      const T* __restrict__ rhs, T relax, int flag, BdryLists bl )
{
   HYB_PDL_PROLOGUE();
   sorIfaceBody< T, VAR >( launchBlk(), tp, lv, op, u, rhs, relax, flag, bl );
}

// One interior colour over all cells: in row (y, z) the points of colour c are the
// residue block r = (c - 2y - 3z) mod 4, one contiguous run of the row; the colour's point
// table lists them in storage order. Odd colours walk the cells in reverse order, so a
// pass starts on the data the previous pass touched last (still in L2).
template < typename T, int VAR >
__device__ __forceinline__ void sorInteriorBody( Blk vb, TopoDev tp, LevelDev lv, OpDev< T > op, T* u,
                                                         const T* rhs, T relax, int colour, int begin,
                                                         int nPts, int nCellBlocks )
{
   constexpr int  K       = interiorBatch< T, VAR >();
   const int32_t* pts     = lv.ptsC + begin;
   const int      nChunks = ( nPts + 32 * K - 1 ) / ( 32 * K );
   // strips only while every warp of the grid still gets at least one strip
   const int strip = max( 1, min( kInteriorStrip, tp.nC * nChunks / ( nCellBlocks * int( blockDim.x >> 5 ) ) ) );
   HYB_CELL_LOOP_STRIP( nChunks, strip )
   {
      const int       item = ( colour & 1 ) ? nItems_ - 1 - it_ : it_;
      const int       cell = item / nChunks;
      PointBatch< K > pb;
      pb.load( pts, lv.blk, nPts, ( item - cell * nChunks ) * 32 * K + int( threadIdx.x & 31 ) );
      InteriorOp< T, VAR > io;
      io.load( op, cell );
      T*       uc = u + size_t( cell ) * lv.stride;
      const T* bc = rhs + size_t( cell ) * lv.stride;
      // constant operator: the diagonal is the cell's stencil centre, one reciprocal per batch
      // (the reference's macro-cell kernel multiplies by the inverse centre weight as well)
      const T relaxInv = VAR ? relax : relax / io.w[0];
      T v[K];
#pragma unroll
      for ( int k = 0; k < K; ++k )
      {
         T         diag, off;
         const int idx = pb.no[k].d[0] + pb.g[k];
         io.row( uc, pb.g[k], pb.no[k], diag, off );
         if constexpr ( VAR )
            v[k] = ( T( 1 ) - relax ) * uc[idx] + relax * ( bc[idx] - off ) / diag;
         else
            v[k] = ( T( 1 ) - relax ) * uc[idx] + relaxInv * ( bc[idx] - off );
      }
      // the K points of a batch have one colour, so none reads another's new value
#pragma unroll
      for ( int k = 0; k < K; ++k )
         if ( pb.valid[k] )
            uc[pb.no[k].d[0] + pb.g[k]] = v[k];
   }
}

template < typename T, int VAR >
__global__ void __launch_bounds__( 128 ) k_sor_interior( TopoDev tp, LevelDev lv, OpDev< T > op, T* __restrict__ u,
                                                         const T* __restrict__ rhs, T relax, int colour, int begin,
                                                         int nPts, int nCellBlocks )
{
   HYB_PDL_PROLOGUE();
   sorInteriorBody< T, VAR >( launchBlk(), tp, lv, op, u, rhs, relax, colour, begin, nPts, nCellBlocks );
}

// All four interior colour passes of a sweep in ONE launch for small levels: a block per
// cell runs the colours one after the other with __syncthreads() in between. Interior
// points of different cells are never coupled, so no other block's progress matters; on
// small levels, where a colour pass has little work, this saves three launches per sweep.
// backwards != 0 runs the colours 3..0 (the backward sweep of a symmetric SOR step).
template < typename T, int VAR >
__global__ void __launch_bounds__( 256 ) k_sor_interior_cells( TopoDev tp, LevelDev lv, OpDev< T > op, T* __restrict__ u,
                                                               const T* __restrict__ rhs, T relax, int o0, int o1, int o2,
                                                               int o3, int o4, int backwards )
{
   HYB_PDL_PROLOGUE();
   const int            cell = blockIdx.x;
   InteriorOp< T, VAR > io;
   io.load( op, cell );
   T*        uc       = u + size_t( cell ) * lv.stride;
   const T*  bc       = rhs + size_t( cell ) * lv.stride;
   const T   relaxInv = VAR ? relax : relax / io.w[0];
   const int off[5]   = { o0, o1, o2, o3, o4 };
#pragma unroll
   for ( int k = 0; k < kInteriorColours; ++k )
   {
      const int c = backwards ? kInteriorColours - 1 - k : k;
      for ( int i = off[c] + int( threadIdx.x ); i < off[c + 1]; i += int( blockDim.x ) )
      {
         const int32_t e  = __ldg( lv.ptsC + i );
         const int     g  = e & 255;
         const NbrOff  no = blockNbr( lv.blk, e >> 8 );
         T             diag, offd;
         io.row( uc, g, no, diag, offd );
         const int idx = no.d[0] + g;
         if constexpr ( VAR )
            uc[idx] = ( T( 1 ) - relax ) * uc[idx] + relax * ( bc[idx] - offd ) / diag;
         else
            uc[idx] = ( T( 1 ) - relax ) * uc[idx] + relaxInv * ( bc[idx] - offd );
      }
      __syncthreads();
   }
}

// ---------------------------------------------------------------------------
// Reference-order SOR (P1Operator::smooth_sor, P1Operator.hpp:352-422; smooth_sor_backwards
// :385-400): the staged lexicographic sweep V -> E -> F -> C of the reference, in which a
// macro-vertex, -edge or -face reads its own closure's current values and every other DoF as
// it was at the start of the sweep (the ghost layers filled before it), and a macro-cell
// reads its whole closure current. The stages run as kernels on the level and on `snap`, a
// copy of the level taken when the sweep starts (and again before each of the last three
// stages of a backward sweep):
//   vertices: independent given the snapshot (lane groups);
//   edges:    a warp per edge walks its points in order, a lane per adjacent cell;
//   faces:    a block per face walks the hyperplanes t = i + 2j of its points;
//   cells:    a block per cell walks the hyperplanes t = x + 2y + 3z (LevelDev::lexCell).
// The hyperplane orders equal the lexicographic order on every coupled pair, so the result
// is the reference's sweep up to the summation order of a row.
// ---------------------------------------------------------------------------

// partialRow of (x, y, z) in `cell` with neighbour q read from the cell's slab of u when
// own(b0, b1, b2, b3) holds for its barycentric micro-coordinates, else from snap's
template < typename T, int VAR, typename Own >
__device__ __forceinline__ void partialRowSel( const OpDev< T >& op, const T* u, const T* snap, int cell, int W, int x,
                                               int y, int z, Own&& own, T& diag, T& off )
{
   const int         N     = W - 1;
   const int         mask  = classMask( N, x, y, z );
   const uint32_t    valid = kValidOffsets[mask];
   const StencilRows R     = stencilRows( W, y, z );
   int               pos[15];
   bool              cur[15];
#pragma unroll
   for ( int q = 0; q < 15; ++q )
   {
      const int xq = x + offX( q ), yq = y + offY( q ), zq = z + offZ( q ), k = offRow( q );
      const bool v = ( valid & ( 1u << q ) ) != 0;
      pos[q]       = v ? R.start[k] + resOff( xq & 3, R.len[k] ) + ( xq >> 2 ) : 0;
      cur[q]       = v && own( N - xq - yq - zq, xq, yq, zq );
   }
   auto val = [&]( int q ) { return cur[q] ? u[pos[q]] : snap[pos[q]]; };
   if constexpr ( !VAR )
   {
      const T* st = op.st + ( size_t( cell ) * 16 + mask ) * 15;
      diag += st[0];
#pragma unroll
      for ( int q = 1; q < 15; ++q )
         if ( valid & ( 1u << q ) )
            off += st[q] * val( q );
   }
   else
   {
      const T*       kv     = op.kap + size_t( cell ) * op.stride;
      const T*       K      = op.K + size_t( cell ) * 96;
      const uint32_t validT = kValidTets[mask];
#pragma unroll
      for ( int i = 0; i < 24; ++i )
      {
         const IncidentTet it = incidentTet( i );
         if ( !( validT & ( 1u << i ) ) )
            continue;
         T ks;
         if constexpr ( VAR == 2 )
            ks = op.kq[( size_t( cell ) * 6 + it.t ) * op.stride + pos[it.q[0]]];
         else
            ks = kv[pos[it.q[0]]] + kv[pos[it.q[1]]] + kv[pos[it.q[2]]] + kv[pos[it.q[3]]];
         const T* Kr = K + it.t * 16 + it.k * 4;
#pragma unroll
         for ( int j = 0; j < 4; ++j )
         {
            if ( j == it.k )
               diag += ks * Kr[j];
            else
               off += ks * Kr[j] * val( it.q[j] );
         }
      }
   }
}

// vertex stage: every vertex from the snapshot (its own value is the snapshot's too)
template < typename T, int VAR >
__global__ void __launch_bounds__( 128 ) k_sorref_vertices( TopoDev tp, LevelDev lv, OpDev< T > op, T* __restrict__ u,
                                                            const T* __restrict__ snap, const T* __restrict__ rhs, T relax,
                                                            int flag )
{
   const Blk       vb          = launchBlk();
   const int       nCellBlocks = 0;
   const BdryLists bl{ nullptr, nullptr, nullptr, tp.nV, 0, 0 };
   HYB_BDRY_LANES( bl )
   {
      const LaneTask  tk     = laneTask( tp, lv, bl, gt );
      const BdryPoint p      = decodeBdry( tp, lv, tk.t );
      const bool      active = tk.valid && ( primBc( tp, p.kind, p.prim ) & flag );
      T               diag, off;
      bdryRowGroup< T, VAR >( tp, lv, op, snap, p, tk, active, diag, off );
      if ( !active )
         continue;
      const size_t r0 = bdryReplica< T >( tp, lv, p, 0 );
      bdryWriteGroup( tp, lv, p, tk, u, ( T( 1 ) - relax ) * snap[r0] + relax * ( rhs[r0] - off ) / diag );
   }
}

// edge stage: warp w of the grid takes edge w and walks its points i = 1 .. N-1 (backwards:
// N-1 .. 1); lane l takes the edge's embeddings l, l + 32, ...; lane 0 (embedding 0) reads
// the point's value and right-hand side alongside its neighbours
template < typename T, int VAR >
__global__ void __launch_bounds__( 128 ) k_sorref_edges( TopoDev tp, LevelDev lv, OpDev< T > op, T* __restrict__ u,
                                                         const T* __restrict__ snap, const T* __restrict__ rhs, T relax,
                                                         int flag, int backwards )
{
   const int e    = int( ( blockIdx.x * blockDim.x + threadIdx.x ) >> 5 );
   const int lane = int( threadIdx.x & 31 );
   if ( e >= tp.nE || lv.N < 2 || !( primBc( tp, 1, e ) & flag ) )
      return;
   const int     ne      = numEmb( tp, 1, e );
   const int32_t packed0 = lane < ne ? embAt( tp, 1, e, lane ) : 0;
   for ( int s = 0; s < lv.N - 1; ++s )
   {
      const int i    = backwards ? lv.N - 1 - s : s + 1;
      T         diag = 0, off = 0, own = 0, bb = 0;
      size_t    rep = 0;
      for ( int k = lane; k < ne; k += 32 )
      {
         const int32_t packed = k == lane ? packed0 : embAt( tp, 1, e, k );
         const int     k0 = ( packed >> 24 ) & 3, k1 = ( packed >> 26 ) & 3;
         // the edge's closure in this cell: barycentric coordinates zero off k0 and k1
         auto own_ = [&]( int b0, int b1, int b2, int b3 ) {
            const int b[4] = { b0, b1, b2, b3 };
            for ( int m = 0; m < 4; ++m )
               if ( m != k0 && m != k1 && b[m] != 0 )
                  return false;
            return true;
         };
         int c, x, y, z;
         embeddingCoords( packed, 1, lv.N, i, 0, c, x, y, z );
         const size_t r = size_t( c ) * lv.stride + sidx( lv.W, x, y, z );
         if ( k == lane )
            rep = r;
         if ( k == 0 )
         {
            own = u[r];
            bb  = rhs[r];
         }
         partialRowSel< T, VAR >( op, u + size_t( c ) * lv.stride, snap + size_t( c ) * lv.stride, c, lv.W, x, y, z, own_,
                                  diag, off );
      }
      diag = groupSum( diag, 32 );
      off  = groupSum( off, 32 );
      T v  = lane == 0 ? ( T( 1 ) - relax ) * own + relax * ( bb - off ) / diag : T( 0 );
      v    = __shfl_sync( 0xffffffffu, v, 0 );
      if ( lane < ne )
         u[rep] = v;
      for ( int k = lane + 32; k < ne; k += 32 )
         u[bdryReplica< T >( tp, lv, BdryPoint{ 1, e, i, 0 }, k )] = v;
      __syncwarp(); // the next point reads this one's replicas
   }
}

// face stage: block f takes face f and walks its hyperplanes t = i + 2j (backwards: the
// reverse); two lanes per point, one per adjacent cell; the first reads the point's value
// and right-hand side alongside its neighbours
template < typename T, int VAR >
__global__ void __launch_bounds__( 256 ) k_sorref_faces( TopoDev tp, LevelDev lv, OpDev< T > op, T* __restrict__ u,
                                                         const T* __restrict__ snap, const T* __restrict__ rhs, T relax,
                                                         int flag, int backwards )
{
   const int f = int( blockIdx.x );
   if ( !( primBc( tp, 2, f ) & flag ) )
      return;
   const int     sub    = int( threadIdx.x & 1 );
   const int     ne     = numEmb( tp, 2, f );
   const int32_t packed = sub < ne ? embAt( tp, 2, f, sub ) : 0;
   const int     k0 = ( packed >> 24 ) & 3, k1 = ( packed >> 26 ) & 3, k2 = ( packed >> 28 ) & 3;
   const int     o  = 6 - k0 - k1 - k2; // the cell-local vertex opposite the face
   auto          own_ = [&]( int b0, int b1, int b2, int b3 ) {
      const int b[4] = { b0, b1, b2, b3 };
      return b[o] == 0;
   };
   const int pairs = int( blockDim.x >> 1 );
   for ( int s = 0; s < lv.nLexFaceT; ++s )
   {
      const int t  = backwards ? lv.nLexFaceT - 1 - s : s;
      const int p0 = lv.lexFaceOff[t], p1 = lv.lexFaceOff[t + 1];
      // whole warps take the same number of rounds, so the pair sums run on full warps
      const int rounds = ( p1 - p0 + pairs - 1 ) / pairs;
      for ( int r = 0; r < rounds; ++r )
      {
         const int  k     = p0 + r * pairs + int( threadIdx.x >> 1 );
         const bool valid = k < p1;
         T          diag = 0, off = 0, own = 0, bb = 0;
         size_t     rep = 0;
         if ( valid && sub < ne )
         {
            const int32_t ij = lv.lexFace[k];
            int           c, x, y, z;
            embeddingCoords( packed, 2, lv.N, ij & 0xffff, ij >> 16, c, x, y, z );
            rep = size_t( c ) * lv.stride + sidx( lv.W, x, y, z );
            if ( sub == 0 )
            {
               own = u[rep];
               bb  = rhs[rep];
            }
            partialRowSel< T, VAR >( op, u + size_t( c ) * lv.stride, snap + size_t( c ) * lv.stride, c, lv.W, x, y, z,
                                     own_, diag, off );
         }
         diag = groupSum( diag, 2 );
         off  = groupSum( off, 2 );
         T v  = valid && sub == 0 ? ( T( 1 ) - relax ) * own + relax * ( bb - off ) / diag : T( 0 );
         v    = __shfl_sync( 0xffffffffu, v, int( threadIdx.x & 30 ) );
         if ( valid && sub < ne )
            u[rep] = v;
      }
      __syncthreads(); // the next hyperplane reads this one's values
   }
}

// cell stage: block c takes cell c's interior and walks its hyperplanes t = x + 2y + 3z
// (backwards: the reverse), reading its closure current; interior points are Inner
// (1024 threads for the stencil operator, whose rows fit 64 registers; 512 for the others)
__host__ __device__ constexpr int sorRefCellThreads( int var ) { return var == 0 ? 1024 : 512; }
template < typename T, int VAR >
__global__ void __launch_bounds__( sorRefCellThreads( VAR ) ) k_sorref_cells( TopoDev tp, LevelDev lv, OpDev< T > op,
                                                                        T* __restrict__ u, const T* __restrict__ rhs,
                                                                        T relax, int backwards )
{
   const int c  = int( blockIdx.x );
   T*        uc = u + size_t( c ) * lv.stride;
   const T*  bc = rhs + size_t( c ) * lv.stride;
   for ( int s = 0; s < lv.nLexCellT; ++s )
   {
      const int t  = backwards ? lv.nLexCellT - 1 - s : s;
      const int p0 = lv.lexCellOff[t], p1 = lv.lexCellOff[t + 1];
      for ( int k = p0 + int( threadIdx.x ); k < p1; k += int( blockDim.x ) )
      {
         const int32_t xyz = lv.lexCell[k];
         const int     x = xyz & 1023, y = ( xyz >> 10 ) & 1023, z = xyz >> 20;
         const int     i   = sidx( lv.W, x, y, z );
         const T       own = uc[i], bb = bc[i];
         T             diag = 0, off = 0;
         partialRow< T, VAR >( op, uc, c, lv.W, x, y, z, diag, off );
         uc[i] = ( T( 1 ) - relax ) * own + relax * ( bb - off ) / diag;
      }
      __syncthreads();
   }
}

// ---------------------------------------------------------------------------
// Reference-order SOR as an affine precompute and a short recurrence. Inside one stage a
// point's new value is x_p = c0_p + sum_{q in E(p)} a_pq x_q, where E(p) holds the points of
// the same primitive that the lexicographic walk updates before p and that p couples to
// (one on an edge, three in a face, seven in a cell), and c0_p collects everything else:
// its old value, its right-hand side and the neighbours read as they were when the stage
// began. c0 and a need no order, so every point computes them at once; the walk then runs
// over on-chip memory only: the edge's points in shared memory, the face's interior in
// shared memory, and for a cell a ring of the last four hyperplanes (every coupling offset
// moves t by 1 to 3). The products are those of the plain walk in another summation order.
// ---------------------------------------------------------------------------
constexpr int kFromSnap = -1, kFromU = -2; // partialRowSplit neighbour classes (else slot 0..2)

// partialRow of (x, y, z) in `cell` split by cls(b0, b1, b2, b3) of each neighbour's
// barycentric micro-coordinates: kFromSnap and kFromU add weight * value (from snap, from u)
// to pre, a slot s in 0..2 adds the weight to a[s]
template < typename T, int VAR, typename Cls >
__device__ __forceinline__ void partialRowSplit( const OpDev< T >& op, const T* u, const T* snap, int cell, int W, int x,
                                                 int y, int z, Cls&& cls, T& diag, T& pre, T ( &a )[3] )
{
   const int         N     = W - 1;
   const int         mask  = classMask( N, x, y, z );
   const uint32_t    valid = kValidOffsets[mask];
   const StencilRows R     = stencilRows( W, y, z );
   int               pos[15];
   int               cl[15];
#pragma unroll
   for ( int q = 0; q < 15; ++q )
   {
      const int  xq = x + offX( q ), yq = y + offY( q ), zq = z + offZ( q ), k = offRow( q );
      const bool v  = ( valid & ( 1u << q ) ) != 0;
      pos[q]        = v ? R.start[k] + resOff( xq & 3, R.len[k] ) + ( xq >> 2 ) : 0;
      cl[q]         = v ? cls( N - xq - yq - zq, xq, yq, zq ) : kFromSnap;
   }
   auto acc = [&]( int q, T w ) {
      const int c = cl[q];
      if ( c == 0 )
         a[0] += w;
      else if ( c == 1 )
         a[1] += w;
      else if ( c == 2 )
         a[2] += w;
      else
         pre += w * ( c == kFromU ? u[pos[q]] : snap[pos[q]] );
   };
   if constexpr ( !VAR )
   {
      const T* st = op.st + ( size_t( cell ) * 16 + mask ) * 15;
      diag += st[0];
#pragma unroll
      for ( int q = 1; q < 15; ++q )
         if ( valid & ( 1u << q ) )
            acc( q, st[q] );
   }
   else
   {
      const T*       kv     = op.kap + size_t( cell ) * op.stride;
      const T*       K      = op.K + size_t( cell ) * 96;
      const uint32_t validT = kValidTets[mask];
#pragma unroll
      for ( int i = 0; i < 24; ++i )
      {
         const IncidentTet it = incidentTet( i );
         if ( !( validT & ( 1u << i ) ) )
            continue;
         T ks;
         if constexpr ( VAR == 2 )
            ks = op.kq[( size_t( cell ) * 6 + it.t ) * op.stride + pos[it.q[0]]];
         else
            ks = kv[pos[it.q[0]]] + kv[pos[it.q[1]]] + kv[pos[it.q[2]]] + kv[pos[it.q[3]]];
         const T* Kr = K + it.t * 16 + it.k * 4;
#pragma unroll
         for ( int j = 0; j < 4; ++j )
         {
            if ( j == it.k )
               diag += ks * Kr[j];
            else
               acc( it.q[j], ks * Kr[j] );
         }
      }
   }
}

// canonical index of face-interior point (i, j): rows j = 1 .. N-2 of N-1-j points
__device__ __forceinline__ int faceInteriorIdx( int N, int i, int j )
{
   return ( j - 1 ) * ( N - 1 ) - ( ( j - 1 ) * j ) / 2 + ( i - 1 );
}
__device__ __forceinline__ bool faceInterior( int N, int i, int j ) { return i >= 1 && j >= 1 && i + j <= N - 1; }

// edge stage: block e takes edge e; shared memory holds c0 and a of the edge's N - 1
// points, a thread per point computes them, thread 0 runs the recurrence
template < typename T, int VAR, int BW >
__global__ void __launch_bounds__( 128 ) k_sorref_edges_fast( TopoDev tp, LevelDev lv, OpDev< T > op, T* __restrict__ u,
                                                              const T* __restrict__ snap, const T* __restrict__ rhs,
                                                              T relax, int flag )
{
   constexpr int backwards = BW;
   extern __shared__ __align__( 16 ) unsigned char sorRefSmem[];
   const int e  = int( blockIdx.x );
   const int n  = lv.N - 1;
   T*        c0 = reinterpret_cast< T* >( sorRefSmem );
   T*        aa = c0 + n;
   if ( n < 1 || !( primBc( tp, 1, e ) & flag ) )
      return;
   const int ne = numEmb( tp, 1, e );
   for ( int i = 1 + int( threadIdx.x ); i <= n; i += int( blockDim.x ) )
   {
      const int ie   = backwards ? i + 1 : i - 1; // the point the walk updates just before i
      T         diag = 0, pre = 0, a[3] = { 0, 0, 0 }, own = 0, bb = 0;
      for ( int k = 0; k < ne; ++k )
      {
         const int32_t packed = embAt( tp, 1, e, k );
         const int     k0 = ( packed >> 24 ) & 3, k1 = ( packed >> 26 ) & 3;
         auto          cls = [&]( int b0, int b1, int b2, int b3 ) {
            const int b[4] = { b0, b1, b2, b3 };
            for ( int m = 0; m < 4; ++m )
               if ( m != k0 && m != k1 && b[m] != 0 )
                  return kFromSnap; // off the edge's closure
            return ( b[k1] == ie && ie >= 1 && ie <= n ) ? 0 : kFromU;
         };
         int c, x, y, z;
         embeddingCoords( packed, 1, lv.N, i, 0, c, x, y, z );
         if ( k == 0 )
         {
            const size_t r = size_t( c ) * lv.stride + sidx( lv.W, x, y, z );
            own            = u[r];
            bb             = rhs[r];
         }
         partialRowSplit< T, VAR >( op, u + size_t( c ) * lv.stride, snap + size_t( c ) * lv.stride, c, lv.W, x, y, z,
                                    cls, diag, pre, a );
      }
      c0[i - 1] = ( T( 1 ) - relax ) * own + relax * ( bb - pre ) / diag;
      aa[i - 1] = -relax * a[0] / diag;
   }
   __syncthreads();
   if ( threadIdx.x == 0 )
   {
      T prev = 0; // a is 0 at the first point: the point before it is a vertex
      for ( int s = 0; s < n; ++s )
      {
         const int i = backwards ? n - s : s + 1;
         prev        = c0[i - 1] + aa[i - 1] * prev;
         c0[i - 1]   = prev;
      }
   }
   __syncthreads();
   for ( int t = int( threadIdx.x ); t < n * ne; t += int( blockDim.x ) )
   {
      const int i = t / ne + 1, k = t - ( i - 1 ) * ne;
      u[bdryReplica< T >( tp, lv, BdryPoint{ 1, e, i, 0 }, k )] = c0[i - 1];
   }
}

// face stage, first kernel: c0 and the three couplings of every face-interior point of
// every face whose flag matches, two lanes (adjacent cells) per point, grid-wide;
// coef[(f * nIntFace + idx) * 4 + {0, 1, 2, 3}] = a0, a1, a2, c0 (idx: canonical index)
template < typename T, int VAR, int BW >
__global__ void __launch_bounds__( 256 ) k_sorref_faces_pre( TopoDev tp, LevelDev lv, OpDev< T > op,
                                                             const T* __restrict__ u, const T* __restrict__ snap,
                                                             const T* __restrict__ rhs, T relax, int flag, T* __restrict__ coef )
{
   constexpr int backwards = BW;
   const int  N = lv.N, nI = lv.nIntFace;
   const long total = long( tp.nF ) * nI * 2;
   const int  sg    = backwards ? 1 : -1;
   // whole warps run the loop together (the pair sums shuffle over full warps)
   for ( long g = long( blockIdx.x ) * blockDim.x + threadIdx.x; g - ( threadIdx.x & 31 ) < total;
         g += long( gridDim.x ) * blockDim.x )
   {
      const bool valid = g < total;
      const long pt    = valid ? g >> 1 : 0;
      const int  f = int( pt / nI ), k = int( pt - long( f ) * nI ), sub = int( g & 1 );
      const bool act   = valid && ( primBc( tp, 2, f ) & flag );
      const int  ne    = numEmb( tp, 2, f );
      T          diag = 0, pre = 0, a[3] = { 0, 0, 0 }, own = 0, bb = 0;
      const int32_t ij = lv.lexFace[k];
      const int     i = ij & 0xffff, j = ij >> 16;
      if ( act && sub < ne )
      {
         const int32_t packed = embAt( tp, 2, f, sub );
         const int     k0 = ( packed >> 24 ) & 3, k1 = ( packed >> 26 ) & 3, k2 = ( packed >> 28 ) & 3;
         const int     o  = 6 - k0 - k1 - k2; // the cell-local vertex opposite the face
         auto          cls = [&]( int b0, int b1, int b2, int b3 ) {
            const int b[4] = { b0, b1, b2, b3 };
            if ( b[o] != 0 )
               return kFromSnap; // off the face's closure
            const int di = b[k1] - i, dj = b[k2] - j;
            if ( !faceInterior( N, b[k1], b[k2] ) )
               return kFromU; // the face's edges and vertices
            if ( di == sg && dj == 0 )
               return 0;
            if ( di == 0 && dj == sg )
               return 1;
            if ( di == -sg && dj == sg )
               return 2;
            return kFromU; // face points the walk reaches later
         };
         int c, x, y, z;
         embeddingCoords( packed, 2, N, i, j, c, x, y, z );
         if ( sub == 0 )
         {
            const size_t rep = size_t( c ) * lv.stride + sidx( lv.W, x, y, z );
            own              = u[rep];
            bb               = rhs[rep];
         }
         partialRowSplit< T, VAR >( op, u + size_t( c ) * lv.stride, snap + size_t( c ) * lv.stride, c, lv.W, x, y, z,
                                    cls, diag, pre, a );
      }
      diag = groupSum( diag, 2 );
      pre  = groupSum( pre, 2 );
      a[0] = groupSum( a[0], 2 );
      a[1] = groupSum( a[1], 2 );
      a[2] = groupSum( a[2], 2 );
      if ( act && sub == 0 )
      {
         T* cf   = coef + ( size_t( f ) * nI + faceInteriorIdx( N, i, j ) ) * 4;
         const T m = -relax / diag;
         cf[0]   = m * a[0];
         cf[1]   = m * a[1];
         cf[2]   = m * a[2];
         cf[3]   = ( T( 1 ) - relax ) * own + relax * ( bb - pre ) / diag;
      }
   }
}

// the k-th point of face hyperplane t = i + 2j (j ascending), or false past its end
__device__ __forceinline__ bool faceHyperplanePoint( int N, int t, int k, int& i, int& j )
{
   const int jlo = max( 1, t - N + 1 ), jhi = min( N - 2, ( t - 1 ) / 2 );
   j             = jlo + k;
   i             = t - 2 * j;
   return j <= jhi;
}

// cell stage, stencil operator: c0 of every interior point of every cell, in storage order
// (the point tables), into snap at the point's hyperplane-list position within its cell's
// slab (snap's entries are not read again before the next snapshot)
template < typename T, int BW >
__global__ void __launch_bounds__( 256 ) k_sorref_cells_pre( TopoDev tp, LevelDev lv, OpDev< T > op,
                                                             const T* __restrict__ u, T* __restrict__ snap,
                                                             const T* __restrict__ rhs, T relax )
{
   constexpr int backwards = BW;
   const long total = long( tp.nC ) * lv.nPts;
   const int  N     = lv.N;
   for ( long gi = long( blockIdx.x ) * blockDim.x + threadIdx.x; gi < total; gi += long( gridDim.x ) * blockDim.x )
   {
      const int      c   = int( gi / lv.nPts );
      const int      k   = int( gi - long( c ) * lv.nPts );
      const int32_t  e   = lv.pts[k];
      const int      b   = e >> 8, g = e & 255;
      const int32_t  p0  = lv.blkXYZ[b];
      const int      x = ( p0 & 1023 ) + 4 * g, y = ( p0 >> 10 ) & 1023, z = p0 >> 20;
      const int32_t* nb  = lv.blk + 16 * b;
      const T*       uc  = u + size_t( c ) * lv.stride;
      const T*       st  = op.st + size_t( c ) * 16 * 15; // interior points are class 0
      T              pre = 0;
#pragma unroll
      for ( int q = 1; q < 15; ++q )
      {
         const int  xq = x + offX( q ), yq = y + offY( q ), zq = z + offZ( q );
         const bool earlier  = backwards ? offT( q ) > 0 : offT( q ) < 0;
         const bool interior = xq >= 1 && yq >= 1 && zq >= 1 && xq + yq + zq <= N - 1;
         if ( !( earlier && interior ) )
            pre += st[q] * uc[nb[q] + g];
      }
      const size_t i = size_t( c ) * lv.stride + size_t( nb[0] + g );
      snap[size_t( c ) * lv.stride + size_t( lv.lexOfPts[k] )] =
          ( T( 1 ) - relax ) * u[i] + relax * ( rhs[i] - pre ) / st[0];
   }
}

// cell stage, stencil operator: block c walks cell c's hyperplanes; the new values of the
// last four hyperplanes stay in a shared ring, indexed by position within the hyperplane;
// each thread loads its next point's c0, neighbour positions and coordinates while it
// updates the current one
template < typename T, int BW >
__global__ void __launch_bounds__( 1024 ) k_sorref_cells_wave( LevelDev lv, OpDev< T > op, T* __restrict__ u,
                                                               const T* __restrict__ snap, T relax )
{
   constexpr int backwards = BW;
   extern __shared__ __align__( 16 ) unsigned char sorRefSmem[];
   T*           ring = reinterpret_cast< T* >( sorRefSmem );
   __shared__ T aq[8];
   const int    c  = int( blockIdx.x );
   const T*     st = op.st + size_t( c ) * 16 * 15;
   if ( threadIdx.x < 7 )
      aq[threadIdx.x] = -relax * st[sorRefEarlier( backwards, int( threadIdx.x ) )] / st[0];
   T*        uc = u + size_t( c ) * lv.stride;
   const T*  sc = snap + size_t( c ) * lv.stride;
   const int M = lv.lexCellMax, nT = lv.nLexCellT, bd = int( blockDim.x );
   struct Item
   {
      int  k, t, i;
      int4 nb;
      T    c0;
      bool ok;
   };
   auto fetch = [&]( int s, int r ) {
      Item it{};
      it.ok = false;
      if ( s >= nT )
         return it;
      it.t        = backwards ? nT - 1 - s : s;
      const int p0 = lv.lexCellOff[it.t], p1 = lv.lexCellOff[it.t + 1];
      it.k         = p0 + int( threadIdx.x ) + r * bd;
      if ( it.k < p1 )
      {
         const int32_t xyz = lv.lexCell[it.k];
         it.i              = sidx( lv.W, xyz & 1023, ( xyz >> 10 ) & 1023, xyz >> 20 );
         it.nb             = lv.lexCellNbr[size_t( backwards ) * lv.nLexCell + it.k];
         it.c0             = sc[it.k];
         it.k -= p0;
         it.ok = true;
      }
      return it;
   };
   auto update = [&]( const Item& it ) {
      const int16_t* p = reinterpret_cast< const int16_t* >( &it.nb );
      T              v = it.c0;
#pragma unroll
      for ( int m = 0; m < 7; ++m )
         if ( p[m] >= 0 )
            v += aq[m] * ring[( ( it.t + offT( sorRefEarlier( backwards, m ) ) ) & 3 ) * M + p[m]];
      ring[( it.t & 3 ) * M + it.k] = v;
      uc[it.i]                      = v;
   };
   __syncthreads();
   Item nxt = fetch( 0, 0 );
   for ( int s = 0; s < nT; ++s )
   {
      const Item cur = nxt;
      nxt            = fetch( s + 1, 0 );
      if ( cur.ok )
         update( cur );
      // hyperplanes longer than the block take further rounds, unprefetched
      for ( int r = 1;; ++r )
      {
         const Item more = fetch( s, r );
         if ( !more.ok )
            break;
         update( more );
      }
      __syncthreads();
   }
}

// Asynchronous global -> shared copies (cp.async, groups committed and awaited in order)
template < int B >
__device__ __forceinline__ void cpAsync( void* dst, const void* src )
{
   const unsigned d = unsigned( __cvta_generic_to_shared( dst ) );
   if constexpr ( B == 16 )
      asm volatile( "cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"( d ), "l"( src ) : "memory" );
   else
      asm volatile( "cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"( d ), "l"( src ), "n"( B ) : "memory" );
}
__device__ __forceinline__ void cpAsyncCommit() { asm volatile( "cp.async.commit_group;\n" ::: "memory" ); }
template < int N >
__device__ __forceinline__ void cpAsyncWait()
{
   asm volatile( "cp.async.wait_group %0;\n" ::"n"( N ) : "memory" );
}

// Stages in flight of the staged wavefronts: the operands of hyperplane s + ahead are copied
// while hyperplane s is updated, into one of ahead + 1 shared stages (faces: six ahead; cells:
// two, as a cell hyperplane holds up to ~N^2/8 points, 1985 at level 7)
constexpr int kSorRefAhead = 6, kSorRefCellAhead = 2;

// shared bytes of k_sorref_cells_stage on a level: ring, stages, hyperplane offsets
template < typename T >
__host__ __device__ inline size_t sorRefCellStageSmem( int M, int nT )
{
   return size_t( 4 ) * M * sizeof( T ) + size_t( kSorRefCellAhead + 1 ) * M * ( 16 + sizeof( T ) ) +
          size_t( nT + 1 ) * 4;
}

// cell stage, stencil operator, staged: as k_sorref_cells_wave, with each hyperplane's c0 and
// neighbour positions copied to shared memory kSorRefCellAhead hyperplanes ahead. The new
// values go back over c0 in snap, in hyperplane order (contiguous stores);
// k_sorref_cells_scatter then moves them to u in storage order.
template < typename T, int BW >
__global__ void __launch_bounds__( 1024 ) k_sorref_cells_stage( LevelDev lv, OpDev< T > op, T* __restrict__ snap,
                                                                T relax )
{
   constexpr int backwards = BW;
   constexpr int A = kSorRefCellAhead, S = A + 1;
   extern __shared__ __align__( 16 ) unsigned char sorRefSmem[];
   const int     M = lv.lexCellMax, nT = lv.nLexCellT, bd = int( blockDim.x ), tid = int( threadIdx.x );
   T*            ring = reinterpret_cast< T* >( sorRefSmem );
   int4*         stNb = reinterpret_cast< int4* >( sorRefSmem + size_t( 4 ) * M * sizeof( T ) );
   T*            stC0 = reinterpret_cast< T* >( stNb + size_t( S ) * M );
   int32_t*      offS = reinterpret_cast< int32_t* >( stC0 + size_t( S ) * M );
   __shared__ T  aq[8];
   const int     c  = int( blockIdx.x );
   const T*      st = op.st + size_t( c ) * 16 * 15;
   if ( tid < 7 )
      aq[tid] = -relax * st[sorRefEarlier( backwards, tid )] / st[0];
   for ( int k = tid; k <= nT; k += bd )
      offS[k] = lv.lexCellOff[k];
   T*          sc     = snap + size_t( c ) * lv.stride;
   const int4* nbBase = lv.lexCellNbr + size_t( backwards ) * lv.nLexCell;
   __syncthreads();
   auto issue = [&]( int s ) {
      if ( s < nT )
      {
         const int t  = backwards ? nT - 1 - s : s;
         const int p0 = offS[t], n = offS[t + 1] - p0, sg = ( s % S ) * M;
         for ( int k = tid; k < n; k += bd )
         {
            cpAsync< 16 >( &stNb[sg + k], &nbBase[p0 + k] );
            cpAsync< int( sizeof( T ) ) >( &stC0[sg + k], &sc[p0 + k] );
         }
      }
      cpAsyncCommit();
   };
   for ( int d = 0; d < A; ++d )
      issue( d );
   for ( int s = 0; s < nT; ++s )
   {
      cpAsyncWait< A - 1 >(); // this thread's copies of hyperplane s have landed
      __syncthreads();        // everyone's, and hyperplane s - 1's ring entries
      issue( s + A );         // into the stage hyperplane s - 1 used
      const int t = backwards ? nT - 1 - s : s;
      const int p0 = offS[t], n = offS[t + 1] - p0, sg = ( s % S ) * M;
      for ( int k = tid; k < n; k += bd )
      {
         const int4     nb = stNb[sg + k];
         const int16_t* p  = reinterpret_cast< const int16_t* >( &nb );
         T              v  = stC0[sg + k];
#pragma unroll
         for ( int m = 0; m < 7; ++m )
            if ( p[m] >= 0 )
               v += aq[m] * ring[( ( t + offT( sorRefEarlier( backwards, m ) ) ) & 3 ) * M + p[m]];
         ring[( t & 3 ) * M + k] = v;
         sc[p0 + k]              = v; // its c0 was copied to the stage before
      }
   }
   cpAsyncWait< 0 >();
}

// cell stage: the new interior values from snap (hyperplane order) to u (storage order)
template < typename T >
__global__ void __launch_bounds__( 256 ) k_sorref_cells_scatter( TopoDev tp, LevelDev lv, T* __restrict__ u,
                                                                 const T* __restrict__ snap )
{
   const long total = long( tp.nC ) * lv.nPts;
   for ( long gi = long( blockIdx.x ) * blockDim.x + threadIdx.x; gi < total; gi += long( gridDim.x ) * blockDim.x )
   {
      const int     c = int( gi / lv.nPts ), k = int( gi - long( c ) * lv.nPts );
      const int32_t e = lv.pts[k];
      u[size_t( c ) * lv.stride + size_t( lv.blk[16 * ( e >> 8 )] + ( e & 255 ) )] =
          snap[size_t( c ) * lv.stride + size_t( lv.lexOfPts[k] )];
   }
}

// face stage, second kernel: block f walks face f's hyperplanes t = i + 2j over the shared
// array X of its interior (c0, then the new values), with the couplings of each
// hyperplane's points copied to shared memory kSorRefAhead hyperplanes ahead; then it
// writes every replica
template < typename T, int BW >
__global__ void __launch_bounds__( 128 ) k_sorref_faces_stage( TopoDev tp, LevelDev lv, T* __restrict__ u,
                                                               const T* __restrict__ coef, int flag )
{
   constexpr int backwards = BW;
   constexpr int S = kSorRefAhead + 1;
   extern __shared__ __align__( 16 ) unsigned char sorRefSmem[];
   const int     f = int( blockIdx.x );
   if ( !( primBc( tp, 2, f ) & flag ) )
      return;
   const int N = lv.N, nI = lv.nIntFace, bd = int( blockDim.x ), tid = int( threadIdx.x ), nT = 2 * N + 1;
   const int P = N / 2 + 1; // most points on one hyperplane
   T*        stA = reinterpret_cast< T* >( sorRefSmem ); // [S][P][4]: a0, a1, a2, c0
   T*        X   = stA + size_t( S ) * P * 4;
   const T*  cf  = coef + size_t( f ) * nI * 4;
   for ( int k = tid; k < nI; k += bd )
      cpAsync< int( sizeof( T ) ) >( &X[k], &cf[4 * k + 3] );
   cpAsyncCommit();
   cpAsyncWait< 0 >();
   const int sg = backwards ? 1 : -1;
   auto issue = [&]( int s ) {
      if ( s < nT )
      {
         const int t = backwards ? nT - 1 - s : s;
         int       i, j;
         for ( int k = tid; faceHyperplanePoint( N, t, k, i, j ); k += bd )
         {
            const T* src = cf + 4 * size_t( faceInteriorIdx( N, i, j ) );
            T*       dst = stA + ( size_t( s % S ) * P + k ) * 4;
            if constexpr ( sizeof( T ) == 8 )
            {
               cpAsync< 16 >( dst, src );
               cpAsync< 8 >( dst + 2, src + 2 );
            }
            else
               cpAsync< 16 >( dst, src );
         }
      }
      cpAsyncCommit();
   };
   __syncthreads();
   for ( int d = 0; d < kSorRefAhead; ++d )
      issue( d );
   for ( int s = 0; s < nT; ++s )
   {
      cpAsyncWait< kSorRefAhead - 1 >();
      __syncthreads();
      issue( s + kSorRefAhead );
      const int t = backwards ? nT - 1 - s : s;
      int       i, j;
      for ( int k = tid; faceHyperplanePoint( N, t, k, i, j ); k += bd )
      {
         const T*  a   = stA + ( size_t( s % S ) * P + k ) * 4;
         const int idx = faceInteriorIdx( N, i, j );
         T         v   = X[idx];
         if ( faceInterior( N, i + sg, j ) )
            v += a[0] * X[faceInteriorIdx( N, i + sg, j )];
         if ( faceInterior( N, i, j + sg ) )
            v += a[1] * X[faceInteriorIdx( N, i, j + sg )];
         if ( faceInterior( N, i - sg, j + sg ) )
            v += a[2] * X[faceInteriorIdx( N, i - sg, j + sg )];
         X[idx] = v;
      }
   }
   cpAsyncWait< 0 >();
   __syncthreads();
   // every replica: two lanes per point, one per adjacent cell, row by row
   const int     sub    = tid & 1;
   const int     ne     = numEmb( tp, 2, f );
   const int32_t packed = sub < ne ? embAt( tp, 2, f, sub ) : 0;
   if ( sub < ne )
      for ( int j = 1; j <= N - 2; ++j )
         for ( int i = 1 + ( tid >> 1 ); i + j <= N - 1; i += bd >> 1 )
         {
            int c, x, y, z;
            embeddingCoords( packed, 2, N, i, j, c, x, y, z );
            u[size_t( c ) * lv.stride + sidx( lv.W, x, y, z )] = X[faceInteriorIdx( N, i, j )];
         }
}

// ---------------------------------------------------------------------------
// diag(A)^-1 at every closure point (all replicas; the full row's diagonal for macro-
// primitive DoFs). zeros: a zero vector of the level, read as the operand of the rows
// whose off-diagonal part is discarded. Cells' interiors on the first nCellBlocks blocks.
// ---------------------------------------------------------------------------
template < typename T, int VAR >
__global__ void __launch_bounds__( 128 ) k_inv_diag( TopoDev tp, LevelDev lv, OpDev< T > op, const T* __restrict__ zeros,
                                                     T* __restrict__ out, int nCellBlocks )
{
   const Blk vb = launchBlk();
   if ( vb.x < nCellBlocks )
   {
      const int nChunks = ( lv.nPts + 31 ) / 32;
      HYB_CELL_LOOP( nChunks )
      {
         const int       cell = it_ / nChunks;
         PointBatch< 1 > pb;
         pb.load( lv.pts, lv.blk, lv.nPts, ( it_ - cell * nChunks ) * 32 + int( threadIdx.x & 31 ) );
         InteriorOp< T, VAR > io;
         io.load( op, cell );
         T diag, off;
         io.row( zeros + size_t( cell ) * lv.stride, pb.g[0], pb.no[0], diag, off );
         if ( pb.valid[0] )
            out[size_t( cell ) * lv.stride + pb.no[0].d[0] + pb.g[0]] = T( 1 ) / diag;
      }
      return;
   }
   const BdryLists bl = fullBdryLists( tp, lv );
   HYB_BDRY_LANES( bl )
   {
      const LaneTask  tk = laneTask( tp, lv, bl, gt );
      const BdryPoint p  = decodeBdry( tp, lv, tk.t );
      T               diag, off;
      bdryRowGroup< T, VAR >( tp, lv, op, zeros, p, tk, tk.valid, diag, off );
      if ( tk.valid )
         bdryWriteGroup( tp, lv, p, tk, out, T( 1 ) / diag );
   }
}

// dst = a * src and dst *= w over a level's slabs (power iteration of the spectral radius
// estimate)
__global__ void k_scale_copy( long long n, const double* __restrict__ src, double* dst, double a )
{
   for ( long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long) gridDim.x * blockDim.x )
      dst[i] = a * src[i];
}
__global__ void k_mul( long long n, const double* __restrict__ w, double* dst )
{
   for ( long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long) gridDim.x * blockDim.x )
      dst[i] *= w[i];
}

// Chebyshev smoother update over a level's slabs: t = inv * t, x += w t (entries outside the
// smoothed DoFs hold t = 0 and stay unchanged)
template < typename T >
__global__ void __launch_bounds__( 256 ) k_cheb_update( long long n, const T* __restrict__ inv, T* __restrict__ t,
                                                        T* __restrict__ x, T w )
{
   HYB_PDL_PROLOGUE();
   for ( long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long) gridDim.x * blockDim.x )
   {
      const T v = inv[i] * t[i];
      t[i]      = v;
      x[i] += w * v;
   }
}

// ---------------------------------------------------------------------------
// Weighted Jacobi (P1Operator::smooth_jac, P1Operator.hpp:424-440):
// dst = src + relax * (rhs - A src) / diag(A)
// ---------------------------------------------------------------------------
template < typename T, int VAR >
__device__ __forceinline__ void jacobiBody( Blk vb, TopoDev tp, LevelDev lv, OpDev< T > op, const T* src,
                                                   T* dst, const T* rhs, T relax, int flag,
                                                   int nCellBlocks )
{
   if ( vb.x < nCellBlocks )
   {
      constexpr int K       = interiorBatch< T, VAR >();
      const int     nChunks = ( lv.nPts + 32 * K - 1 ) / ( 32 * K );
      HYB_CELL_LOOP( nChunks )
      {
         const int       cell = it_ / nChunks;
         PointBatch< K > pb;
         pb.load( lv.pts, lv.blk, lv.nPts, ( it_ - cell * nChunks ) * 32 * K + int( threadIdx.x & 31 ) );
         InteriorOp< T, VAR > io;
         io.load( op, cell );
         const size_t co = size_t( cell ) * lv.stride;
         const T* su = src + co;
         T v[K];
#pragma unroll
         for ( int k = 0; k < K; ++k )
         {
            T         diag, off;
            const int idx = pb.no[k].d[0] + pb.g[k];
            io.row( su, pb.g[k], pb.no[k], diag, off );
            const T s = su[idx];
            v[k]      = s + relax * ( rhs[co + idx] - off - diag * s ) / diag;
         }
#pragma unroll
         for ( int k = 0; k < K; ++k )
            if ( pb.valid[k] )
               dst[co + pb.no[k].d[0] + pb.g[k]] = v[k];
      }
      return;
   }
   const BdryLists bl = fullBdryLists( tp, lv );
   HYB_BDRY_LANES( bl )
   {
      const LaneTask  tk     = laneTask( tp, lv, bl, gt );
      const BdryPoint p      = decodeBdry( tp, lv, tk.t );
      const bool      active = tk.valid && ( primBc( tp, p.kind, p.prim ) & flag );
      T               diag, off;
      bdryRowGroup< T, VAR >( tp, lv, op, src, p, tk, active, diag, off );
      if ( !active )
         continue;
      const size_t r0 = bdryReplica< T >( tp, lv, p, 0 );
      const T      s  = src[r0];
      bdryWriteGroup( tp, lv, p, tk, dst, T( s + relax * ( rhs[r0] - off - diag * s ) / diag ) );
   }
}

template < typename T, int VAR >
__global__ void __launch_bounds__( 128 ) k_jacobi( TopoDev tp, LevelDev lv, OpDev< T > op, const T* __restrict__ src,
                                                   T* __restrict__ dst, const T* __restrict__ rhs, T relax, int flag,
                                                   int nCellBlocks )
{
   HYB_PDL_PROLOGUE();
   jacobiBody< T, VAR >( launchBlk(), tp, lv, op, src, dst, rhs, relax, flag, nCellBlocks );
}

// ---------------------------------------------------------------------------
// Linear prolongation (P1toP1LinearProlongation.cpp:194-410): a fine micro-vertex
// either coincides with a coarse one (weight 1) or bisects a coarse micro-edge
// (weights 1/2, 1/2). Computed in gather form inside any one adjacent cell.
// ---------------------------------------------------------------------------
template < typename T >
__device__ __forceinline__ T interpolateFine( const T* coarse, int Wc, int X, int Y, int Z )
{
   const int px = X & 1, py = Y & 1, pz = Z & 1;
   if ( !( px | py | pz ) )
      return coarse[sidx( Wc, X >> 1, Y >> 1, Z >> 1 )];
   int       ox = 0, oy = 0, oz = 0;
   const int pat = px | ( py << 1 ) | ( pz << 2 );
   switch ( pat )
   {
   case 1: ox = 1; break;
   case 2: oy = 1; break;
   case 4: oz = 1; break;
   case 3: ox = -1; oy = 1; break;
   case 5: ox = -1; oz = 1; break;
   case 6: oy = -1; oz = 1; break;
   default: ox = -1; oy = 1; oz = -1; break;
   }
   return T( 0.5 ) * ( coarse[sidx( Wc, ( X - ox ) >> 1, ( Y - oy ) >> 1, ( Z - oz ) >> 1 )] +
                       coarse[sidx( Wc, ( X + ox ) >> 1, ( Y + oy ) >> 1, ( Z + oz ) >> 1 )] );
}

template < typename T, bool ADD >
__device__ __forceinline__ void prolongateBody( Blk vb, TopoDev tp, LevelDev lv, int Wc, int strideC,
                                                       const T* coarse, T* fine, int flag,
                                                       int nCellBlocks )
{
   if ( vb.x < nCellBlocks )
   {
      // fine interior points from the point table: the points of one block share the
      // parity pattern (x steps by 4) and their coarse rows, whose positions the level's
      // prolongation table holds (LevelDev::pro)
      constexpr int K       = 2;
      const int     nChunks = ( lv.nPts + 32 * K - 1 ) / ( 32 * K );
      HYB_CELL_LOOP( nChunks )
      {
         const int cell = it_ / nChunks;
         const int i0   = ( it_ - cell * nChunks ) * 32 * K + int( threadIdx.x & 31 );
         T         v[K];
         size_t    fi[K];
         bool      ok[K];
#pragma unroll
         for ( int k = 0; k < K; ++k )
         {
            const int i     = i0 + 32 * k;
            ok[k]           = i < lv.nPts;
            const int32_t e = __ldg( lv.pts + ( ok[k] ? i : lv.nPts - 1 ) );
            const int     g  = e & 255, b = e >> 8;
            const int4    P0 = __ldg( lv.pro + 2 * b ), P1 = __ldg( lv.pro + 2 * b + 1 );
            const T*      cc = coarse + size_t( cell ) * strideC;
            fi[k]            = size_t( cell ) * lv.stride + __ldg( lv.blk + 16 * size_t( b ) ) + g;
            const T a        = cc[( ( g & 1 ) ? P0.y : P0.x ) + ( ( P0.z + 2 * g ) >> 2 )];
            v[k]             = P1.z ? a : T( 0.5 ) * ( a + cc[( ( g & 1 ) ? P1.x : P0.w ) + ( ( P1.y + 2 * g ) >> 2 )] );
         }
#pragma unroll
         for ( int k = 0; k < K; ++k )
            if ( ok[k] )
               fine[fi[k]] = ADD ? fine[fi[k]] + v[k] : v[k];
      }
      return;
   }
   const BdryLists bl = fullBdryLists( tp, lv );
   HYB_BDRY_LANES( bl )
   {
      const LaneTask  tk = laneTask( tp, lv, bl, gt );
      const BdryPoint p  = decodeBdry( tp, lv, tk.t );
      if ( !tk.valid || !( primBc( tp, p.kind, p.prim ) & flag ) )
         continue;
      int c, x, y, z;
      embeddingCoords( embAt( tp, p.kind, p.prim, 0 ), p.kind, lv.N, p.i, p.j, c, x, y, z );
      T v = interpolateFine( coarse + size_t( c ) * strideC, Wc, x, y, z );
      if ( ADD )
         v += fine[size_t( c ) * lv.stride + sidx( lv.W, x, y, z )];
      // every lane of the group has read the old value before any replica is written
      __syncwarp( __activemask() );
      bdryWriteGroup( tp, lv, p, tk, fine, v );
   }
}

template < typename T, bool ADD >
__global__ void __launch_bounds__( 128 ) k_prolongate( TopoDev tp, LevelDev lv, int Wc, int strideC,
                                                       const T* __restrict__ coarse, T* __restrict__ fine, int flag,
                                                       int nCellBlocks )
{
   HYB_PDL_PROLOGUE();
   prolongateBody< T, ADD >( launchBlk(), tp, lv, Wc, strideC, coarse, fine, flag, nCellBlocks );
}

// ---------------------------------------------------------------------------
// Full-weighting restriction (P1toP1LinearRestriction.cpp:168-345 with the generated
// pull kernel): r_c(P) = r_f(2P) + 1/2 sum of r_f over the fine neighbours of 2P. A
// boundary coarse DoF gathers in every adjacent cell, each fine point scaled by
// 1/#cells of the primitive it lies on, so every fine point counts exactly once.
// ---------------------------------------------------------------------------
template < typename T >
__device__ __forceinline__ void restrictBody( Blk vb, TopoDev tp, LevelDev lv, int Wf, int strideF, const T* fine,
                                                     T* coarse, int flag, int nCellBlocks )
{
   if ( vb.x < nCellBlocks )
   {
      HYB_CELL_LOOP( lv.nSeg )
      {
         const int     cell = it_ / lv.nSeg;
         const int32_t sp   = lv.seg[it_ - cell * lv.nSeg];
         const int     z = sp & 1023, y = ( sp >> 10 ) & 1023, x = ( sp >> 20 ) + ( threadIdx.x & 31 );
         if ( x + y + z > lv.N - 1 )
            continue;
         // the fine point 2P = (4g' + r', 2y, 2z) with r' = 2x mod 4, g' = 2x div 4
         const T*     f  = fine + size_t( cell ) * strideF;
         const int    gf = ( 2 * x ) >> 2;
         const NbrOff no = residueNbr( Wf, 2 * y, 2 * z, ( 2 * x ) & 3 );
         T            s  = 0;
#pragma unroll
         for ( int q = 1; q < 15; ++q )
            s += f[no.d[q] + gf];
         coarse[size_t( cell ) * lv.stride + sidx( lv.W, x, y, z )] = f[no.d[0] + gf] + T( 0.5 ) * s;
      }
      return;
   }
   const int       Nf = Wf - 1;
   const BdryLists bl = fullBdryLists( tp, lv );
   HYB_BDRY_LANES( bl )
   {
      const LaneTask  tk     = laneTask( tp, lv, bl, gt );
      const BdryPoint p      = decodeBdry( tp, lv, tk.t );
      const bool      active = tk.valid && ( primBc( tp, p.kind, p.prim ) & flag );
      T               acc    = 0;
      if ( active )
      {
         const int ne = numEmb( tp, p.kind, p.prim );
         for ( int e = tk.sub; e < ne; e += tk.G )
         {
            int c, x, y, z;
            embeddingCoords( embAt( tp, p.kind, p.prim, e ), p.kind, lv.N, p.i, p.j, c, x, y, z );
            const int       X = 2 * x, Y = 2 * y, Z = 2 * z;
            const T*        f     = fine + size_t( c ) * strideF;
            const ClassDev* cc    = tp.cls + size_t( c ) * 16;
            const int       mask  = classMask( Nf, X, Y, Z );
            const uint32_t  valid = kValidOffsets[mask];
            acc += T( cc[mask].invN ) * f[sidx( Wf, X, Y, Z )];
            for ( int q = 1; q < 15; ++q )
               if ( valid & ( 1u << q ) )
               {
                  const int xq = X + offX( q ), yq = Y + offY( q ), zq = Z + offZ( q );
                  const int mq = classMask( Nf, xq, yq, zq );
                  acc += T( 0.5 * cc[mq].invN ) * f[sidx( Wf, xq, yq, zq )];
               }
         }
      }
      acc = groupSum( acc, tk.G );
      if ( active )
         bdryWriteGroup( tp, lv, p, tk, coarse, acc );
   }
}

template < typename T >
__global__ void __launch_bounds__( 128 ) k_restrict( TopoDev tp, LevelDev lv, int Wf, int strideF, const T* __restrict__ fine,
                                                     T* __restrict__ coarse, int flag, int nCellBlocks )
{
   HYB_PDL_PROLOGUE();
   restrictBody< T >( launchBlk(), tp, lv, Wf, strideF, fine, coarse, flag, nCellBlocks );
}

// ---------------------------------------------------------------------------
// Pointwise vector kernels over whole cell slabs (all replicas; consistent by
// construction). blockIdx.y = cell.
// ---------------------------------------------------------------------------
template < typename T >
__global__ void k_lincomb( TopoDev tp, LevelDev lv, T* __restrict__ dst, int n, T s0, const T* a0, T s1, const T* a1, T s2,
                           const T* a2, int add, int flag )
{
   HYB_PDL_PROLOGUE();
   const int idx = blockIdx.x * blockDim.x + threadIdx.x;
   if ( idx >= lv.S )
      return;
   const int cell = blockIdx.y;
   const int p    = lv.xyz[idx];
   const int mask = classMask( lv.N, p & 1023, ( p >> 10 ) & 1023, p >> 20 );
   if ( !( tp.cls[cell * 16 + mask].bc & flag ) )
      return;
   const size_t i = size_t( cell ) * lv.stride + idx;
   T            v = add ? dst[i] : T( 0 );
   if ( n > 0 )
      v += s0 * a0[i];
   if ( n > 1 )
      v += s1 * a1[i];
   if ( n > 2 )
      v += s2 * a2[i];
   dst[i] = v;
}

// ---------------------------------------------------------------------------
// Seeded synthetic inputs evaluated on the device at every closure point (replicas get
// identical values: they depend on the position only).
//   * uniform right-hand side: f ~ U[-1,1] from a SplitMix64 hash of the point's integer
//     position on the lattice of spacing 1/lattice and the seed;
//   * random-Fourier-feature coefficient: k = exp( radial (1 - |x|) + sigma sqrt(2/M) sum_m cos(w_m . x + p_m) ).
// Cell geometry: cellCoords[c] = 4 vertices x 3 in the cell's local order; cellOrder[c] packs
// the local indices of the vertices sorted by global id (2 bits each). The position is the
// barycentric sum taken in global vertex order, so every replica of a shared point (whose
// weights on the other vertices are exactly zero) evaluates the same expression and gets
// the same bits.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void closurePosition( const double* __restrict__ cellCoords,
                                                 const int32_t* __restrict__ cellOrder, int cell, int N, int x, int y,
                                                 int z, double p[3] )
{
   const double* v     = cellCoords + size_t( cell ) * 12;
   const int     order = cellOrder[cell];
   const double  b[4]  = { double( N - x - y - z ), double( x ), double( y ), double( z ) };
   for ( int d = 0; d < 3; ++d )
   {
      double acc = 0.0;
      for ( int j = 0; j < 4; ++j )
      {
         const int k = ( order >> ( 2 * j ) ) & 3;
         acc += b[k] * v[3 * k + d];
      }
      p[d] = acc / N;
   }
}

__device__ __forceinline__ uint64_t splitmix64( uint64_t x )
{
   x += 0x9E3779B97F4A7C15ull;
   uint64_t z = x;
   z          = ( z ^ ( z >> 30 ) ) * 0xBF58476D1CE4E5B9ull;
   z          = ( z ^ ( z >> 27 ) ) * 0x94D049BB133111EBull;
   return z ^ ( z >> 31 );
}

template < typename T >
__global__ void k_fill_uniform_hash( TopoDev tp, LevelDev lv, const double* __restrict__ cellCoords,
                                     const int32_t* __restrict__ cellOrder, T* __restrict__ dst, uint64_t seed,
                                     double lattice )
{
   HYB_PDL_PROLOGUE();
   const int idx = blockIdx.x * blockDim.x + threadIdx.x;
   if ( idx >= lv.S )
      return;
   const int cell = blockIdx.y;
   const int pk   = lv.xyz[idx];
   double    p[3];
   closurePosition( cellCoords, cellOrder, cell, lv.N, pk & 1023, ( pk >> 10 ) & 1023, pk >> 20, p );
   const uint64_t kx = uint64_t( llrint( p[0] * lattice ) ), ky = uint64_t( llrint( p[1] * lattice ) ),
                  kz = uint64_t( llrint( p[2] * lattice ) );
   const uint64_t key = ( kx * 1000003ull + ky ) * 1000033ull + kz;
   const uint64_t h   = splitmix64( key ^ ( seed * 0xD1B54A32D192ED03ull ) );
   dst[size_t( cell ) * lv.stride + idx] = T( double( h >> 11 ) / 9007199254740992.0 * 2.0 - 1.0 );
}

template < typename T >
__global__ void k_fill_rff_coefficient( TopoDev tp, LevelDev lv, const double* __restrict__ cellCoords,
                                        const int32_t* __restrict__ cellOrder, T* __restrict__ dst,
                                        const double* __restrict__ w, const double* __restrict__ phase, int modes,
                                        double sigma, double radial )
{
   HYB_PDL_PROLOGUE();
   const int idx = blockIdx.x * blockDim.x + threadIdx.x;
   if ( idx >= lv.S )
      return;
   const int cell = blockIdx.y;
   const int pk   = lv.xyz[idx];
   double    p[3];
   closurePosition( cellCoords, cellOrder, cell, lv.N, pk & 1023, ( pk >> 10 ) & 1023, pk >> 20, p );
   double g = 0;
   for ( int m = 0; m < modes; ++m )
      g += cos( w[3 * m] * p[0] + w[3 * m + 1] * p[1] + w[3 * m + 2] * p[2] + phase[m] );
   const double r = sqrt( p[0] * p[0] + p[1] * p[1] + p[2] * p[2] );
   dst[size_t( cell ) * lv.stride + idx] = T( exp( radial * ( 1.0 - r ) + sigma * sqrt( 2.0 / modes ) * g ) );
}

// Coefficient functions of the quadrature-point operator (the reference form's callback):
// kind 1: tanh(2 (x - 1/2)) + 2 (ElementwiseDivKGradCGConvergenceTest.cpp:41-137);
// kind 2: exp( radial (1 - |x|) + sigma sqrt(2/M) sum_m cos( w_m . x + phase_m ) ), the random
// Fourier-feature field (w: M x 3, phase: M).
struct CoefFn
{
   int           kind, modes;
   double        sigma, radial;
   const double* w;
   const double* phase;
};

__device__ __forceinline__ double coefValue( const CoefFn& f, const double p[3] )
{
   if ( f.kind == 1 )
      return tanh( 2.0 * ( p[0] - 0.5 ) ) + 2.0;
   double g = 0;
   for ( int m = 0; m < f.modes; ++m )
      g += cos( f.w[3 * m] * p[0] + f.w[3 * m + 1] * p[1] + f.w[3 * m + 2] * p[2] + f.phase[m] );
   const double r = sqrt( p[0] * p[0] + p[1] * p[1] + p[2] * p[2] );
   return exp( f.radial * ( 1.0 - r ) + f.sigma * sqrt( 2.0 / f.modes ) * g );
}

// nodal values of a coefficient function (closure layout)
__global__ void k_fill_coefficient( LevelDev lv, const double* __restrict__ cellCoords,
                                    const int32_t* __restrict__ cellOrder, double* __restrict__ dst, CoefFn f )
{
   const int idx = blockIdx.x * blockDim.x + threadIdx.x;
   if ( idx >= lv.S )
      return;
   const int cell = blockIdx.y;
   const int pk   = lv.xyz[idx];
   double    p[3];
   closurePosition( cellCoords, cellOrder, cell, lv.N, pk & 1023, ( pk >> 10 ) & 1023, pk >> 20, p );
   dst[size_t( cell ) * lv.stride + idx] = coefValue( f, p );
}

// The quadrature factors of OpDev::kq: for every micro-tet (type t, vertex 0 at closure point
// idx) inside the closure, 24 sum_q w_q k(x_q) with the 5-point degree-3 rule of
// p1_div_k_grad_affine_q3 (centroid, weight -2/15; the points with barycentric coordinates
// (1/2, 1/6, 1/6, 1/6), weight 3/40; p1_div_k_grad_affine_q3.cpp:179+). Slots of micro-tets
// that leave the closure are set to 0 and never read.
__global__ void k_fill_tet_factors( LevelDev lv, const double* __restrict__ cellCoords,
                                    const int32_t* __restrict__ cellOrder, double* __restrict__ dst, CoefFn f )
{
   const int idx = blockIdx.x * blockDim.x + threadIdx.x;
   if ( idx >= lv.S )
      return;
   const int cell = blockIdx.y;
   const int pk   = lv.xyz[idx];
   const int x = pk & 1023, y = ( pk >> 10 ) & 1023, z = pk >> 20;
   for ( int t = 0; t < 6; ++t )
   {
      // the micro-tet of type t with this point as its vertex 0 (role 0 of incidentTet)
      int q[4] = { 0, 0, 0, 0 };
      for ( int i = 0; i < 24; ++i )
      {
         const IncidentTet it = incidentTet( i );
         if ( it.t == t && it.k == 0 )
            for ( int j = 0; j < 4; ++j )
               q[j] = it.q[j];
      }
      double X[4][3];
      bool   inside = true;
      for ( int j = 0; j < 4 && inside; ++j )
      {
         const int xx = x + offX( q[j] ), yy = y + offY( q[j] ), zz = z + offZ( q[j] );
         inside       = xx >= 0 && yy >= 0 && zz >= 0 && xx + yy + zz <= lv.N;
         if ( inside )
            closurePosition( cellCoords, cellOrder, cell, lv.N, xx, yy, zz, X[j] );
      }
      double s = 0;
      if ( inside )
         for ( int qp = 0; qp < 5; ++qp )
         {
            double p[3];
            for ( int d = 0; d < 3; ++d )
            {
               double acc = 0;
               for ( int j = 0; j < 4; ++j )
                  acc += ( qp == 0 ? 0.25 : ( j == qp - 1 ? 0.5 : 1.0 / 6.0 ) ) * X[j][d];
               p[d] = acc;
            }
            s += ( qp == 0 ? -2.0 / 15.0 : 3.0 / 40.0 ) * coefValue( f, p );
         }
      dst[( size_t( cell ) * 6 + t ) * lv.stride + idx] = 24.0 * s;
   }
}

// VertexDoFFunction::interpolate(constant, level, flag)
template < typename T >
__global__ void k_fill( TopoDev tp, LevelDev lv, T* __restrict__ dst, T value, int flag )
{
   HYB_PDL_PROLOGUE();
   const int idx = blockIdx.x * blockDim.x + threadIdx.x;
   if ( idx >= lv.S )
      return;
   const int cell = blockIdx.y;
   const int p    = lv.xyz[idx];
   const int mask = classMask( lv.N, p & 1023, ( p >> 10 ) & 1023, p >> 20 );
   if ( tp.cls[cell * 16 + mask].bc & flag )
      dst[size_t( cell ) * lv.stride + idx] = value;
}

template < typename TD, typename TS >
__global__ void k_convert( LevelDev lv, TD* __restrict__ dst, const TS* __restrict__ src, int nCells )
{
   HYB_PDL_PROLOGUE();
   const size_t i = size_t( blockIdx.x ) * blockDim.x + threadIdx.x;
   if ( i < size_t( nCells ) * lv.stride )
      dst[i] = TD( src[i] );
}

// x64 += e (FP32 correction) on flagged points
template < typename T, typename TE >
__global__ void k_add_correction( TopoDev tp, LevelDev lv, T* __restrict__ x, const TE* __restrict__ e, int flag )
{
   HYB_PDL_PROLOGUE();
   const int idx = blockIdx.x * blockDim.x + threadIdx.x;
   if ( idx >= lv.S )
      return;
   const int cell = blockIdx.y;
   const int p    = lv.xyz[idx];
   const int mask = classMask( lv.N, p & 1023, ( p >> 10 ) & 1023, p >> 20 );
   if ( !( tp.cls[cell * 16 + mask].bc & flag ) )
      return;
   const size_t i = size_t( cell ) * lv.stride + idx;
   x[i] += T( e[i] );
}

// Partial dot products over the canonical replica of every DoF whose BC is in flag. With
// cvt given, the pass also writes float(a) at every closure point (the mixed-precision
// refinement's FP32 right-hand side from the FP64 residual, read once for both).
template < typename T >
__global__ void k_dot_partial( TopoDev tp, LevelDev lv, const T* __restrict__ a, const T* __restrict__ b, int flag,
                               double* __restrict__ partial, float* __restrict__ cvt )
{
   HYB_PDL_PROLOGUE();
   __shared__ double red[32];
   const int idx  = blockIdx.x * blockDim.x + threadIdx.x;
   const int cell = blockIdx.y;
   double    v    = 0;
   if ( idx < lv.S )
   {
      if ( cvt )
         cvt[size_t( cell ) * lv.stride + idx] = float( a[size_t( cell ) * lv.stride + idx] );
      const int p    = lv.xyz[idx];
      const int mask = classMask( lv.N, p & 1023, ( p >> 10 ) & 1023, p >> 20 );
      const ClassDev cd = tp.cls[cell * 16 + mask];
      if ( cd.owned && ( cd.bc & flag ) )
      {
         const size_t i = size_t( cell ) * lv.stride + idx;
         v              = double( a[i] ) * double( b[i] );
      }
   }
   for ( int o = 16; o > 0; o >>= 1 )
      v += __shfl_down_sync( 0xffffffffu, v, o );
   if ( ( threadIdx.x & 31 ) == 0 )
      red[threadIdx.x >> 5] = v;
   __syncthreads();
   if ( threadIdx.x < 32 )
   {
      v = threadIdx.x < ( blockDim.x >> 5 ) ? red[threadIdx.x] : 0.0;
      for ( int o = 16; o > 0; o >>= 1 )
         v += __shfl_down_sync( 0xffffffffu, v, o );
      if ( threadIdx.x == 0 )
         partial[size_t( blockIdx.y ) * gridDim.x + blockIdx.x] = v;
   }
}

// Deterministic second pass: one block sums the partials in a fixed order.
__global__ void k_reduce_final( const double* __restrict__ partial, int n, double* __restrict__ out )
{
   HYB_PDL_PROLOGUE();
   __shared__ double red[32];
   double            v = 0;
   for ( int i = threadIdx.x; i < n; i += blockDim.x )
      v += partial[i];
   for ( int o = 16; o > 0; o >>= 1 )
      v += __shfl_down_sync( 0xffffffffu, v, o );
   if ( ( threadIdx.x & 31 ) == 0 )
      red[threadIdx.x >> 5] = v;
   __syncthreads();
   if ( threadIdx.x < 32 )
   {
      v = threadIdx.x < ( blockDim.x >> 5 ) ? red[threadIdx.x] : 0.0;
      for ( int o = 16; o > 0; o >>= 1 )
         v += __shfl_down_sync( 0xffffffffu, v, o );
      if ( threadIdx.x == 0 )
         *out = v;
   }
}

// Canonical DoF order <-> cell slabs (see oracle/hyteg_oracle.h for the order).
__device__ __forceinline__ int64_t canonicalDof( const TopoDev& tp, const LevelDev& lv, int cell, int x, int y, int z )
{
   const int       N    = lv.N;
   const int       mask = classMask( N, x, y, z );
   const ClassDev& cd   = tp.cls[cell * 16 + mask];
   const int       b[4] = { N - x - y - z, x, y, z };
   const int64_t   offE = tp.nV, offF = offE + int64_t( tp.nE ) * ( N - 1 ), offC = offF + int64_t( tp.nF ) * lv.nIntFace;
   switch ( cd.kind )
   {
   case 0: return cd.id;
   case 1: return offE + int64_t( cd.id ) * ( N - 1 ) + ( b[cd.k1] - 1 );
   case 2: {
      const int i = b[cd.k1], j = b[cd.k2];
      return offF + int64_t( cd.id ) * lv.nIntFace + ( j - 1 ) * ( N - 1 ) - ( j - 1 ) * j / 2 + ( i - 1 );
   }
   default: return offC + int64_t( cell ) * lv.nIntCell + cidx( N - 3, x - 1, y - 1, z - 1 );
   }
}

template < typename T >
__global__ void k_from_dofs( TopoDev tp, LevelDev lv, T* __restrict__ slab, const T* __restrict__ dofs )
{
   HYB_PDL_PROLOGUE();
   const int idx = blockIdx.x * blockDim.x + threadIdx.x;
   if ( idx >= lv.S )
      return;
   const int cell = blockIdx.y;
   const int p    = lv.xyz[idx];
   slab[size_t( cell ) * lv.stride + idx] = dofs[canonicalDof( tp, lv, cell, p & 1023, ( p >> 10 ) & 1023, p >> 20 )];
}

template < typename T >
__global__ void k_to_dofs( TopoDev tp, LevelDev lv, const T* __restrict__ slab, T* __restrict__ dofs )
{
   HYB_PDL_PROLOGUE();
   const int idx = blockIdx.x * blockDim.x + threadIdx.x;
   if ( idx >= lv.S )
      return;
   const int cell = blockIdx.y;
   const int p    = lv.xyz[idx];
   const int x = p & 1023, y = ( p >> 10 ) & 1023, z = p >> 20;
   if ( !tp.cls[cell * 16 + classMask( lv.N, x, y, z )].owned )
      return;
   dofs[canonicalDof( tp, lv, cell, x, y, z )] = slab[size_t( cell ) * lv.stride + idx];
}

// ---------------------------------------------------------------------------
// Coarse-grid CG (CGSolver::solve, src/hyteg/solvers/CGSolver.hpp:66-135, init :237+),
// identity preconditioner, absolute test sqrt(r.r) < tol, flag Inner|Neumann|Freeslip.
// The whole iteration runs in ONE thread block (coarse levels hold at most a few
// thousand DoFs); scalars stay on the device, so it can be captured in a CUDA graph.
// status[0] = iterations, status[1] = 1 if converged, 2 if the budget ran out.
// ---------------------------------------------------------------------------
template < int VAR >
__device__ void cgApplyAll( const TopoDev& tp, const LevelDev& lv, const OpDev< double >& op, const double* src,
                            double* dst, int flag )
{
   // interior points
   const int nInt = lv.nIntCell;
   for ( int t = threadIdx.x; t < tp.nC * lv.S; t += blockDim.x )
   {
      const int cell = t / lv.S, idx = t % lv.S;
      const int p    = lv.xyz[idx];
      const int x = p & 1023, y = ( p >> 10 ) & 1023, z = p >> 20;
      if ( classMask( lv.N, x, y, z ) != 0 )
         continue;
      double d = 0, o = 0;
      partialRow< double, VAR >( op, src + size_t( cell ) * lv.stride, cell, lv.W, x, y, z, d, o );
      const size_t i = size_t( cell ) * lv.stride + idx;
      dst[i]         = d * src[i] + o;
   }
   (void) nInt;
   for ( int t = threadIdx.x; t < lv.nBdry; t += blockDim.x )
   {
      const BdryPoint pnt = decodeBdry( tp, lv, t );
      if ( !( primBc( tp, pnt.kind, pnt.prim ) & flag ) )
         continue;
      double d = 0, o = 0;
      bdryRow< double, VAR >( tp, lv, op, src, pnt, d, o );
      bdryWriteAll( tp, lv, pnt, dst, d * src[bdryReplica< double >( tp, lv, pnt, 0 )] + o );
   }
}

__device__ double blockSum( double v, double* red )
{
   for ( int o = 16; o > 0; o >>= 1 )
      v += __shfl_down_sync( 0xffffffffu, v, o );
   __syncthreads();
   if ( ( threadIdx.x & 31 ) == 0 )
      red[threadIdx.x >> 5] = v;
   __syncthreads();
   double s = 0;
   for ( int w = 0; w < int( blockDim.x >> 5 ); ++w )
      s += red[w];
   return s;
}

__device__ double cgDot( const TopoDev& tp, const LevelDev& lv, const double* a, const double* b, int flag, double* red )
{
   double v = 0;
   for ( int t = threadIdx.x; t < tp.nC * lv.S; t += blockDim.x )
   {
      const int cell = t / lv.S, idx = t % lv.S;
      const int p    = lv.xyz[idx];
      const ClassDev cd = tp.cls[cell * 16 + classMask( lv.N, p & 1023, ( p >> 10 ) & 1023, p >> 20 )];
      if ( cd.owned && ( cd.bc & flag ) )
         v += a[size_t( cell ) * lv.stride + idx] * b[size_t( cell ) * lv.stride + idx];
   }
   return blockSum( v, red );
}

// y = a*x + b*y over flagged points of all replicas
__device__ void cgAxpby( const TopoDev& tp, const LevelDev& lv, double a, const double* x, double b, double* y, int flag )
{
   for ( int t = threadIdx.x; t < tp.nC * lv.S; t += blockDim.x )
   {
      const int cell = t / lv.S, idx = t % lv.S;
      const int p    = lv.xyz[idx];
      if ( !( tp.cls[cell * 16 + classMask( lv.N, p & 1023, ( p >> 10 ) & 1023, p >> 20 )].bc & flag ) )
         continue;
      const size_t i = size_t( cell ) * lv.stride + idx;
      y[i]           = a * x[i] + b * y[i];
   }
}

// the whole CG in the calling thread block; red = 32 doubles of shared memory
template < int VAR, bool BLEND = false >
__device__ void cgBody( const TopoDev& tp, const LevelDev& lv, const OpDev< double >& op, double* x, const double* b,
                        double* r, double* p, double* ap, double tol, int maxIter, int* status, double* red,
                        const RowPass& rp )
{
   const int flag = 1 | 4 | 8;
   // the operator through the level's row table when there is one
   auto applyA = [&]( const double* src, double* dst ) {
      if ( BLEND || rp.rows )
         rowPassBody< double, kRowApply, VAR, BLEND >( rp, op, const_cast< double* >( src ), nullptr, dst, 0.0, flag,
                                                       threadIdx.x, blockDim.x );
      else
         cgApplyAll< VAR >( tp, lv, op, src, dst, flag );
   };
   applyA( x, p );
   __syncthreads();
   // r = b - A x ; p = r
   for ( int t = threadIdx.x; t < tp.nC * lv.S; t += blockDim.x )
   {
      const int cell = t / lv.S, idx = t % lv.S;
      const int pp   = lv.xyz[idx];
      if ( !( tp.cls[cell * 16 + classMask( lv.N, pp & 1023, ( pp >> 10 ) & 1023, pp >> 20 )].bc & flag ) )
         continue;
      const size_t i = size_t( cell ) * lv.stride + idx;
      r[i]           = b[i] - p[i];
      p[i]           = r[i];
   }
   __syncthreads();
   double prsold = cgDot( tp, lv, r, r, flag, red );
   int    it     = 0;
   int    conv   = sqrt( prsold ) < tol ? 1 : 0;
   while ( !conv && it < maxIter )
   {
      applyA( p, ap );
      __syncthreads();
      const double pAp   = cgDot( tp, lv, p, ap, flag, red );
      const double alpha = prsold / pAp;
      cgAxpby( tp, lv, alpha, p, 1.0, x, flag );
      cgAxpby( tp, lv, -alpha, ap, 1.0, r, flag );
      __syncthreads();
      const double rsnew = cgDot( tp, lv, r, r, flag, red );
      ++it;
      if ( sqrt( rsnew ) < tol )
      {
         conv = 1;
         break;
      }
      const double beta = rsnew / prsold;
      cgAxpby( tp, lv, 1.0, r, beta, p, flag );
      __syncthreads();
      prsold = rsnew;
   }
   if ( threadIdx.x == 0 )
   {
      status[0] = it;
      status[1] = conv ? 1 : 2;
   }
}

template < int VAR, bool BLEND = false >
__global__ void __launch_bounds__( 256 ) k_cg( TopoDev tp, LevelDev lv, OpDev< double > op, double* x, const double* b,
                                                double* r, double* p, double* ap, double tol, int maxIter, int* status,
                                                RowPass rp )
{
   HYB_PDL_PROLOGUE();
   __shared__ double red[32];
   cgBody< VAR, BLEND >( tp, lv, op, x, b, r, p, ap, tol, maxIter, status, red, rp );
}

// ---------------------------------------------------------------------------
// Device-side stopping test of an iterated solve (GeometricMultigridSolver's outer loop
// without a host round trip per cycle): scalars[0] = ||b - A x||^2 of the current iterate,
// scalars[1] = ||b||^2. With init the cycle count starts at 0 and ||b|| is taken; otherwise
// one more cycle has run. The graph's WHILE condition stays set while the relative residual
// is above the tolerance, finite, and the cycle budget is not spent.
// ---------------------------------------------------------------------------
struct SolveCtl
{
   double tol;
   int    maxCycles;
   int    cycles;
   double nb;  // ||b|| (1 if b = 0)
   double rel; // relative residual of the last iterate
};

__global__ void k_solve_ctl( cudaGraphConditionalHandle h, SolveCtl* c, const double* __restrict__ scalars, int init )
{
   if ( init )
   {
      c->cycles = 0;
      c->nb     = scalars[1] > 0 ? sqrt( scalars[1] ) : 1.0;
   }
   else
      c->cycles += 1;
   const double rel = sqrt( scalars[0] ) / c->nb;
   c->rel           = rel;
   cudaGraphSetConditional( h, ( rel > c->tol && c->cycles < c->maxCycles ) ? 1u : 0u ); // NaN stops too
}

} // namespace hyb
