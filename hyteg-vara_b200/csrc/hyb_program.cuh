// Program kernel: the small levels of a V-cycle in ONE launch of ONE thread block.
//
// On coarse levels every smoother pass, residual and transfer is a launch of a few
// microseconds, so a V-cycle's coarse part is bound by launch latency, not by work. The
// host records those level operations as a list of phases (the same bodies the separate
// kernels run) and a single thread block executes the list, separating consecutive phases
// by __syncthreads(): within one block that is both the execution and the memory barrier
// (measured on B200, a grid-wide barrier across blocks costs 1-2.5 us, a kernel node of a
// CUDA graph about 4 us, __syncthreads a few tens of ns). The small levels' data stays in
// the multiprocessor's L1.
#pragma once

#include "hyb_kernels.cuh"

namespace hyb {

enum PhaseKind : int
{
   kPhSorIface    = 0, // one interface colour: p0 = u, p1 = rhs, bl, flag, relax
   kPhSorInterior = 1, // one interior colour: p0 = u, p1 = rhs, a0 = colour, a1 = begin, a2 = count, relax
   kPhJacobi      = 2, // p0 = src (old iterate), p1 = dst, p2 = rhs, flag, relax
   kPhCopy        = 3, // p0 = dst, p1 = src, n elements of T
   kPhResidual    = 4, // p0 = x, p1 = r, p2 = b, flag
   kPhRestrict    = 5, // p0 = fine, p1 = coarse (level = coarse level), flag
   kPhProlongAdd  = 6, // p0 = coarse, p1 = fine (level = fine level), flag
   kPhZero        = 7, // p0 = dst, n elements of T
   kPhToF64       = 8, // p0 = double dst, p1 = float src, n elements
   kPhToF32       = 9, // p0 = float dst, p1 = double src, n elements
   kPhCg          = 10, // FP64 CG on the level: p0 = x, p1 = b, p2 = r, p3 = p, p4 = ap, status, relax = tol, a0 = maxIter
   // phases of a whole solve (k_solve_batch); all FP64 except where noted
   kPhDot     = 11, // scalar slot a0 = p0 . p1 over the owned DoFs on flag; p2: float(p0) at every closure point, or null
   kPhAddCorr = 12, // p0 += (double) p1 (float) on the closure points on flag
   kPhCtl     = 13  // stopping test (SolveCtl at p0): a1 = 1 starts the count; go on at phase a0 while it fails
};

struct Phase
{
   int             kind;
   int             level;      // index into the level table
   int             blocks;     // virtual blocks: the cell-interior loop's, then the surface loop's
   int             cellBlocks; // of which the cell-interior loop's
   int             a0, a1, a2;
   int             flag;
   int             dtype; // HYB_F64 or HYB_F32: the value type of the phase's data (k_solve_batch)
   int             pad;
   double          relax;
   long long       n;
   void*           p0;
   void*           p1;
   void*           p2;
   void*           p3;
   void*           p4;
   int*            status;
   BdryLists       bl;
   OpDev< float >  op32; // operator of the phase's level in both types
   OpDev< double > op64;
   RowPass         rp;   // row table of the pass (constant operator, small levels) or rows = nullptr
};

template < typename T >
__device__ __forceinline__ const OpDev< T >& phaseOp( const Phase& P );
template <>
__device__ __forceinline__ const OpDev< float >& phaseOp< float >( const Phase& P )
{
   return P.op32;
}
template <>
__device__ __forceinline__ const OpDev< double >& phaseOp< double >( const Phase& P )
{
   return P.op64;
}

constexpr int kProgramThreads = 512;

constexpr int kProgramLevels = 8; // level descriptors staged in shared memory

// One phase of a program, run by the program's thread blocks (block pb of npb): a row pass
// spreads its rows over every thread, any other phase steps through its virtual blocks.
// sL holds the first kProgramLevels level descriptors (staged in shared memory), lvs all.
template < typename T, int VAR >
__device__ __forceinline__ void runPhase( const TopoDev& tp, const Phase& P, const LevelDev* sL,
                                          const LevelDev* __restrict__ lvs, double* red, int pb, int npb )
{
   auto levelAt = [&]( int l ) -> const LevelDev& { return l < kProgramLevels ? sL[l] : lvs[l]; };
   const int      kind   = P.kind;
   const int      blocks = P.blocks;
   // row passes spread over every thread of the block
   const bool rowPass = P.rp.rows && ( kind == kPhSorIface || kind == kPhSorInterior || kind == kPhResidual );
   if ( rowPass )
   {
      const long long start = (long long) pb * blockDim.x + threadIdx.x, step = (long long) npb * blockDim.x;
      if ( kind == kPhResidual )
         rowPassBody< T, kRowResidual, VAR >( P.rp, phaseOp< T >( P ), (T*) P.p0, (const T*) P.p2, (T*) P.p1, T( 0 ),
                                              P.flag, start, step );
      else
         rowPassBody< T, kRowSor, VAR >( P.rp, phaseOp< T >( P ), (T*) P.p0, (const T*) P.p1, nullptr, T( P.relax ),
                                         kind == kPhSorIface ? P.flag : 0xff, start, step );
   }
   for ( int b = pb; !rowPass && b < blocks; b += npb )
   {
      const LevelDev& lv = levelAt( P.level );
      const Blk       vb{ b, blocks };
      const long long t0 = (long long) b * blockDim.x + threadIdx.x, step = (long long) blocks * blockDim.x;
      switch ( kind )
      {
      case kPhSorIface:
         sorIfaceBody< T, VAR >( vb, tp, lv, phaseOp< T >( P ), (T*) P.p0, (const T*) P.p1, T( P.relax ), P.flag, P.bl );
         break;
      case kPhSorInterior:
         sorInteriorBody< T, VAR >( vb, tp, lv, phaseOp< T >( P ), (T*) P.p0, (const T*) P.p1, T( P.relax ), P.a0, P.a1,
                                    P.a2, P.cellBlocks );
         break;
      case kPhJacobi:
         jacobiBody< T, VAR >( vb, tp, lv, phaseOp< T >( P ), (const T*) P.p0, (T*) P.p1, (const T*) P.p2, T( P.relax ),
                               P.flag, P.cellBlocks );
         break;
      case kPhCopy:
         for ( long long i = t0; i < P.n; i += step )
            ( (T*) P.p0 )[i] = ( (const T*) P.p1 )[i];
         break;
      case kPhResidual:
         applyBody< T, VAR, kResidual >( vb, tp, lv, phaseOp< T >( P ), (const T*) P.p0, (T*) P.p1, (const T*) P.p2,
                                         P.flag, P.cellBlocks );
         break;
      case kPhRestrict:
      {
         const LevelDev& F = levelAt( P.level + 1 );
         restrictBody< T >( vb, tp, lv, F.W, F.stride, (const T*) P.p0, (T*) P.p1, P.flag, P.cellBlocks );
         break;
      }
      case kPhProlongAdd:
      {
         const LevelDev& C = levelAt( P.level - 1 );
         prolongateBody< T, true >( vb, tp, lv, C.W, C.stride, (const T*) P.p0, (T*) P.p1, P.flag, P.cellBlocks );
         break;
      }
      case kPhZero:
         for ( long long i = t0; i < P.n; i += step )
            ( (T*) P.p0 )[i] = T( 0 );
         break;
      case kPhToF64:
         for ( long long i = t0; i < P.n; i += step )
            ( (double*) P.p0 )[i] = double( ( (const float*) P.p1 )[i] );
         break;
      case kPhToF32:
         for ( long long i = t0; i < P.n; i += step )
            ( (float*) P.p0 )[i] = float( ( (const double*) P.p1 )[i] );
         break;
      case kPhCg:
         cgBody< VAR >( tp, lv, P.op64, (double*) P.p0, (const double*) P.p1, (double*) P.p2, (double*) P.p3,
                        (double*) P.p4, P.relax, P.a0, P.status, red, P.rp );
         break;
      default: break;
      }
   }
}

// The phase descriptors are staged in shared memory one phase ahead (each thread of the
// first warps loads one 8-byte word of the next descriptor while the current phase runs),
// and the level descriptors once per launch: a phase then starts without a dependent L2
// round trip for its own description.
template < typename T, int VAR >
__global__ void __launch_bounds__( kProgramThreads ) k_program( TopoDev tp, const LevelDev* __restrict__ lvs,
                                                                const Phase* __restrict__ prog, int nPhases, int nLv )
{
   static_assert( sizeof( Phase ) % 8 == 0 && sizeof( Phase ) / 8 <= kProgramThreads, "phase staging" );
   static_assert( sizeof( LevelDev ) % 4 == 0 && sizeof( LevelDev ) / 4 <= kProgramThreads, "level staging" );
   constexpr int       nWords = int( sizeof( Phase ) / 8 );
   __shared__ double   red[32];
   __shared__ Phase    sP[2];
   __shared__ LevelDev sL[kProgramLevels];
   HYB_PDL_PROLOGUE();
   for ( int l = 0; l < kProgramLevels && l < nLv; ++l )
      if ( threadIdx.x < sizeof( LevelDev ) / 4 )
         reinterpret_cast< int* >( &sL[l] )[threadIdx.x] = reinterpret_cast< const int* >( lvs + l )[threadIdx.x];
   if ( nPhases > 0 && threadIdx.x < nWords )
      reinterpret_cast< unsigned long long* >( &sP[0] )[threadIdx.x] =
          reinterpret_cast< const unsigned long long* >( prog )[threadIdx.x];
   __syncthreads();
   for ( int ph = 0; ph < nPhases; ++ph )
   {
      unsigned long long next = 0;
      if ( ph + 1 < nPhases && threadIdx.x < nWords )
         next = reinterpret_cast< const unsigned long long* >( prog + ph + 1 )[threadIdx.x];
      runPhase< T, VAR >( tp, sP[ph & 1], sL, lvs, red, int( blockIdx.x ), int( gridDim.x ) );
      // the next descriptor goes into the buffer the previous phase used (all threads have
      // left that phase at the last barrier)
      if ( ph + 1 < nPhases && threadIdx.x < nWords )
         reinterpret_cast< unsigned long long* >( &sP[( ph + 1 ) & 1] )[threadIdx.x] = next;
      // a phase's results are read by other threads in the next one
      __syncthreads();
   }
}

// ---------------------------------------------------------------------------
// Batched whole solves: one thread block per solve, each running its own solve program
// (recorded per hierarchy by ensureSolveProgram): ||b||^2, the start residual and its
// norm, then V-cycles (or mixed-precision refinement steps), each followed by the residual
// norm and the stopping test of k_solve_ctl, until the tolerance or the cycle limit. So one
// launch carries every small solve of a batch from right-hand side to converged solution,
// with no launch or host round trip per cycle and no kernel per solve. The blocks are
// independent: a solve's result does not depend on which batch it ran in.
// ---------------------------------------------------------------------------
struct SolveJob
{
   TopoDev         td;
   const LevelDev* lvs;
   const Phase*    prog;
   int             nLv, n;
};

// scalar slot = a . b over the owned DoFs on flag (cgDot's sum), float(a) into cvt at every
// closure point when given
__device__ __forceinline__ void dotPhase( const TopoDev& tp, const LevelDev& lv, const double* a, const double* b,
                                          float* cvt, int flag, double* red, double* slot )
{
   double          v     = 0;
   const long long total = (long long) tp.nC * lv.S;
   for ( long long t = threadIdx.x; t < total; t += blockDim.x )
   {
      const int    cell = int( t / lv.S ), idx = int( t - (long long) cell * lv.S );
      const size_t i    = size_t( cell ) * lv.stride + idx;
      if ( cvt )
         cvt[i] = float( a[i] );
      const int      p  = lv.xyz[idx];
      const ClassDev cd = tp.cls[cell * 16 + classMask( lv.N, p & 1023, ( p >> 10 ) & 1023, p >> 20 )];
      if ( cd.owned && ( cd.bc & flag ) )
         v += a[i] * b[i];
   }
   const double s = blockSum( v, red );
   if ( threadIdx.x == 0 )
      *slot = s;
}

template < int VAR >
__device__ __forceinline__ void solveBatchBody( const SolveJob* jobs )
{
   constexpr int       nWords = int( sizeof( Phase ) / 8 );
   __shared__ double   red[32];
   __shared__ double   sc[2]; // 0: ||r||^2, 1: ||b||^2
   __shared__ Phase    sP;
   __shared__ LevelDev sL[kProgramLevels];
   __shared__ SolveJob J;
   static_assert( sizeof( SolveJob ) % 8 == 0 && sizeof( SolveJob ) / 8 <= kProgramThreads, "job staging" );
   HYB_PDL_PROLOGUE();
   if ( threadIdx.x < sizeof( SolveJob ) / 8 )
      reinterpret_cast< unsigned long long* >( &J )[threadIdx.x] =
          reinterpret_cast< const unsigned long long* >( jobs + blockIdx.x )[threadIdx.x];
   __syncthreads();
   for ( int l = 0; l < kProgramLevels && l < J.nLv; ++l )
      if ( threadIdx.x < sizeof( LevelDev ) / 4 )
         reinterpret_cast< int* >( &sL[l] )[threadIdx.x] = reinterpret_cast< const int* >( J.lvs + l )[threadIdx.x];
   int    cycles = 0;
   double nb     = 1;
   for ( int ph = 0; ph < J.n; )
   {
      __syncthreads(); // the previous phase is done with sP (and, at the start, J and sL are in)
      if ( threadIdx.x < nWords )
         reinterpret_cast< unsigned long long* >( &sP )[threadIdx.x] =
             reinterpret_cast< const unsigned long long* >( J.prog + ph )[threadIdx.x];
      __syncthreads();
      const Phase& P    = sP;
      int          next = ph + 1;
      if ( P.kind == kPhDot )
      {
         const LevelDev& lv = P.level < kProgramLevels ? sL[P.level] : J.lvs[P.level];
         dotPhase( J.td, lv, (const double*) P.p0, (const double*) P.p1, (float*) P.p2, P.flag, red, &sc[P.a0] );
      }
      else if ( P.kind == kPhAddCorr )
      {
         const LevelDev& lv    = P.level < kProgramLevels ? sL[P.level] : J.lvs[P.level];
         const long long total = (long long) J.td.nC * lv.S;
         for ( long long t = threadIdx.x; t < total; t += blockDim.x )
         {
            const int cell = int( t / lv.S ), idx = int( t - (long long) cell * lv.S );
            const int p    = lv.xyz[idx];
            if ( !( J.td.cls[cell * 16 + classMask( lv.N, p & 1023, ( p >> 10 ) & 1023, p >> 20 )].bc & P.flag ) )
               continue;
            const size_t i = size_t( cell ) * lv.stride + idx;
            ( (double*) P.p0 )[i] += double( ( (const float*) P.p1 )[i] );
         }
      }
      else if ( P.kind == kPhCtl )
      {
         __syncthreads(); // the dot's slot is written by thread 0
         SolveCtl* c = (SolveCtl*) P.p0;
         if ( P.a1 )
         {
            cycles = 0;
            nb     = sc[1] > 0 ? sqrt( sc[1] ) : 1.0;
         }
         else
            ++cycles;
         const double rel = sqrt( sc[0] ) / nb;
         if ( threadIdx.x == 0 )
         {
            c->cycles = cycles;
            c->nb     = nb;
            c->rel    = rel;
         }
         if ( rel > c->tol && cycles < c->maxCycles ) // NaN stops too
            next = P.a0;
      }
      else if ( P.dtype == HYB_F32 )
         runPhase< float, VAR >( J.td, P, sL, J.lvs, red, 0, 1 );
      else
         runPhase< double, VAR >( J.td, P, sL, J.lvs, red, 0, 1 );
      ph = next;
   }
}

} // namespace hyb
