// Test infrastructure: a plain-pointer C ABI around the reference's own,
// unmodified generated macro-cell kernels (compiled from the reference source
// tree by oracle/Makefile into oracle/_ref/). Only the tests' fixture generator
// and the CPU baseline use it; it is never part of the product path.
//
// Kernels wrapped (paths relative to the reference project root):
//   src/hyteg/p1functionspace/generatedKernels/apply_3D_macrocell_vertexdof_to_vertexdof_{replace,add}.cpp:31-73
//   src/hyteg/p1functionspace/generatedKernels/sor_3D_macrocell_P1{,_backwards}.cpp:31-77
//   src/hyteg/gridtransferoperators/generatedKernels/prolongate_3D_macrocell_P1_push_additive.cpp:32-437
//   src/hyteg/gridtransferoperators/generatedKernels/restrict_3D_macrocell_P1_pull_additive.cpp:31-300
//   src/hyteg/forms/form_fenics_generated/p1_tet_diffusion.h:4093+ (tabulate_tensor)
//
// Stencil weights cross this ABI as 15 doubles in the offset order used
// throughout this repository:
//   0:(0,0,0) 1:(1,0,0) 2:(-1,0,0) 3:(0,1,0) 4:(0,-1,0) 5:(0,0,1) 6:(0,0,-1)
//   7:(-1,1,0) 8:(1,-1,0) 9:(-1,0,1) 10:(1,0,-1) 11:(0,-1,1) 12:(0,1,-1)
//   13:(-1,1,-1) 14:(1,-1,1)
#include <map>

#include "hyteg/fenics/ufc.h"
#include "hyteg/forms/form_fenics_generated/p1_tet_diffusion.h"
#include "hyteg/gridtransferoperators/generatedKernels/prolongate_3D_macrocell_P1_push_additive.hpp"
#include "hyteg/gridtransferoperators/generatedKernels/restrict_3D_macrocell_P1_pull_additive.hpp"
#include "hyteg/p1functionspace/generatedKernels/apply_3D_macrocell_vertexdof_to_vertexdof_add.hpp"
#include "hyteg/p1functionspace/generatedKernels/apply_3D_macrocell_vertexdof_to_vertexdof_replace.hpp"
#include "hyteg/p1functionspace/generatedKernels/sor_3D_macrocell_P1.hpp"
#include "hyteg/p1functionspace/generatedKernels/sor_3D_macrocell_P1_backwards.hpp"

namespace {
const int kOffsets[15][3] = { { 0, 0, 0 },   { 1, 0, 0 },  { -1, 0, 0 }, { 0, 1, 0 },  { 0, -1, 0 },
                              { 0, 0, 1 },   { 0, 0, -1 }, { -1, 1, 0 }, { 1, -1, 0 }, { -1, 0, 1 },
                              { 1, 0, -1 },  { 0, -1, 1 }, { 0, 1, -1 }, { -1, 1, -1 }, { 1, -1, 1 } };

std::map< hyteg::indexing::Index, double > toMap( const double* st )
{
   std::map< hyteg::indexing::Index, double > m;
   for ( int o = 0; o < 15; ++o )
      m[hyteg::indexing::Index( kOffsets[o][0], kOffsets[o][1], kOffsets[o][2] )] = st[o];
   return m;
}
} // namespace

extern "C" {

void ref_apply_cell( double* dst, const double* src, int level, const double* stencil15, int add )
{
   using namespace hyteg::vertexdof::macrocell::generated;
   if ( add )
      apply_3D_macrocell_vertexdof_to_vertexdof_add( dst, src, level, toMap( stencil15 ) );
   else
      apply_3D_macrocell_vertexdof_to_vertexdof_replace( dst, src, level, toMap( stencil15 ) );
}

void ref_sor_cell( double* dst, const double* rhs, int level, const double* stencil15, double relax, int backwards )
{
   using namespace hyteg::vertexdof::macrocell::generated;
   if ( backwards )
      sor_3D_macrocell_P1_backwards( dst, rhs, level, toMap( stencil15 ), relax );
   else
      sor_3D_macrocell_P1( dst, rhs, level, toMap( stencil15 ), relax );
}

// nbr[0..5] = #cells at local edges 0..5, nbr[6..9] = faces 0..3, nbr[10..13] = vertices 0..3
void ref_prolongate_cell( const double* coarse, double* fine, int coarseLevel, const double* nbr )
{
   hyteg::vertexdof::macrocell::generated::prolongate_3D_macrocell_P1_push_additive( coarse,
                                                                                     fine,
                                                                                     coarseLevel,
                                                                                     nbr[0],
                                                                                     nbr[1],
                                                                                     nbr[2],
                                                                                     nbr[3],
                                                                                     nbr[4],
                                                                                     nbr[5],
                                                                                     nbr[6],
                                                                                     nbr[7],
                                                                                     nbr[8],
                                                                                     nbr[9],
                                                                                     nbr[10],
                                                                                     nbr[11],
                                                                                     nbr[12],
                                                                                     nbr[13] );
}

void ref_restrict_cell( double* coarse, const double* fine, int coarseLevel, const double* nbr )
{
   hyteg::vertexdof::macrocell::generated::restrict_3D_macrocell_P1_pull_additive( coarse,
                                                                                   fine,
                                                                                   coarseLevel,
                                                                                   nbr[0],
                                                                                   nbr[1],
                                                                                   nbr[2],
                                                                                   nbr[3],
                                                                                   nbr[4],
                                                                                   nbr[5],
                                                                                   nbr[6],
                                                                                   nbr[7],
                                                                                   nbr[8],
                                                                                   nbr[9],
                                                                                   nbr[10],
                                                                                   nbr[11],
                                                                                   nbr[12],
                                                                                   nbr[13] );
}

// Element stiffness of the P1 Laplacian on one tetrahedron; coords = 4 vertices x 3.
void ref_p1_tet_diffusion( const double* coords12, double* A16 )
{
   p1_tet_diffusion_cell_integral_0_otherwise integral;
   integral.tabulate_tensor( A16, nullptr, coords12, 0 );
}

} // extern "C"
